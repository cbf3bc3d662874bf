// Test-oracle stand-in for oneTBB's blocked_range (half-open [begin, end)).
#pragma once
#include <cstddef>

namespace tbb {

template <typename Value>
class blocked_range {
public:
    blocked_range(Value b, Value e, std::size_t grain = 1) : b_(b), e_(e), g_(grain) {}
    Value begin() const { return b_; }
    Value end() const { return e_; }
    std::size_t size() const { return std::size_t(e_ - b_); }
    std::size_t grainsize() const { return g_; }
    bool empty() const { return !(b_ < e_); }
private:
    Value b_, e_;
    std::size_t g_;
};

} // namespace tbb
