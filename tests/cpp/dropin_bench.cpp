// End-to-end timing through the C++ drop-in, as reference code uses it:
// mcl::BVHTree<double, 3> with append_pair / append_discrete hooks set,
// update(V0, V1, F, nf, 3) and traverse(V0, V1, F) on host arrays every
// step (the reference's signatures, BVHTree.hpp:81-86), V1 alternating
// between two draws.  Each step's wall time covers the host-to-device copies,
// the device step, the copy of every hit back and the hook calls.
//
//   dropin_bench scene.bin warmup steps
// scene.bin: int32 nv, nf; f64 eta; nv x 3 f64 V0, V1a, V1b; nf x 3 int32 F.
// Prints one JSON object: per-step ms, hits and discrete pairs delivered.
// options.threaded is on (the reference's default), so append_pair runs on
// several host threads; the hook counts into thread-local accumulators that
// each dispatch thread adds to the totals when it ends.
#include "mclccd_b200/BVHTree.hpp"

#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <vector>

namespace {
std::mutex g_m;
long long g_hits = 0;
double g_toi = 0;
struct Acc {
    long long hits = 0;
    double toi = 0;
    void flush()
    {
        std::lock_guard<std::mutex> g(g_m);
        g_hits += hits;
        g_toi += toi;
        hits = 0;
        toi = 0;
    }
    ~Acc() { flush(); }
};
thread_local Acc t_acc;
} // namespace

int main(int argc, char **argv)
{
    if (argc != 4) return 2;
    const int warmup = std::atoi(argv[2]), steps = std::atoi(argv[3]);
    FILE *f = std::fopen(argv[1], "rb");
    if (!f) return 2;
    int hdr[2];
    double eta = 0;
    if (std::fread(hdr, sizeof(int), 2, f) != 2 || std::fread(&eta, sizeof(double), 1, f) != 1) return 2;
    const int nv = hdr[0], nf = hdr[1];
    std::vector<double> V0(3 * (size_t)nv), V1a(3 * (size_t)nv), V1b(3 * (size_t)nv);
    std::vector<int> F(3 * (size_t)nf);
    for (auto *v : {&V0, &V1a, &V1b})
        if (std::fread(v->data(), sizeof(double), v->size(), f) != v->size()) return 2;
    if (std::fread(F.data(), sizeof(int), F.size(), f) != F.size()) return 2;
    std::fclose(f);

    mcl::BVHTree<double, 3> tree;
    tree.options.box_eta = tree.options.vf_ccd_eta = tree.options.ee_ccd_eta = eta;
    long long hits = 0, disc = 0;
    double toi_sum = 0;
    tree.append_pair = [](const mcl::Stencil &, bool, const double &toi) {
        ++t_acc.hits;
        t_acc.toi += toi;
    };
    tree.append_discrete = [&](int, int) -> bool { ++disc; return false; };
    tree.update(V0.data(), V1a.data(), F.data(), nf, 3);   // first update: full build, untimed
    const double *V1s[2] = {V1b.data(), V1a.data()};
    std::vector<double> ms;
    long long last_hits = 0, last_disc = 0;
    for (int i = 0; i < warmup + steps; ++i) {
        const double *V1 = V1s[i % 2];
        disc = 0;
        g_hits = 0;
        g_toi = 0;
        const auto t0 = std::chrono::steady_clock::now();
        tree.update(V0.data(), V1, F.data(), nf, 3);
        tree.traverse(V0.data(), V1, F.data());
        t_acc.flush();   // this thread's share (the others flushed as they ended)
        const auto t1 = std::chrono::steady_clock::now();
        hits = g_hits;
        toi_sum = g_toi;
        if (i >= warmup) ms.push_back(std::chrono::duration<double, std::milli>(t1 - t0).count());
        last_hits = hits;
        last_disc = disc;
    }
    std::printf("{\"ms\": [");
    for (size_t i = 0; i < ms.size(); ++i) std::printf("%s%.4f", i ? ", " : "", ms[i]);
    std::printf("], \"hits\": %lld, \"discrete\": %lld, \"toi_sum\": %.17g}\n", last_hits, last_disc, toi_sum);
    return 0;
}
