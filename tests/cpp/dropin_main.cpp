// Drives the C++ drop-in header the way reference code drives mcl::BVHTree:
// update(V0, V1, F) then traverse(V0, V1, F) with append_pair /
// append_discrete collecting into vectors.  Scene in, results out, as raw
// little-endian binaries (written / read by tests/test_cpp_dropin.py).
// A third argument "float" runs mcl::BVHTree<float, 3> on the coordinates
// rounded to float (toi written widened to double); "serial" sets
// options.threaded = false (hooks on the calling thread, in order); "throw"
// makes append_pair throw on its 100th call and exits 3 when traverse()
// rethrows it.
#include "mclccd_b200/BVHTree.hpp"

#include <atomic>
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <stdexcept>
#include <vector>

template <typename T>
int run(const std::vector<double> &V0d, const std::vector<double> &V1d, const std::vector<int> &F, int np, double eta,
        const char *out_path)
{
    const std::vector<T> V0(V0d.begin(), V0d.end()), V1(V1d.begin(), V1d.end());
    mcl::BVHTree<T, 3> tree;
    tree.options.box_eta = tree.options.vf_ccd_eta = tree.options.ee_ccd_eta = (T)eta;
    std::vector<int> hs, ds;
    std::vector<double> ht;
    std::vector<unsigned char> hv;
    std::mutex m;   // append_pair runs on several threads (options.threaded)
    tree.append_pair = [&](const mcl::Stencil &s, bool is_vf, const T &toi) {
        std::lock_guard<std::mutex> g(m);
        for (int i = 0; i < 4; ++i) hs.push_back(s[i]);
        hv.push_back(is_vf ? 1 : 0);
        ht.push_back((double)toi);
    };
    tree.append_discrete = [&](int p0, int p1) { ds.push_back(p0); ds.push_back(p1); return false; };
    try {
        tree.update(V0.data(), V1.data(), F.data(), np, 3);
        tree.traverse(V0.data(), V1.data(), F.data());
    } catch (const mcl::CCDError &e) {
        std::fprintf(stderr, "CCDError %d: %s\n", e.status, e.what());
        return 1;
    }
    FILE *o = std::fopen(out_path, "wb");
    if (!o) return 2;
    int64_t n[2] = {(int64_t)hv.size(), (int64_t)ds.size() / 2};
    std::fwrite(n, 8, 2, o);
    std::fwrite(hs.data(), 4, hs.size(), o);
    std::fwrite(hv.data(), 1, hv.size(), o);
    std::fwrite(ht.data(), 8, ht.size(), o);
    std::fwrite(ds.data(), 4, ds.size(), o);
    std::fclose(o);
    std::printf("hits %lld discrete %lld\n", (long long)n[0], (long long)n[1]);
    return 0;
}

int main(int argc, char **argv)
{
    if (argc != 3 && argc != 4) { std::fprintf(stderr, "usage: %s scene.bin out.bin [float]\n", argv[0]); return 2; }
    FILE *f = std::fopen(argv[1], "rb");
    if (!f) return 2;
    int32_t hdr[3];   // nv, np, dim (== 3)
    double eta;
    if (std::fread(hdr, 4, 3, f) != 3 || std::fread(&eta, 8, 1, f) != 1) return 2;
    const int nv = hdr[0], np = hdr[1];
    std::vector<double> V0(3 * (size_t)nv), V1(3 * (size_t)nv);
    std::vector<int> F(3 * (size_t)np);
    if (std::fread(V0.data(), 8, V0.size(), f) != V0.size() || std::fread(V1.data(), 8, V1.size(), f) != V1.size() ||
        std::fread(F.data(), 4, F.size(), f) != F.size())
        return 2;
    std::fclose(f);
    const char *mode = argc == 4 ? argv[3] : "";
    if (!std::strcmp(mode, "float")) return run<float>(V0, V1, F, np, eta, argv[2]);
    const bool throws = !std::strcmp(mode, "throw");

    mcl::BVHTree<double, 3> tree;
    tree.options.box_eta = tree.options.vf_ccd_eta = tree.options.ee_ccd_eta = eta;
    if (!std::strcmp(mode, "serial")) tree.options.threaded = false;
    std::vector<int> hs, ds;
    std::vector<double> ht;
    std::vector<unsigned char> hv;
    std::mutex m;   // append_pair runs on several threads (options.threaded)
    std::atomic<long long> calls(0);
    tree.append_pair = [&](const mcl::Stencil &s, bool is_vf, const double &toi) {
        if (throws && calls.fetch_add(1) == 99) throw std::runtime_error("hook failed");
        std::lock_guard<std::mutex> g(m);
        for (int i = 0; i < 4; ++i) hs.push_back(s[i]);
        hv.push_back(is_vf ? 1 : 0);
        ht.push_back(toi);
    };
    tree.append_discrete = [&](int p0, int p1) { ds.push_back(p0); ds.push_back(p1); return false; };
    try {
        tree.update(V0.data(), V1.data(), F.data(), np, 3);
        tree.traverse(V0.data(), V1.data(), F.data());
        // again: the hits now stream into the staging sized by the first call
        hs.clear(); hv.clear(); ht.clear(); ds.clear();
        tree.traverse(V0.data(), V1.data(), F.data());
    } catch (const mcl::CCDError &e) {
        std::fprintf(stderr, "CCDError %d: %s\n", e.status, e.what());
        return 1;
    } catch (const std::runtime_error &e) {
        std::fprintf(stderr, "hook exception: %s\n", e.what());
        return 3;
    }
    if (throws) return 4;   // the hook's exception was lost
    FILE *o = std::fopen(argv[2], "wb");
    int64_t n[2] = {(int64_t)hv.size(), (int64_t)ds.size() / 2};
    std::fwrite(n, 8, 2, o);
    std::fwrite(hs.data(), 4, hs.size(), o);
    std::fwrite(hv.data(), 1, hv.size(), o);
    std::fwrite(ht.data(), 8, ht.size(), o);
    std::fwrite(ds.data(), 4, ds.size(), o);
    std::fclose(o);
    std::printf("hits %lld discrete %lld\n", (long long)n[0], (long long)n[1]);
    return 0;
}
