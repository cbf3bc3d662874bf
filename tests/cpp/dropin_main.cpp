// Drives the C++ drop-in header the way reference code drives mcl::BVHTree:
// update(V0, V1, F) then traverse(V0, V1, F) with append_pair /
// append_discrete collecting into vectors.  Scene in, results out, as raw
// little-endian binaries (written / read by tests/test_cpp_dropin.py).
#include "mclccd_b200/BVHTree.hpp"

#include <cstdio>
#include <cstdint>
#include <vector>

int main(int argc, char **argv)
{
    if (argc != 3) { std::fprintf(stderr, "usage: %s scene.bin out.bin\n", argv[0]); return 2; }
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

    mcl::BVHTree<double, 3> tree;
    tree.options.box_eta = tree.options.vf_ccd_eta = tree.options.ee_ccd_eta = eta;
    std::vector<int> hs, ds;
    std::vector<double> ht;
    std::vector<unsigned char> hv;
    tree.append_pair = [&](const mcl::Stencil &s, bool is_vf, const double &toi) {
        for (int i = 0; i < 4; ++i) hs.push_back(s[i]);
        hv.push_back(is_vf ? 1 : 0);
        ht.push_back(toi);
    };
    tree.append_discrete = [&](int p0, int p1) { ds.push_back(p0); ds.push_back(p1); return false; };
    try {
        tree.update(V0.data(), V1.data(), F.data(), np, 3);
        tree.traverse(V0.data(), V1.data(), F.data());
    } catch (const mcl::CCDError &e) {
        std::fprintf(stderr, "CCDError %d: %s\n", e.status, e.what());
        return 1;
    }
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
