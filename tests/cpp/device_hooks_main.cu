// Driver for the device-hook API (include/mclccd_b200/device_hooks.cuh):
// reads a scene, runs mcl::BVHTree<double, 3> on device arrays, then
//   A: a filter functor (skip stencils whose first vertex is odd) with the
//      library's ACCD on the survivors;
//   B: a custom narrow-phase functor (VF: toi = (first vertex % 5) / 10,
//      EE: no hit) on every candidate.
// Writes nA, nB, then each hit list (int4 stencils, u8 kinds, f64 toi).
#include <cstdio>
#include <vector>

#include "mclccd_b200/device_hooks.cuh"

struct SkipOddFirst {
    __device__ bool operator()(int4 s, bool) const { return (s.x & 1) != 0; }
};

struct VfByVertex {
    __device__ double operator()(int4 s, bool is_vf, const double *, const double *) const
    {
        return is_vf ? (double)(s.x % 5) / 10.0 : -1.0;
    }
};

int main(int argc, char **argv)
{
    if (argc != 3) return 2;
    FILE *f = std::fopen(argv[1], "rb");
    if (!f) return 2;
    int hdr[3];
    double eta;
    if (std::fread(hdr, sizeof(int), 3, f) != 3 || std::fread(&eta, sizeof(double), 1, f) != 1) return 2;
    const int nv = hdr[0], np = hdr[1];
    std::vector<double> V0(3 * (size_t)nv), V1(3 * (size_t)nv);
    std::vector<int> P(3 * (size_t)np);
    if (std::fread(V0.data(), sizeof(double), V0.size(), f) != V0.size() ||
        std::fread(V1.data(), sizeof(double), V1.size(), f) != V1.size() ||
        std::fread(P.data(), sizeof(int), P.size(), f) != P.size())
        return 2;
    std::fclose(f);
    double *dV0, *dV1;
    int *dP;
    cudaMalloc(&dV0, V0.size() * sizeof(double));
    cudaMalloc(&dV1, V1.size() * sizeof(double));
    cudaMalloc(&dP, P.size() * sizeof(int));
    cudaMemcpy(dV0, V0.data(), V0.size() * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(dV1, V1.data(), V1.size() * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(dP, P.data(), P.size() * sizeof(int), cudaMemcpyHostToDevice);

    mcl::BVHTree<double, 3> tree;
    tree.options.box_eta = tree.options.vf_ccd_eta = tree.options.ee_ccd_eta = eta;
    tree.update(dV0, dV1, nv, dP, np, 3, nullptr, MCLCCD_MEM_DEVICE);
    tree.traverse();

    std::vector<int> cs;
    std::vector<unsigned char> cv;
    tree.candidates(cs, cv);
    const long long cap = (long long)cv.size() + 16;
    mcl::b200::DeviceHits out[2];
    for (auto &o : out) {
        cudaMalloc(&o.sten, cap * sizeof(int4));
        cudaMalloc(&o.is_vf, cap);
        cudaMalloc(&o.toi, cap * sizeof(double));
        o.capacity = cap;
    }
    long long n[2];
    n[0] = mcl::b200::apply_device_filter(tree, dV0, dV1, nv, SkipOddFirst{}, out[0]);
    n[1] = mcl::b200::apply_device_hooks(tree, dV0, dV1, mcl::b200::KeepAll{}, VfByVertex{}, out[1]);

    FILE *g = std::fopen(argv[2], "wb");
    if (!g) return 2;
    std::fwrite(n, sizeof(long long), 2, g);
    for (int k = 0; k < 2; ++k) {
        std::vector<int4> s((size_t)n[k]);
        std::vector<unsigned char> v((size_t)n[k]);
        std::vector<double> t((size_t)n[k]);
        cudaMemcpy(s.data(), out[k].sten, n[k] * sizeof(int4), cudaMemcpyDeviceToHost);
        cudaMemcpy(v.data(), out[k].is_vf, n[k], cudaMemcpyDeviceToHost);
        cudaMemcpy(t.data(), out[k].toi, n[k] * sizeof(double), cudaMemcpyDeviceToHost);
        std::fwrite(s.data(), sizeof(int4), s.size(), g);
        std::fwrite(v.data(), 1, v.size(), g);
        std::fwrite(t.data(), sizeof(double), t.size(), g);
    }
    std::fclose(g);
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 1;
}
