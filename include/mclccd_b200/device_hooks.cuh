// Device-side filter_pair / narrow_phase hooks for mcl::BVHTree<double, DIM>.
//
// The reference's std::function hooks filter_pair and narrow_phase
// (include/MCL/BVHTree.hpp:109-119, called per candidate in
// BVHTree.cpp:345-347, 368-370, 393-395) become device functors passed as
// template parameters.  They are applied on the GPU to the candidate
// stencils of the last traverse() and never leave the device.  Header-only:
// include it from a .cu file compiled by nvcc (for sm_100a) and link
// libmclccd_b200.so.
//
//   struct Filter {   // true = skip the stencil (the reference's filter_pair)
//       __device__ bool operator()(int4 sten, bool is_vf) const;
//   };
//   struct Narrow {   // toi of the stencil, < 0 = no hit (the reference's narrow_phase)
//       __device__ double operator()(int4 sten, bool is_vf, const double *V0, const double *V1) const;
//   };
//
//   mcl::BVHTree<double, 3> tree;  tree.update(dV0, dV1, nv, dP, np, 3, nullptr, MCLCCD_MEM_DEVICE);
//   tree.traverse();
//   long long n = mcl::b200::apply_device_hooks(tree, dV0, dV1, Filter{}, Narrow{}, hits);   // custom narrow phase
//   long long m = mcl::b200::apply_device_filter(tree, dV0, dV1, nv, Filter{}, hits);        // library ACCD on survivors
//
// Hits (toi >= 0, as collide() delivers them, BVHTree.cpp:262) are appended
// to caller-owned device arrays in no particular order; more than `capacity`
// hits throws mcl::CCDError(MCLCCD_ERR_OVERFLOW) after writing the first
// `capacity`.  V0/V1 are the device arrays the traverse used.  Functors are
// called concurrently from many threads and must not keep mutable state
// outside their own stencil.
#pragma once

#include "BVHTree.hpp"

#include <cuda_runtime.h>

namespace mcl {
namespace b200 {

// Caller-owned device arrays receiving the hits.
struct DeviceHits {
    int4 *sten = nullptr;
    unsigned char *is_vf = nullptr;
    double *toi = nullptr;
    long long capacity = 0;
};

// Filter that keeps every stencil.
struct KeepAll {
    __device__ bool operator()(int4, bool) const { return false; }
};

namespace detail {

template <class Filter, class Narrow>
__global__ void k_apply_hooks(const int4 *__restrict__ cand, const unsigned char *__restrict__ cand_vf, long long n,
                              const double *__restrict__ V0, const double *__restrict__ V1, Filter filter,
                              Narrow narrow, DeviceHits out, unsigned long long *n_out)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int4 s = cand[i];
        const bool vf = cand_vf[i] != 0;
        if (filter(s, vf)) continue;
        const double toi = narrow(s, vf, V0, V1);
        if (toi >= 0.0) {
            const unsigned long long slot = atomicAdd(n_out, 1ull);
            if ((long long)slot < out.capacity) { out.sten[slot] = s; out.is_vf[slot] = vf ? 1 : 0; out.toi[slot] = toi; }
        }
    }
}

// Compacts the stencils the filter keeps (order preserved within a block's
// stride, not globally; the library ACCD does not depend on order).
template <class Filter>
__global__ void k_apply_filter(const int4 *__restrict__ cand, const unsigned char *__restrict__ cand_vf, long long n,
                               Filter filter, int4 *__restrict__ keep, unsigned char *__restrict__ keep_vf,
                               unsigned long long *n_keep)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int4 s = cand[i];
        const bool vf = cand_vf[i] != 0;
        if (filter(s, vf)) continue;
        const unsigned long long slot = atomicAdd(n_keep, 1ull);
        keep[slot] = s;
        keep_vf[slot] = vf ? 1 : 0;
    }
}

// toi >= 0 hits of the bulk ACCD -> the caller's hit arrays.
static __global__ void k_collect_hits(const int4 *__restrict__ sten, const unsigned char *__restrict__ is_vf,
                                      const double *__restrict__ toi, const int *__restrict__ hit, long long n,
                                      DeviceHits out, unsigned long long *n_out)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        if (!hit[i] || !(toi[i] >= 0.0)) continue;
        const unsigned long long slot = atomicAdd(n_out, 1ull);
        if ((long long)slot < out.capacity) { out.sten[slot] = sten[i]; out.is_vf[slot] = is_vf[i]; out.toi[slot] = toi[i]; }
    }
}

inline void cuda_check(cudaError_t e, const char *what)
{
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw CCDError(e == cudaErrorMemoryAllocation ? MCLCCD_ERR_NOMEM : MCLCCD_ERR_CUDA,
                       std::string(what) + ": " + cudaGetErrorString(e));
    }
}

// Device scratch freed on scope exit.
struct Scratch {
    void *p = nullptr;
    explicit Scratch(size_t bytes) { cuda_check(cudaMalloc(&p, bytes < 16 ? 16 : bytes), "cudaMalloc"); }
    ~Scratch() { cudaFree(p); }
    Scratch(const Scratch &) = delete;
    Scratch &operator=(const Scratch &) = delete;
};

inline int grid_for(long long n) { return (int)(n < 1 ? 1 : (n + 255) / 256 < 148 * 16 ? (n + 255) / 256 : 148 * 16); }

template <int DIM>
long long candidates_on_device(const BVHTree<double, DIM> &tree, Scratch &buf, int4 *&sten, unsigned char *&vf)
{
    long long nvf = 0, nee = 0;
    int rc = mclccd_counts(tree.handle(), nullptr, nullptr, &nvf, &nee, nullptr);
    if (rc != MCLCCD_OK) throw CCDError(rc, mclccd_status_string(rc));
    const long long n = nvf + nee;
    sten = static_cast<int4 *>(buf.p);
    vf = reinterpret_cast<unsigned char *>(sten + n);
    rc = mclccd_get_candidates(tree.handle(), MCLCCD_MEM_DEVICE, n, reinterpret_cast<int *>(sten), vf);
    if (rc != MCLCCD_OK) throw CCDError(rc, mclccd_status_string(rc));
    return n;
}

template <int DIM>
long long candidate_count(const BVHTree<double, DIM> &tree)
{
    long long nvf = 0, nee = 0;
    const int rc = mclccd_counts(tree.handle(), nullptr, nullptr, &nvf, &nee, nullptr);
    if (rc != MCLCCD_OK) throw CCDError(rc, mclccd_status_string(rc));
    return nvf + nee;
}

inline long long finish(unsigned long long *d_count, long long capacity, cudaStream_t st)
{
    unsigned long long n = 0;
    cuda_check(cudaMemcpyAsync(&n, d_count, sizeof(n), cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
    cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
    if ((long long)n > capacity) throw CCDError(MCLCCD_ERR_OVERFLOW, "device hooks: more hits than capacity");
    return (long long)n;
}

} // namespace detail

// Custom narrow phase: for each candidate stencil of the last traverse that
// `filter` keeps, toi = narrow(...); stencils with toi >= 0 are the hits.
// Returns the number of hits.
template <int DIM, class Filter, class Narrow>
long long apply_device_hooks(const BVHTree<double, DIM> &tree, const double *V0, const double *V1, Filter filter,
                             Narrow narrow, DeviceHits out, cudaStream_t stream = nullptr)
{
    const long long n = detail::candidate_count(tree);
    detail::Scratch buf((size_t)n * (sizeof(int4) + 1) + 256);
    detail::Scratch cnt(sizeof(unsigned long long));
    int4 *sten;
    unsigned char *vf;
    detail::candidates_on_device(tree, buf, sten, vf);
    detail::cuda_check(cudaMemsetAsync(cnt.p, 0, sizeof(unsigned long long), stream), "cudaMemsetAsync");
    detail::k_apply_hooks<<<detail::grid_for(n), 256, 0, stream>>>(sten, vf, n, V0, V1, filter, narrow, out,
                                                                   static_cast<unsigned long long *>(cnt.p));
    detail::cuda_check(cudaGetLastError(), "k_apply_hooks");
    return detail::finish(static_cast<unsigned long long *>(cnt.p), out.capacity, stream);
}

// filter_pair only: the library's ACCD (the reference's default narrow
// phase) scores the stencils the filter keeps, with the tree's etas.
template <int DIM, class Filter>
long long apply_device_filter(const BVHTree<double, DIM> &tree, const double *V0, const double *V1, int nv,
                              Filter filter, DeviceHits out, cudaStream_t stream = nullptr)
{
    const long long n = detail::candidate_count(tree);
    detail::Scratch buf((size_t)n * (sizeof(int4) + 1) + 256);
    detail::Scratch keep((size_t)n * (sizeof(int4) + 1 + sizeof(double) + sizeof(int)) + 256);
    detail::Scratch cnt(2 * sizeof(unsigned long long));
    int4 *sten;
    unsigned char *vf;
    detail::candidates_on_device(tree, buf, sten, vf);
    auto *counts = static_cast<unsigned long long *>(cnt.p);
    detail::cuda_check(cudaMemsetAsync(counts, 0, 2 * sizeof(unsigned long long), stream), "cudaMemsetAsync");
    int4 *ks = static_cast<int4 *>(keep.p);
    double *kt = reinterpret_cast<double *>(ks + n);
    int *kh = reinterpret_cast<int *>(kt + n);
    unsigned char *kv = reinterpret_cast<unsigned char *>(kh + n);
    detail::k_apply_filter<<<detail::grid_for(n), 256, 0, stream>>>(sten, vf, n, filter, ks, kv, counts);
    detail::cuda_check(cudaGetLastError(), "k_apply_filter");
    unsigned long long nk = 0;
    detail::cuda_check(cudaMemcpyAsync(&nk, counts, sizeof(nk), cudaMemcpyDeviceToHost, stream), "cudaMemcpyAsync");
    detail::cuda_check(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
    double vf_eta = 0, ee_eta = 0;
    mclccd_get_options(tree.handle(), nullptr, &vf_eta, &ee_eta, nullptr);
    const int rc = mclccd_narrow_phase_bulk(DIM, V0, V1, nv, reinterpret_cast<const int *>(ks), kv, (long long)nk,
                                            vf_eta, ee_eta, kt, kh, MCLCCD_MEM_DEVICE, stream);
    if (rc != MCLCCD_OK) throw CCDError(rc, mclccd_status_string(rc));
    detail::k_collect_hits<<<detail::grid_for((long long)nk), 256, 0, stream>>>(ks, kv, kt, kh, (long long)nk, out,
                                                                                counts + 1);
    detail::cuda_check(cudaGetLastError(), "k_collect_hits");
    return detail::finish(counts + 1, out.capacity, stream);
}

} // namespace b200
} // namespace mcl
