// FP64 ACCD narrow phase over stencil buffers.
//
// Replaces BVHTree::default_narrow_phase (BVHTree.cpp:429-461) ->
// NarrowPhaseACCD::query_ccd_vf/ee -> additive_ccd (NarrowPhase.cpp:609-711).
// One thread per stencil: gather 2 x (DIM+1) vertices, run ACCD, and either
// append hits to the compacted contact buffer (warp-aggregated) or write the
// per-stencil (toi, hit) of the bulk call.  Compiled with -fmad=false.
#include "common.cuh"
#include "ctcd.cuh"
#include "geom.cuh"
#include "kernels.cuh"

namespace mclccd {

template <int DIM>
__device__ __forceinline__ bool gather_stencil(const int *s, const double *__restrict__ V0, const double *__restrict__ V1,
                                               int nv, double (&x0)[DIM + 1][DIM], double (&x1)[DIM + 1][DIM])
{
    bool ok = true;
#pragma unroll
    for (int i = 0; i < DIM + 1; ++i) {
        int v = s[i];
        if (v < 0 || v >= nv) { ok = false; v = 0; }
#pragma unroll
        for (int k = 0; k < DIM; ++k) {
            x0[i][k] = __ldg(V0 + (size_t)v * DIM + k);
            x1[i][k] = __ldg(V1 + (size_t)v * DIM + k);
        }
    }
    return ok;
}

// The reference loop as written, out of line with its own gathers, for the
// rare stencil whose iteration 0 is not an exact no-op (non-finite or -0.0
// coordinates): the callers' arrays stay in registers.  -1 on a miss.
template <int DIM, bool VF>
__device__ __noinline__ double literal_regather(int4 s4, const double *__restrict__ V0, const double *__restrict__ V1,
                                                int nv, double eta, Counters *cnt)
{
    const int s[4] = {s4.x, s4.y, s4.z, s4.w};
    double v0[DIM + 1][DIM], v1[DIM + 1][DIM], toi = -1.0;
    int iters;
    gather_stencil<DIM>(s, V0, V1, nv, v0, v1);
    const int hit = accd_literal<DIM, VF>(v0, v1, eta, toi, iters);
    if (iters >= 1000) atomicOr(&cnt->err, kErrAccdIters);
    return hit ? toi : -1.0;
}

// ACCD of one gathered stencil with the literal path out of line; toi = -1
// on a miss, otherwise the reference's toi.
template <int DIM, bool VF>
__device__ __forceinline__ double accd_stencil(const int4 &s4, const double (&v0)[DIM + 1][DIM],
                                               const double (&v1)[DIM + 1][DIM], const double *__restrict__ V0,
                                               const double *__restrict__ V1, int nv, double eta, Counters *cnt)
{
    double p[DIM + 1][DIM], x[DIM + 1][DIM], l_p, d0, t_l1;
    bool noop;
    accd_setup<DIM, VF, true>(v0, v1, p, x, l_p, noop);
    const int h = accd_head_fast<DIM, VF>(x, l_p, noop, eta, d0, t_l1);
    if (h == kHeadHit) return 0.0;
    if (h == kHeadMiss) return -1.0;
    if (h == kHeadLiteral) return literal_regather<DIM, VF>(s4, V0, V1, nv, eta, cnt);
    double toi = -1.0;
    int iters;
    const int hit = accd_resume<DIM, VF>(x, p, l_p, eta, d0, toi, iters);
    if (iters >= 1000) atomicOr(&cnt->err, kErrAccdIters);
    return hit ? toi : -1.0;
}

// Resident 128-thread blocks per SM the pipeline ACCD kernel is compiled for
// (register cap = 64K / (128 x this)); the kernel is latency-bound, so more
// resident warps beat a few spilled registers.
#ifndef MCLCCD_ACCD_MIN_BLOCKS
#define MCLCCD_ACCD_MIN_BLOCKS 8
#endif

// Pipeline form: stencils from the expansion kernel, count read on device.
template <int DIM, bool VF>
__global__ void __launch_bounds__(128, MCLCCD_ACCD_MIN_BLOCKS)
k_accd_pipeline(const int4 *__restrict__ sten, const unsigned long long *n_ptr, unsigned long long cap,
                const double *__restrict__ V0, const double *__restrict__ V1, int nv, double eta,
                int4 *__restrict__ hit_sten, double *__restrict__ hit_toi, unsigned char *__restrict__ hit_isvf,
                unsigned long long hit_cap, Counters *cnt, const unsigned long long *lo_ptr)
{
    // stencils [lo, n): the whole list, or one query chunk's part of it
    unsigned long long n = *(volatile const unsigned long long *)n_ptr;
    if (n > cap) n = cap;
    const unsigned long long lo = lo_ptr ? min(*(volatile const unsigned long long *)lo_ptr, n) : 0ull;
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long i = lo + (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const int4 s4 = sten[i];
        const int s[4] = {s4.x, s4.y, s4.z, s4.w};
        double x0[DIM + 1][DIM], x1[DIM + 1][DIM];
        if (!gather_stencil<DIM>(s, V0, V1, nv, x0, x1)) { atomicOr(&cnt->err, kErrBadIndex); continue; }
        const double toi = accd_stencil<DIM, VF>(s4, x0, x1, V0, V1, nv, eta, cnt);
        // collide() delivers a hit only when toi >= 0 (BVHTree.cpp:262): a
        // degenerate stencil can report hit == 1 with toi = NaN, which the
        // comparison rejects.
        if (toi >= 0.0) {
            const unsigned long long slot = warp_append(&cnt->n_hits);
            if (slot < hit_cap) {
                hit_sten[slot] = s4;
                hit_toi[slot] = toi;
                hit_isvf[slot] = VF ? 1 : 0;
            }
        }
    }
}

// Re-binned pipeline form: the head of ACCD (setup, first distance,
// immediate hit, the miss decided before iteration 1's distance) runs for
// one stencil per thread; stencils that go on are queued in shared memory
// with their first distance d0 and motion bound l_p, and whenever a full
// block's worth is queued every thread runs the tail of one of them.  A
// warp then runs either heads or tails, never both, so the lanes that miss
// after one distance no longer idle through the others' two or more.  The
// tail rebuilds the exact state entering iteration 1 -- x = v0, toi = 0,
// t_l and g from d0 and l_p, p from a re-gather (setup without the norms)
// -- so (hit, toi) are bit-identical to the unbinned kernel.  A stencil
// whose iteration 0 is not an exact no-op runs its tail in place (rare).
constexpr int kRebinBlock = 128;

template <int DIM, bool VF>
__device__ __forceinline__ void rebin_emit(const int4 &s4, double toi, bool ok, Counters *cnt, int4 *hit_sten,
                                           double *hit_toi, unsigned char *hit_isvf, unsigned long long hit_cap)
{
    if (ok) {
        const unsigned long long slot = warp_append(&cnt->n_hits);
        if (slot < hit_cap) {
            hit_sten[slot] = s4;
            hit_toi[slot] = toi;
            hit_isvf[slot] = VF ? 1 : 0;
        }
    }
}

template <int DIM, bool VF>
__global__ void __launch_bounds__(kRebinBlock, MCLCCD_ACCD_MIN_BLOCKS)
k_accd_rebin(const int4 *__restrict__ sten, const unsigned long long *n_ptr, unsigned long long cap,
             const double *__restrict__ V0, const double *__restrict__ V1, int nv, double eta,
             int4 *__restrict__ hit_sten, double *__restrict__ hit_toi, unsigned char *__restrict__ hit_isvf,
             unsigned long long hit_cap, Counters *cnt, const unsigned long long *lo_ptr)
{
    __shared__ int4 q_sten[2 * kRebinBlock];
    __shared__ double q_d0[2 * kRebinBlock], q_lp[2 * kRebinBlock];
    __shared__ int q_n;
    unsigned long long n = *(volatile const unsigned long long *)n_ptr;
    if (n > cap) n = cap;
    const int tid = threadIdx.x;
    if (tid == 0) q_n = 0;
    __syncthreads();
    const double xx = eta * eta;
    auto tail = [&](int j) {   // tail of queued stencil j
        const int4 s4 = q_sten[j];
        const double d0 = q_d0[j], l_p = q_lp[j];
        const int s[4] = {s4.x, s4.y, s4.z, s4.w};
        double v0[DIM + 1][DIM], v1[DIM + 1][DIM], p[DIM + 1][DIM], x[DIM + 1][DIM], unused;
        bool noop;
        gather_stencil<DIM>(s, V0, V1, nv, v0, v1);   // indices checked by the head
        accd_setup<DIM, VF, false>(v0, v1, p, x, unused, noop);
        const double A = d0 * d0 - xx;
        const double g = (1.0 * A) / (d0 - eta);
        double toi = 0.0;
        int iters;
        const int hit = accd_tail<DIM, VF>(x, p, l_p, eta, g, toi, 0.9 * A / ((d0 + eta) * l_p), iters);
        if (iters >= 1000) atomicOr(&cnt->err, kErrAccdIters);
        return hit && toi >= 0.0 ? toi : -1.0;
    };
    const unsigned long long lo = lo_ptr ? min(*(volatile const unsigned long long *)lo_ptr, n) : 0ull;
    const unsigned long long stride = (unsigned long long)gridDim.x * kRebinBlock;
    for (unsigned long long base = lo + (unsigned long long)blockIdx.x * kRebinBlock; base < n; base += stride) {
        const unsigned long long i = base + tid;
        int4 s4 = make_int4(0, 0, 0, 0);
        double toi = -1.0;
        bool hit = false;
        if (i < n) {
            s4 = sten[i];
            const int s[4] = {s4.x, s4.y, s4.z, s4.w};
            double v0[DIM + 1][DIM], v1[DIM + 1][DIM];
            if (!gather_stencil<DIM>(s, V0, V1, nv, v0, v1)) {
                atomicOr(&cnt->err, kErrBadIndex);
            } else {
                double p[DIM + 1][DIM], x[DIM + 1][DIM], l_p, d0, g, t_l;
                bool noop, skip;
                accd_setup<DIM, VF, true>(v0, v1, p, x, l_p, noop);
                const int h = accd_head<DIM, VF>(x, p, l_p, noop, eta, d0, g, toi, t_l, skip);
                if (h == kHeadHit) {
                    hit = toi >= 0.0;
                } else if (h == kHeadContinue) {
                    if (skip) {
                        const int j = atomicAdd(&q_n, 1);   // < 2 * kRebinBlock: < kRebinBlock held before
                        q_sten[j] = s4;
                        q_d0[j] = d0;
                        q_lp[j] = l_p;
                    } else {
                        int iters;
                        hit = accd_tail<DIM, VF>(x, p, l_p, eta, g, toi, t_l, iters) && toi >= 0.0;
                        if (iters >= 1000) atomicOr(&cnt->err, kErrAccdIters);
                    }
                }
            }
        }
        rebin_emit<DIM, VF>(s4, toi, hit, cnt, hit_sten, hit_toi, hit_isvf, hit_cap);
        __syncthreads();
        const int queued = q_n;
        if (queued >= kRebinBlock) {   // one tail per thread
            const double t = tail(tid);
            rebin_emit<DIM, VF>(q_sten[tid], t, t >= 0.0, cnt, hit_sten, hit_toi, hit_isvf, hit_cap);
            __syncthreads();
            const int left = queued - kRebinBlock;
            int4 ms;
            double md = 0, ml = 0;
            if (tid < left) { ms = q_sten[kRebinBlock + tid]; md = q_d0[kRebinBlock + tid]; ml = q_lp[kRebinBlock + tid]; }
            __syncthreads();
            if (tid < left) { q_sten[tid] = ms; q_d0[tid] = md; q_lp[tid] = ml; }
            if (tid == 0) q_n = left;
            __syncthreads();
        }
    }
    const int queued = q_n;   // last partial bin
    if (tid < queued) {
        const double t = tail(tid);
        rebin_emit<DIM, VF>(q_sten[tid], t, t >= 0.0, cnt, hit_sten, hit_toi, hit_isvf, hit_cap);
    }
}

// Split form (MCLCCD_TUNE_ACCD_REBIN = 2): the head of ACCD in one kernel
// over the whole list, the tail in a second kernel over the stencils that go
// on.  About 40% of a cloth's stencils are decided by their first distance
// and the rest need two more, so in the one-kernel form the lanes of a warp
// wait on each other; here every warp of the head kernel runs one distance
// per lane and every warp of the tail kernel (almost always) two.  The head
// appends (list index, d0, l_p) of each continuing stencil to a queue; the
// tail re-gathers the stencil and its positions, rebuilds the motion exactly
// (setup without the norms) and resumes the reference loop at iteration 1,
// so (hit, toi) are bit-identical to the one-kernel form.
template <int DIM, bool VF>
__global__ void __launch_bounds__(128, MCLCCD_ACCD_MIN_BLOCKS)
k_accd_head(const int4 *__restrict__ sten, const unsigned long long *n_ptr, unsigned long long cap,
            const double *__restrict__ V0, const double *__restrict__ V1, int nv, double eta,
            int4 *__restrict__ hit_sten, double *__restrict__ hit_toi, unsigned char *__restrict__ hit_isvf,
            unsigned long long hit_cap, Counters *cnt, const unsigned long long *lo_ptr, unsigned *__restrict__ q_idx,
            double2 *__restrict__ q_state, unsigned long long *q_count)
{
    unsigned long long n = *(volatile const unsigned long long *)n_ptr;
    if (n > cap) n = cap;
    const unsigned long long lo = lo_ptr ? min(*(volatile const unsigned long long *)lo_ptr, n) : 0ull;
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long i = lo + (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const int4 s4 = sten[i];
        const int s[4] = {s4.x, s4.y, s4.z, s4.w};
        double v0[DIM + 1][DIM], v1[DIM + 1][DIM];
        if (!gather_stencil<DIM>(s, V0, V1, nv, v0, v1)) { atomicOr(&cnt->err, kErrBadIndex); continue; }
        double p[DIM + 1][DIM], x[DIM + 1][DIM], l_p, d0 = 0.0, t_l1;
        bool noop;
        accd_setup<DIM, VF, true>(v0, v1, p, x, l_p, noop);
        const int h = accd_head_fast<DIM, VF>(x, l_p, noop, eta, d0, t_l1);
        double toi = -1.0;
        bool hit = false;
        if (h == kHeadHit) {
            toi = 0.0;
            hit = true;
        } else if (h == kHeadLiteral) {   // iteration 0 is not an exact no-op: the reference loop as written
            toi = literal_regather<DIM, VF>(s4, V0, V1, nv, eta, cnt);
            hit = toi >= 0.0;
        } else if (h == kHeadContinue) {
            const unsigned long long slot = warp_append(q_count);   // < cap: one entry per stencil
            q_idx[slot] = (unsigned)i;
            q_state[slot] = make_double2(d0, l_p);
        }
        if (hit && toi >= 0.0) {   // collide() delivers a hit only when toi >= 0 (BVHTree.cpp:262)
            const unsigned long long slot = warp_append(&cnt->n_hits);
            if (slot < hit_cap) {
                hit_sten[slot] = s4;
                hit_toi[slot] = toi;
                hit_isvf[slot] = VF ? 1 : 0;
            }
        }
    }
}

#ifndef MCLCCD_ACCD_TAIL_MIN_BLOCKS
#define MCLCCD_ACCD_TAIL_MIN_BLOCKS 6
#endif
template <int DIM, bool VF>
__global__ void __launch_bounds__(128, MCLCCD_ACCD_TAIL_MIN_BLOCKS)
k_accd_tail(const int4 *__restrict__ sten, const double *__restrict__ V0, const double *__restrict__ V1, int nv,
            double eta, int4 *__restrict__ hit_sten, double *__restrict__ hit_toi, unsigned char *__restrict__ hit_isvf,
            unsigned long long hit_cap, Counters *cnt, const unsigned *__restrict__ q_idx,
            const double2 *__restrict__ q_state, const unsigned long long *q_count)
{
    const unsigned long long n = *(volatile const unsigned long long *)q_count;
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long j = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) {
        const int4 s4 = sten[q_idx[j]];
        const double2 st = q_state[j];
        const int s[4] = {s4.x, s4.y, s4.z, s4.w};
        double v0[DIM + 1][DIM], v1[DIM + 1][DIM], p[DIM + 1][DIM], x[DIM + 1][DIM], unused;
        bool noop;
        gather_stencil<DIM>(s, V0, V1, nv, v0, v1);   // indices checked by the head
        accd_setup<DIM, VF, false>(v0, v1, p, x, unused, noop);
        double toi = -1.0;
        int iters;
        const int hit = accd_resume<DIM, VF>(x, p, st.y, eta, st.x, toi, iters);
        if (iters >= 1000) atomicOr(&cnt->err, kErrAccdIters);
        if (hit && toi >= 0.0) {
            const unsigned long long slot = warp_append(&cnt->n_hits);
            if (slot < hit_cap) {
                hit_sten[slot] = s4;
                hit_toi[slot] = toi;
                hit_isvf[slot] = VF ? 1 : 0;
            }
        }
    }
}

void launch_accd_split(int dim, bool vf, const int4 *sten, const unsigned long long *n_ptr, unsigned long long cap,
                       const double *V0, const double *V1, int nv, double eta, int4 *hit_sten, double *hit_toi,
                       unsigned char *hit_isvf, unsigned long long hit_cap, Counters *cnt, int grid, unsigned *q_idx,
                       double2 *q_state, unsigned long long *q_count, cudaStream_t st,
                       const unsigned long long *lo_ptr)
{
    cudaMemsetAsync(q_count, 0, sizeof(unsigned long long), st);
#define MCLCCD_SPLIT(D, K)                                                                                         \
    {                                                                                                              \
        k_accd_head<D, K><<<grid, 128, 0, st>>>(sten, n_ptr, cap, V0, V1, nv, eta, hit_sten, hit_toi, hit_isvf,    \
                                                hit_cap, cnt, lo_ptr, q_idx, q_state, q_count);                    \
        k_accd_tail<D, K><<<grid, 128, 0, st>>>(sten, V0, V1, nv, eta, hit_sten, hit_toi, hit_isvf, hit_cap, cnt,  \
                                                q_idx, q_state, q_count);                                          \
    }
    if (dim == 3) {
        if (vf) MCLCCD_SPLIT(3, true) else MCLCCD_SPLIT(3, false)
    } else {
        MCLCCD_SPLIT(2, true)
    }
#undef MCLCCD_SPLIT
}

// One-sided VF narrow phase (CTCD with the wrong-side test): 1 hit, 0 no
// contact, -1 only wrong-side contacts.
template <int DIM>
__device__ __forceinline__ int ctcd_vf(const double (&x0)[DIM + 1][DIM], const double (&x1)[DIM + 1][DIM], double eta,
                                       double &toi)
{
    if constexpr (DIM == 3) return ctcd::query_vf3(x0, x1, eta, toi);
    else return ctcd::query_vf2(x0, x1, toi);
}

// Pipeline form of the one-sided VF narrow phase (vf_one_sided): the VF
// list of the expansion kernel -> compacted hits.
template <int DIM>
__global__ void __launch_bounds__(128)
k_ctcd_pipeline(const int4 *__restrict__ sten, const unsigned long long *n_ptr, unsigned long long cap,
                const double *__restrict__ V0, const double *__restrict__ V1, int nv, double eta,
                int4 *__restrict__ hit_sten, double *__restrict__ hit_toi, unsigned char *__restrict__ hit_isvf,
                unsigned long long hit_cap, Counters *cnt, const unsigned long long *lo_ptr)
{
    unsigned long long n = *(volatile const unsigned long long *)n_ptr;
    if (n > cap) n = cap;
    const unsigned long long lo = lo_ptr ? min(*(volatile const unsigned long long *)lo_ptr, n) : 0ull;
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long i = lo + (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const int4 s4 = sten[i];
        const int s[4] = {s4.x, s4.y, s4.z, s4.w};
        double x0[DIM + 1][DIM], x1[DIM + 1][DIM];
        if (!gather_stencil<DIM>(s, V0, V1, nv, x0, x1)) { atomicOr(&cnt->err, kErrBadIndex); continue; }
        double toi = -1.0;
        // default_narrow_phase keeps ret == 1 only; collide() needs toi >= 0
        if (ctcd_vf<DIM>(x0, x1, eta, toi) == 1 && toi >= 0.0) {
            const unsigned long long slot = warp_append(&cnt->n_hits);
            if (slot < hit_cap) {
                hit_sten[slot] = s4;
                hit_toi[slot] = toi;
                hit_isvf[slot] = 1;
            }
        }
    }
}

// Bulk form: caller-given stencils (int32 x 4 each, any alignment), per-stencil
// outputs in input order.  toi = -1 on a miss, as default_narrow_phase returns.
// ONE_SIDED: VF stencils take the CTCD one-sided narrow phase.
template <int DIM, bool ONE_SIDED>
__global__ void __launch_bounds__(128)
k_accd_bulk(const int *__restrict__ sten, const unsigned char *__restrict__ is_vf, long long n,
            const double *__restrict__ V0, const double *__restrict__ V1, int nv, double vf_eta, double ee_eta,
            double *__restrict__ out_toi, int *__restrict__ out_hit, Counters *cnt)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const int s[4] = {sten[4 * i], sten[4 * i + 1], sten[4 * i + 2], sten[4 * i + 3]};
        double x0[DIM + 1][DIM], x1[DIM + 1][DIM];
        double toi = -1.0;
        int hit = 0, iters = 0;
        if (!gather_stencil<DIM>(s, V0, V1, nv, x0, x1)) {
            atomicOr(&cnt->err, kErrBadIndex);
        } else if (DIM == 3 && !is_vf[i]) {
            hit = accd<DIM, false>(x0, x1, ee_eta, toi, iters);
        } else if (ONE_SIDED) {
            hit = ctcd_vf<DIM>(x0, x1, vf_eta, toi) == 1 ? 1 : 0;
        } else {
            hit = accd<DIM, true>(x0, x1, vf_eta, toi, iters);
        }
        if (iters >= 1000) atomicOr(&cnt->err, kErrAccdIters);
        out_toi[i] = hit ? toi : -1.0;
        out_hit[i] = hit;
    }
}

void launch_accd_pipeline(int dim, bool vf, const int4 *sten, const unsigned long long *n_ptr, unsigned long long cap,
                          const double *V0, const double *V1, int nv, double eta, int4 *hit_sten, double *hit_toi,
                          unsigned char *hit_isvf, unsigned long long hit_cap, Counters *cnt, int grid, bool rebin,
                          cudaStream_t st, const unsigned long long *lo_ptr)
{
    if (rebin) {
        if (dim == 3) {
            if (vf) k_accd_rebin<3, true><<<grid, kRebinBlock, 0, st>>>(sten, n_ptr, cap, V0, V1, nv, eta, hit_sten, hit_toi, hit_isvf, hit_cap, cnt, lo_ptr);
            else k_accd_rebin<3, false><<<grid, kRebinBlock, 0, st>>>(sten, n_ptr, cap, V0, V1, nv, eta, hit_sten, hit_toi, hit_isvf, hit_cap, cnt, lo_ptr);
        } else {
            k_accd_rebin<2, true><<<grid, kRebinBlock, 0, st>>>(sten, n_ptr, cap, V0, V1, nv, eta, hit_sten, hit_toi, hit_isvf, hit_cap, cnt, lo_ptr);
        }
        return;
    }
    if (dim == 3) {
        if (vf) k_accd_pipeline<3, true><<<grid, 128, 0, st>>>(sten, n_ptr, cap, V0, V1, nv, eta, hit_sten, hit_toi, hit_isvf, hit_cap, cnt, lo_ptr);
        else k_accd_pipeline<3, false><<<grid, 128, 0, st>>>(sten, n_ptr, cap, V0, V1, nv, eta, hit_sten, hit_toi, hit_isvf, hit_cap, cnt, lo_ptr);
    } else {
        k_accd_pipeline<2, true><<<grid, 128, 0, st>>>(sten, n_ptr, cap, V0, V1, nv, eta, hit_sten, hit_toi, hit_isvf, hit_cap, cnt, lo_ptr);
    }
}

void launch_accd_bulk(int dim, const int *sten, const unsigned char *is_vf, long long n, const double *V0,
                      const double *V1, int nv, double vf_eta, double ee_eta, double *out_toi, int *out_hit,
                      Counters *cnt, cudaStream_t st, bool vf_one_sided)
{
    if (n <= 0) return;
    long long g = (n + 127) / 128;
    if (g > 148 * 32) g = 148 * 32;
    if (vf_one_sided) {
        if (dim == 3) k_accd_bulk<3, true><<<(int)g, 128, 0, st>>>(sten, is_vf, n, V0, V1, nv, vf_eta, ee_eta, out_toi, out_hit, cnt);
        else k_accd_bulk<2, true><<<(int)g, 128, 0, st>>>(sten, is_vf, n, V0, V1, nv, vf_eta, ee_eta, out_toi, out_hit, cnt);
        return;
    }
    if (dim == 3) k_accd_bulk<3, false><<<(int)g, 128, 0, st>>>(sten, is_vf, n, V0, V1, nv, vf_eta, ee_eta, out_toi, out_hit, cnt);
    else k_accd_bulk<2, false><<<(int)g, 128, 0, st>>>(sten, is_vf, n, V0, V1, nv, vf_eta, ee_eta, out_toi, out_hit, cnt);
}

void launch_ctcd_pipeline(int dim, const int4 *sten, const unsigned long long *n_ptr, unsigned long long cap,
                          const double *V0, const double *V1, int nv, double eta, int4 *hit_sten, double *hit_toi,
                          unsigned char *hit_isvf, unsigned long long hit_cap, Counters *cnt, int grid, cudaStream_t st,
                          const unsigned long long *lo_ptr)
{
    if (dim == 3) k_ctcd_pipeline<3><<<grid, 128, 0, st>>>(sten, n_ptr, cap, V0, V1, nv, eta, hit_sten, hit_toi, hit_isvf, hit_cap, cnt, lo_ptr);
    else k_ctcd_pipeline<2><<<grid, 128, 0, st>>>(sten, n_ptr, cap, V0, V1, nv, eta, hit_sten, hit_toi, hit_isvf, hit_cap, cnt, lo_ptr);
}

} // namespace mclccd
