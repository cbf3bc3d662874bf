// FP32-certified ACCD narrow phase.
//
// Same answers as the FP64 path -- hit/miss identical, toi bit-identical for
// every stencil that stops at ACCD's second distance test (the common case),
// otherwise never later than the FP64 toi and within 1e-6 relative of it --
// with the iterations after the first in FP32.  Per stencil:
//   * the head runs in FP64 exactly as the reference does (NarrowPhase.cpp:
//     647-683): relative motion p, l_p, the first distance d0, g and the
//     first step L1.  That decides "no motion", "already within eta" and the
//     miss at iteration 1 exactly, and makes the toi of a stencil that stops
//     at iteration 2 the exact FP64 value L1;
//   * iterations k >= 1 run in FP32 on an interval [s_lo, s_hi] that contains
//     the exact sum s_k = L1 + ... + Lk of the FP64 steps.  The iterate
//     x0 + s p is evaluated in a frame that moves with the stencil's first
//     vertex (distances are translation-invariant), so its FP32 coordinates
//     stay at the stencil's size.  The distance over the interval follows
//     from one FP32 evaluation at the midpoint: the distance is
//     l_p-Lipschitz in s (two points of the two primitives separate at most
//     at |p_a| + |p_b| <= l_p);
//   * each FP32 distance is a rigorous bracket [lo, hi] on the value the
//     reference's FP64 routine returns: hi from explicit points of the
//     primitives, lo from the support function along the computed
//     separation, widened by every rounding (FP32 evaluation, FP32 inputs,
//     FP64 iterate accumulation) and by DELTA64 = 2^-36 S, the allowance for
//     how far the FP64 evaluation of a well-conditioned closest-point problem
//     sits from the exact distance (S = coordinate magnitude).  That
//     allowance is the one assumption; triangles with sin^2 of an angle below
//     2^-10 go to FP64.  Where the FP64 routine's own branch choice is
//     uncertain the bracket is the union over every branch it can take: the
//     reference's point_on_triangle returns a point off the closest one in
//     one branch (Projection.hpp:131, s = -e/c on edge e0), and edge_to_edge
//     on near-parallel edges returns the distance for some s in an interval
//     that the FP32 error bounds give (Projection.hpp:242-302);
//   * ACCD's decisions (break when eps < g, miss when toi > 1) are taken only
//     when the brackets decide them.  Anything undecided is queued and a
//     second kernel runs the exact FP64 ACCD on the queue, so FP64 work does
//     not stall the warps of the FP32 pass.
// Compiled with -fmad=false like the FP64 units (the FP64 head and the queue
// pass must stay bit-exact); the FP32 bounds hold with or without
// contraction, and the FP32 dot products use explicit fused multiply-adds.
#include "common.cuh"
#include "geom.cuh"
#include "kernels.cuh"
#include "cert.cuh"

namespace mclccd {

// FP32 pass over one stencil list: certified hits are appended, undecided
// stencils are queued (by index) for the FP64 pass.
#ifndef MCLCCD_CERT_MIN_BLOCKS
#define MCLCCD_CERT_MIN_BLOCKS 4
#endif

template <int DIM, bool VF>
__global__ void __launch_bounds__(128, MCLCCD_CERT_MIN_BLOCKS)
k_accd_certified(const int4 *__restrict__ sten, const unsigned long long *n_ptr, unsigned long long cap,
                 const double *__restrict__ V0, const double *__restrict__ V1, int nv, double eta,
                 int4 *__restrict__ hit_sten, double *__restrict__ hit_toi, unsigned char *__restrict__ hit_isvf,
                 unsigned long long hit_cap, unsigned *__restrict__ queue, Counters *cnt)
{
    unsigned long long n = *(volatile const unsigned long long *)n_ptr;
    if (n > cap) n = cap;
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const int4 s4 = sten[i];
        const int s[4] = {s4.x, s4.y, s4.z, s4.w};
        double x0[DIM + 1][DIM], x1[DIM + 1][DIM];
        if (!gather_c<DIM>(s, V0, V1, nv, x0, x1)) { atomicOr(&cnt->err, kErrBadIndex); continue; }
        double toi = -1.0;
        bool bound;
        const int c = accd_certified<DIM, VF>(x0, x1, eta, toi, bound);
        if (c == kCertFallback) {
            const unsigned long long q = warp_append(&cnt->n_fp64[VF ? 0 : 1]);
            if (q < cap) queue[q] = (unsigned)i;
        } else if (c == kCertHit && toi >= 0.0) {
            if (bound) atomicAdd(&cnt->n_bound_toi, 1ull);
            const unsigned long long slot = warp_append(&cnt->n_hits);
            if (slot < hit_cap) { hit_sten[slot] = s4; hit_toi[slot] = toi; hit_isvf[slot] = VF ? 1 : 0; }
        }
    }
}

// FP64 pass: the exact ACCD on the queued stencils.
template <int DIM, bool VF>
__global__ void __launch_bounds__(128, 8)
k_accd_queue(const int4 *__restrict__ sten, const unsigned *__restrict__ queue, const unsigned long long *q_ptr,
             unsigned long long cap, const double *__restrict__ V0, const double *__restrict__ V1, int nv, double eta,
             int4 *__restrict__ hit_sten, double *__restrict__ hit_toi, unsigned char *__restrict__ hit_isvf,
             unsigned long long hit_cap, Counters *cnt)
{
    unsigned long long n = *(volatile const unsigned long long *)q_ptr;
    if (n > cap) n = cap;
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long j = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) {
        const unsigned i = queue[j];
        if (i >= cap) { atomicOr(&cnt->err, kErrBadIndex); continue; }
        const int4 s4 = sten[i];
        const int s[4] = {s4.x, s4.y, s4.z, s4.w};
        double x0[DIM + 1][DIM], x1[DIM + 1][DIM];
        if (!gather_c<DIM>(s, V0, V1, nv, x0, x1)) { atomicOr(&cnt->err, kErrBadIndex); continue; }
        double toi = -1.0;
        int iters;
        const int hit = accd<DIM, VF>(x0, x1, eta, toi, iters);
        if (iters >= 1000) atomicOr(&cnt->err, kErrAccdIters);
        if (hit && toi >= 0.0) {
            const unsigned long long slot = warp_append(&cnt->n_hits);
            if (slot < hit_cap) { hit_sten[slot] = s4; hit_toi[slot] = toi; hit_isvf[slot] = VF ? 1 : 0; }
        }
    }
}

template <int DIM>
__global__ void __launch_bounds__(128)
k_accd_certified_bulk(const int *__restrict__ sten, const unsigned char *__restrict__ is_vf, long long n,
                      const double *__restrict__ V0, const double *__restrict__ V1, int nv, double vf_eta,
                      double ee_eta, double *__restrict__ out_toi, int *__restrict__ out_hit,
                      long long *__restrict__ queue, Counters *cnt)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const int s[4] = {sten[4 * i], sten[4 * i + 1], sten[4 * i + 2], sten[4 * i + 3]};
        double x0[DIM + 1][DIM], x1[DIM + 1][DIM];
        double toi = -1.0;
        bool bound = false;
        int c = kCertMiss;
        if (!gather_c<DIM>(s, V0, V1, nv, x0, x1)) atomicOr(&cnt->err, kErrBadIndex);
        else if (DIM == 3 && !is_vf[i]) c = accd_certified<DIM, false>(x0, x1, ee_eta, toi, bound);
        else c = accd_certified<DIM, true>(x0, x1, vf_eta, toi, bound);
        if (c == kCertFallback) {
            const unsigned long long q = warp_append(&cnt->n_fp64[0]);
            if (q < (unsigned long long)n) queue[q] = i;
            continue;
        }
        if (c == kCertHit && bound) atomicAdd(&cnt->n_bound_toi, 1ull);
        out_toi[i] = c == kCertHit ? toi : -1.0;
        out_hit[i] = c == kCertHit;
    }
}

template <int DIM>
__global__ void __launch_bounds__(128)
k_accd_queue_bulk(const int *__restrict__ sten, const unsigned char *__restrict__ is_vf, long long n,
                  const long long *__restrict__ queue, const unsigned long long *q_ptr, const double *__restrict__ V0,
                  const double *__restrict__ V1, int nv, double vf_eta, double ee_eta, double *__restrict__ out_toi,
                  int *__restrict__ out_hit, Counters *cnt)
{
    long long m = (long long)*(volatile const unsigned long long *)q_ptr;
    if (m > n) m = n;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < m; j += stride) {
        const long long i = queue[j];
        if (i < 0 || i >= n) { atomicOr(&cnt->err, kErrBadIndex); continue; }
        const int s[4] = {sten[4 * i], sten[4 * i + 1], sten[4 * i + 2], sten[4 * i + 3]};
        double x0[DIM + 1][DIM], x1[DIM + 1][DIM];
        double toi = -1.0;
        int hit = 0, iters = 0;
        if (!gather_c<DIM>(s, V0, V1, nv, x0, x1)) atomicOr(&cnt->err, kErrBadIndex);
        else if (DIM == 3 && !is_vf[i]) hit = accd<DIM, false>(x0, x1, ee_eta, toi, iters);
        else hit = accd<DIM, true>(x0, x1, vf_eta, toi, iters);
        if (iters >= 1000) atomicOr(&cnt->err, kErrAccdIters);
        out_toi[i] = hit ? toi : -1.0;
        out_hit[i] = hit;
    }
}

void launch_accd_certified(int dim, bool vf, const int4 *sten, const unsigned long long *n_ptr,
                           unsigned long long cap, const double *V0, const double *V1, int nv, double eta,
                           int4 *hit_sten, double *hit_toi, unsigned char *hit_isvf, unsigned long long hit_cap,
                           unsigned *queue, Counters *cnt, int grid, cudaStream_t st)
{
    const unsigned long long *q_ptr = &cnt->n_fp64[vf ? 0 : 1];
    if (dim == 3 && vf) {
        k_accd_certified<3, true><<<grid, 128, 0, st>>>(sten, n_ptr, cap, V0, V1, nv, eta, hit_sten, hit_toi, hit_isvf, hit_cap, queue, cnt);
        k_accd_queue<3, true><<<grid, 128, 0, st>>>(sten, queue, q_ptr, cap, V0, V1, nv, eta, hit_sten, hit_toi, hit_isvf, hit_cap, cnt);
    } else if (dim == 3) {
        k_accd_certified<3, false><<<grid, 128, 0, st>>>(sten, n_ptr, cap, V0, V1, nv, eta, hit_sten, hit_toi, hit_isvf, hit_cap, queue, cnt);
        k_accd_queue<3, false><<<grid, 128, 0, st>>>(sten, queue, q_ptr, cap, V0, V1, nv, eta, hit_sten, hit_toi, hit_isvf, hit_cap, cnt);
    } else {
        k_accd_certified<2, true><<<grid, 128, 0, st>>>(sten, n_ptr, cap, V0, V1, nv, eta, hit_sten, hit_toi, hit_isvf, hit_cap, queue, cnt);
        k_accd_queue<2, true><<<grid, 128, 0, st>>>(sten, queue, q_ptr, cap, V0, V1, nv, eta, hit_sten, hit_toi, hit_isvf, hit_cap, cnt);
    }
}

void launch_accd_certified_bulk(int dim, const int *sten, const unsigned char *is_vf, long long n, const double *V0,
                                const double *V1, int nv, double vf_eta, double ee_eta, double *out_toi, int *out_hit,
                                long long *queue, Counters *cnt, cudaStream_t st)
{
    if (n <= 0) return;
    long long g = (n + 127) / 128;
    if (g > 148 * 32) g = 148 * 32;
    const unsigned long long *q_ptr = &cnt->n_fp64[0];
    if (dim == 3) {
        k_accd_certified_bulk<3><<<(int)g, 128, 0, st>>>(sten, is_vf, n, V0, V1, nv, vf_eta, ee_eta, out_toi, out_hit, queue, cnt);
        k_accd_queue_bulk<3><<<(int)g, 128, 0, st>>>(sten, is_vf, n, queue, q_ptr, V0, V1, nv, vf_eta, ee_eta, out_toi, out_hit, cnt);
    } else {
        k_accd_certified_bulk<2><<<(int)g, 128, 0, st>>>(sten, is_vf, n, V0, V1, nv, vf_eta, ee_eta, out_toi, out_hit, queue, cnt);
        k_accd_queue_bulk<2><<<(int)g, 128, 0, st>>>(sten, is_vf, n, queue, q_ptr, V0, V1, nv, vf_eta, ee_eta, out_toi, out_hit, cnt);
    }
}

} // namespace mclccd
