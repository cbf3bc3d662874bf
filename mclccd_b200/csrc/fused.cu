// Leaf pairs -> candidate stencils -> discrete test -> ACCD, in one kernel.
//
// Replaces the expansion kernel plus the two ACCD launches of the FP64 path
// (get_candidates BVHTree.cpp:305-398, default_discrete_test :464-500,
// default_narrow_phase :429-461 -> NarrowPhaseACCD::additive_ccd
// NarrowPhase.cpp:634-711) without writing the candidate lists to memory.
//
// Work is warp-local.  A warp takes 32 leaf pairs (one per lane), runs the
// discrete test on them and expands their stencils into two queues in
// shared memory, one per kind (VF, EE), so that every ACCD batch runs 32
// stencils of one kind on 32 lanes:
//   * head batch: gather, relative motion, l_p, first distance.  A stencil
//     is decided here when it has no relative motion, starts within eta, or
//     its first conservative step already leaves the time step (about 40%
//     of the candidates of a cloth); otherwise it goes to the kind's tail
//     queue with its first distance and l_p;
//   * tail batch: 32 queued stencils resume the reference loop at
//     iteration 1 (the positions and motion are gathered again).
// So lanes that stop after one distance never wait for lanes that need
// three.  Queues hold 64 entries; a batch runs whenever 32 are waiting, and
// a warp drains what is left when it runs out of pairs.
//
// Results are the reference's bit for bit (the same functions as the
// stencil-list kernels, geom.cuh); hits reach the contact buffer in another
// order.  The candidate lists are not materialised: their counts are kept,
// and mclccd_get_candidates rebuilds them from the leaf pairs on request.
#include "common.cuh"
#include "geom.cuh"
#include "kernels.cuh"
#include "lbvh.cuh"

namespace mclccd {

namespace {

constexpr int kWarps = 4;    // warps per block
constexpr int kQ = 64;       // queue entries per warp and kind

struct __align__(16) TailEntry {
    int4 s;
    double d0, l_p;
};

template <int DIM>
__device__ __forceinline__ bool fgather(const int4 &s4, const double *__restrict__ V0, const double *__restrict__ V1,
                                        int nv, double (&x0)[DIM + 1][DIM], double (&x1)[DIM + 1][DIM])
{
    const int s[4] = {s4.x, s4.y, s4.z, s4.w};
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

// The reference loop as written, out of line: only stencils whose
// iteration 0 is not an exact no-op (non-finite or -0.0 coordinates) take it.
// It gathers its own inputs, so the caller's arrays stay in registers.
template <int DIM, bool VF>
__device__ __noinline__ double literal_accd(int4 s4, const double *__restrict__ V0, const double *__restrict__ V1,
                                            int nv, double eta, Counters *cnt)
{
    double v0[DIM + 1][DIM], v1[DIM + 1][DIM], toi = -1.0;
    int iters;
    fgather<DIM>(s4, V0, V1, nv, v0, v1);
    const int hit = accd_literal<DIM, VF>(v0, v1, eta, toi, iters);
    if (iters >= 1000) atomicOr(&cnt->err, kErrAccdIters);
    return hit ? toi : -1.0;
}

// Discrete test of one leaf pair at V1 (default_discrete_test,
// BVHTree.cpp:464-500), out of line with its own gathers.
template <int DIM>
__device__ __noinline__ int discrete_pair(int a0, int a1, int a2, int b0, int b1, int b2,
                                          const double *__restrict__ V1)
{
    const int fa[3] = {a0, a1, a2}, fb[3] = {b0, b1, b2};
    double A[DIM][DIM], B[DIM][DIM];
#pragma unroll
    for (int i = 0; i < DIM; ++i)
#pragma unroll
        for (int k = 0; k < DIM; ++k) {
            A[i][k] = __ldg(V1 + (size_t)fa[i] * DIM + k);
            B[i][k] = __ldg(V1 + (size_t)fb[i] * DIM + k);
        }
    if constexpr (DIM == 3) return tri_tri(A[0], A[1], A[2], B[0], B[1], B[2]);
    else return seg_seg(A[0], A[1], B[0], B[1]);
}

struct Out {
    const double *V0, *V1;
    int nv;
    int4 *hit_sten;
    double *hit_toi;
    unsigned char *hit_isvf;
    unsigned long long hit_cap;
    Counters *cnt;
};

// collide() delivers a hit only when toi >= 0 (BVHTree.cpp:262).
template <bool VF>
__device__ __forceinline__ void emit(const Out &o, const int4 &s4, double toi)
{
    if (toi >= 0.0) {
        const unsigned long long slot = warp_append(&o.cnt->n_hits);
        if (slot < o.hit_cap) {
            o.hit_sten[slot] = s4;
            o.hit_toi[slot] = toi;
            o.hit_isvf[slot] = VF ? 1 : 0;
        }
    }
}

// Tails of entries [first, first + take) (take <= 32) of a tail queue;
// called by the whole warp.  Out of line: the batch functions each get the
// kernel's registers to themselves.
template <int DIM, bool VF>
__device__ __noinline__ void tail_batch(Out o, double eta, const TailEntry *tq, int first, int take)
{
    const int lane = (int)lane_id();
    if (lane < take) {
        const TailEntry e = tq[first + lane];
        double v0[DIM + 1][DIM], v1[DIM + 1][DIM], p[DIM + 1][DIM], x[DIM + 1][DIM], unused;
        bool noop;
        fgather<DIM>(e.s, o.V0, o.V1, o.nv, v0, v1);   // indices checked by the head
        accd_setup<DIM, VF, false>(v0, v1, p, x, unused, noop);
        double toi = -1.0;
        int iters;
        const int hit = accd_resume<DIM, VF>(x, p, e.l_p, eta, e.d0, toi, iters);
        if (iters >= 1000) atomicOr(&o.cnt->err, kErrAccdIters);
        if (hit) emit<VF>(o, e.s, toi);
    }
    __syncwarp();
}

// Heads of the first `take` (<= 32) entries of a head queue; stencils that
// go on are appended to the tail queue at nt.  Returns the new tail count.
template <int DIM, bool VF>
__device__ __noinline__ int head_batch(Out o, double eta, const int4 *hq, int take, TailEntry *tq, int nt)
{
    const int lane = (int)lane_id();
    bool go_on = false;
    int4 s4 = make_int4(0, 0, 0, 0);
    double d0 = 0.0, l_p = 0.0;
    if (lane < take) {
        s4 = hq[lane];
        double v0[DIM + 1][DIM], v1[DIM + 1][DIM];
        if (!fgather<DIM>(s4, o.V0, o.V1, o.nv, v0, v1)) {
            atomicOr(&o.cnt->err, kErrBadIndex);
        } else {
            double p[DIM + 1][DIM], x[DIM + 1][DIM], t_l1;
            bool noop;
            accd_setup<DIM, VF, true>(v0, v1, p, x, l_p, noop);
            const int h = accd_head_fast<DIM, VF>(x, l_p, noop, eta, d0, t_l1);
            if (h == kHeadHit) {
                emit<VF>(o, s4, 0.0);
            } else if (h == kHeadContinue) {
                go_on = true;
            } else if (h == kHeadLiteral) {   // iteration 0 is not an exact no-op: the reference loop as written
                const double toi = literal_accd<DIM, VF>(s4, o.V0, o.V1, o.nv, eta, o.cnt);
                if (toi >= 0.0) emit<VF>(o, s4, toi);
            }
        }
    }
    const unsigned ballot = __ballot_sync(0xffffffffu, go_on);
    if (go_on) tq[nt + __popc(ballot & lanemask_lt())] = TailEntry{s4, d0, l_p};
    __syncwarp();
    return nt + __popc(ballot);
}

// A head batch of the queue's `take` entries, then a tail batch if 32 wait.
template <int DIM, bool VF>
__device__ __forceinline__ void run_heads(const Out &o, double eta, const int4 *hq, int &nh, int take, TailEntry *tq,
                                          int &nt)
{
    nt = head_batch<DIM, VF>(o, eta, hq, take, tq, nt);
    nh -= take;
    if (nt >= 32) {
        tail_batch<DIM, VF>(o, eta, tq, nt - 32, 32);
        nt -= 32;
    }
}

// Per-warp expansion state of the current 32 leaf pairs: faces, the stencil
// bits of each kind, and the exclusive prefix of one kind's counts.
template <int DIM>
struct WarpPairs {
    int fa[32][DIM], fb[32][DIM];
    unsigned bits[2][32];   // [0] VF bits (a->b slot i = bit i, b->a slot i = bit 3 + i), [1] EE bits (3i + j)
    int pre[32];
};

// Stencils 0 .. total-1 of one kind of the warp's 32 pairs, in lane order,
// generated 32 - nh at a time into the head queue (so it never holds more
// than 32): output position k belongs to the last lane l with pre[l] <= k,
// as that lane's (k - pre[l])-th set bit.  Warp-uniform; the pairs' data is
// read from shared memory, so little is live while the ACCD batches run.
template <int DIM, bool VF>
__device__ __forceinline__ void generate(const Out &o, double eta, const WarpPairs<DIM> &wp, int total, int4 *hq,
                                         int &nh, TailEntry *tq, int &nt)
{
    const int lane = (int)lane_id();
    for (int k = 0; k < total;) {
        const int chunk = min(32 - nh, total - k);
        if (lane < chunk) {
            const int pos = k + lane;
            int l = 0;   // l + step stays <= 31
#pragma unroll
            for (int step = 16; step; step >>= 1)
                if (wp.pre[l + step] <= pos) l += step;
            unsigned m = wp.bits[VF ? 0 : 1][l];
            for (int r = pos - wp.pre[l]; r > 0; --r) m &= m - 1;
            const int b = __ffs(m) - 1;
            int4 st;
            if constexpr (VF) {
                const int *vs = b < 3 ? wp.fa[l] : wp.fb[l];
                const int *fs = b < 3 ? wp.fb[l] : wp.fa[l];
                st = make_int4(vs[b % 3], fs[0], fs[1], DIM == 3 ? fs[DIM - 1] : -1);
            } else {
                const int i = b / 3, j = b % 3;
                st = make_int4(wp.fa[l][i], wp.fa[l][(i + 1) % 3], wp.fb[l][j], wp.fb[l][(j + 1) % 3]);
            }
            hq[nh + lane] = st;
        }
        nh += chunk;
        k += chunk;
        __syncwarp();
        if (nh == 32) run_heads<DIM, VF>(o, eta, hq, nh, 32, tq, nt);
    }
}

// Exclusive prefix of this lane's count c into wp.pre; returns the total.
template <int DIM>
__device__ __forceinline__ int warp_prefix(WarpPairs<DIM> &wp, unsigned c)
{
    unsigned incl = c;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const unsigned v = __shfl_up_sync(0xffffffffu, incl, off);
        if ((int)lane_id() >= off) incl += v;
    }
    wp.pre[lane_id()] = (int)(incl - c);
    __syncwarp();
    return (int)__shfl_sync(0xffffffffu, incl, 31);
}

template <int DIM, bool VF>
__device__ __forceinline__ void drain(const Out &o, double eta, int4 *hq, int &nh, TailEntry *tq, int &nt)
{
    if (nh > 0) run_heads<DIM, VF>(o, eta, hq, nh, nh, tq, nt);
    while (nt > 0) {
        const int take = min(nt, 32);
        tail_batch<DIM, VF>(o, eta, tq, nt - take, take);
        nt -= take;
    }
}

} // namespace

#ifndef MCLCCD_FUSED_MIN_BLOCKS
#define MCLCCD_FUSED_MIN_BLOCKS 6
#endif

template <int DIM>
__global__ void __launch_bounds__(kWarps * 32, MCLCCD_FUSED_MIN_BLOCKS)
k_narrow_fused(const int2 *__restrict__ pairs, unsigned long long pair_cap, const int *__restrict__ P,
               const unsigned char *__restrict__ flags, const double *__restrict__ V0, const double *__restrict__ V1,
               int nv, double vf_eta, double ee_eta, int continuous, int discrete, int2 *__restrict__ disc,
               unsigned long long disc_cap, int4 *__restrict__ hit_sten, double *__restrict__ hit_toi,
               unsigned char *__restrict__ hit_isvf, unsigned long long hit_cap, Counters *cnt,
               const unsigned long long *lo_ptr, const unsigned long long *hi_ptr)
{
    constexpr int K = DIM == 3 ? 2 : 1;
    __shared__ int4 s_head[K][kWarps][32];
    __shared__ TailEntry s_tail[K][kWarps][kQ];
    __shared__ WarpPairs<DIM> s_pairs[kWarps];
    const int w = threadIdx.x >> 5;
    const int lane = (int)lane_id();
    const Out o{V0, V1, nv, hit_sten, hit_toi, hit_isvf, hit_cap, cnt};
    WarpPairs<DIM> &wp = s_pairs[w];
    int4 *hq_vf = s_head[0][w];
    TailEntry *tq_vf = s_tail[0][w];
    int4 *hq_ee = s_head[K - 1][w];
    TailEntry *tq_ee = s_tail[K - 1][w];
    int nh_vf = 0, nt_vf = 0, nh_ee = 0, nt_ee = 0;
    unsigned long long sum_vf = 0, sum_ee = 0;

    // pairs [lo, hi): the whole list, or one query chunk's part of it
    unsigned long long n = *(volatile const unsigned long long *)hi_ptr;
    if (n > pair_cap) n = pair_cap;
    unsigned long long lo = lo_ptr ? *(volatile const unsigned long long *)lo_ptr : 0ull;
    if (lo > n) lo = n;
    const unsigned long long stride = (unsigned long long)gridDim.x * kWarps * 32;
    for (unsigned long long base = lo + ((unsigned long long)blockIdx.x * kWarps + w) * 32; base < n;
         base += stride) {
        const unsigned long long idx = base + lane;
        const bool valid = idx < n;
        unsigned bits = 0;
        {
            int2 pr = make_int2(0, 0);
            int fa[DIM], fb[DIM];
            bool inb = true;
            if (valid) {
                pr = pairs[idx];
#pragma unroll
                for (int k = 0; k < DIM; ++k) {
                    fa[k] = __ldg(P + (size_t)pr.x * DIM + k);
                    fb[k] = __ldg(P + (size_t)pr.y * DIM + k);
                    inb = inb && fa[k] >= 0 && fa[k] < nv && fb[k] >= 0 && fb[k] < nv;
                }
                if (continuous) bits = stencil_bits<DIM>(fa, fb, __ldg(flags + pr.x), __ldg(flags + pr.y));
            } else {
#pragma unroll
                for (int k = 0; k < DIM; ++k) fa[k] = fb[k] = 0;
            }
            if (discrete && valid) {
                bool shared = false;
#pragma unroll
                for (int i = 0; i < DIM; ++i)
#pragma unroll
                    for (int j = 0; j < DIM; ++j) shared |= fa[i] == fb[j];
                if (!inb) atomicOr(&cnt->err, kErrBadIndex);
                int hit = 0;
                if (!shared && inb)
                    hit = discrete_pair<DIM>(fa[0], fa[1], DIM == 3 ? fa[DIM - 1] : 0, fb[0], fb[1],
                                             DIM == 3 ? fb[DIM - 1] : 0, V1);
                if (hit) {
                    const unsigned long long slot = warp_append(&cnt->n_discrete);
                    if (slot < disc_cap) disc[slot] = pr;
                }
            }
            if (!continuous) continue;
#pragma unroll
            for (int k = 0; k < DIM; ++k) { wp.fa[lane][k] = fa[k]; wp.fb[lane][k] = fb[k]; }
            wp.bits[0][lane] = bits & 0x3fu;
            wp.bits[1][lane] = bits >> 6;
        }
        const unsigned cvf = __popc(bits & 0x3fu), cee = DIM == 3 ? __popc(bits >> 6) : 0u;
        sum_vf += cvf;
        sum_ee += cee;
        generate<DIM, true>(o, vf_eta, wp, warp_prefix<DIM>(wp, cvf), hq_vf, nh_vf, tq_vf, nt_vf);
        if constexpr (DIM == 3) generate<DIM, false>(o, ee_eta, wp, warp_prefix<DIM>(wp, cee), hq_ee, nh_ee, tq_ee, nt_ee);
        __syncwarp();
    }
    if (continuous) {
        drain<DIM, true>(o, vf_eta, hq_vf, nh_vf, tq_vf, nt_vf);
        if constexpr (DIM == 3) drain<DIM, false>(o, ee_eta, hq_ee, nh_ee, tq_ee, nt_ee);
        // candidate counts: one atomic per warp
#pragma unroll
        for (int off = 16; off; off >>= 1) {
            sum_vf += __shfl_down_sync(0xffffffffu, sum_vf, off);
            sum_ee += __shfl_down_sync(0xffffffffu, sum_ee, off);
        }
        if (lane == 0) {
            if (sum_vf) atomicAdd(&cnt->n_vf, sum_vf);
            if (DIM == 3 && sum_ee) atomicAdd(&cnt->n_ee, sum_ee);
        }
    }
}

void launch_narrow_fused(int dim, const int2 *pairs, unsigned long long pair_cap, const int *P,
                         const unsigned char *flags, const double *V0, const double *V1, int nv, double vf_eta,
                         double ee_eta, int continuous, int discrete, int2 *disc, unsigned long long disc_cap,
                         int4 *hit_sten, double *hit_toi, unsigned char *hit_isvf, unsigned long long hit_cap,
                         Counters *cnt, int grid, cudaStream_t st, const unsigned long long *lo_ptr,
                         const unsigned long long *hi_ptr)
{
    if (!hi_ptr) hi_ptr = &cnt->n_pairs;
    if (dim == 3)
        k_narrow_fused<3><<<grid, kWarps * 32, 0, st>>>(pairs, pair_cap, P, flags, V0, V1, nv, vf_eta, ee_eta,
                                                         continuous, discrete, disc, disc_cap, hit_sten, hit_toi,
                                                         hit_isvf, hit_cap, cnt, lo_ptr, hi_ptr);
    else
        k_narrow_fused<2><<<grid, kWarps * 32, 0, st>>>(pairs, pair_cap, P, flags, V0, V1, nv, vf_eta, ee_eta,
                                                         continuous, discrete, disc, disc_cap, hit_sten, hit_toi,
                                                         hit_isvf, hit_cap, cnt, lo_ptr, hi_ptr);
}

} // namespace mclccd
