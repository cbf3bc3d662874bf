// Device building blocks of the LBVH shared by the single-scene path
// (build.cu, traverse.cu) and the batched path (batch.cu).
#pragma once

#include "common.cuh"

namespace mclccd {

// ---------------------------------------------------------------------------
// Leaf box of primitive `prim` (BVHTree.cpp:95-119): hull of its vertices at
// t0 and at t1, padded by eta.  Returns false if a vertex index is invalid.
// ---------------------------------------------------------------------------
template <int DIM>
__device__ __forceinline__ bool compute_leaf_box(const double *__restrict__ V0, const double *__restrict__ V1,
                                                 const int *__restrict__ P, int pdim, int nv, int prim, double eta,
                                                 const int *__restrict__ active, LeafBox<DIM> &b, bool &act)
{
    bool ok = true;
#pragma unroll
    for (int k = 0; k < DIM; ++k) { b.lo0[k] = b.lo1[k] = 1.7976931348623157e308; b.hi0[k] = b.hi1[k] = -1.7976931348623157e308; }
    act = active == nullptr;
    for (int j = 0; j < pdim; ++j) {
        int v = __ldg(P + (size_t)prim * pdim + j);
        if (v < 0 || v >= nv) { ok = false; continue; }
#pragma unroll
        for (int k = 0; k < DIM; ++k) {
            double a = __ldg(V0 + (size_t)v * DIM + k), c = __ldg(V1 + (size_t)v * DIM + k);
            if (a < b.lo0[k]) b.lo0[k] = a;
            if (b.hi0[k] < a) b.hi0[k] = a;
            if (c < b.lo1[k]) b.lo1[k] = c;
            if (b.hi1[k] < c) b.hi1[k] = c;
        }
        if (active != nullptr && __ldg(active + v)) act = true;
    }
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
        b.lo0[k] -= eta; b.lo1[k] -= eta;
        b.hi0[k] += eta; b.hi1[k] += eta;
    }
    return ok;
}

__device__ __forceinline__ unsigned expand_bits3(unsigned v)   // 10 bits -> every 3rd bit
{
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}
__device__ __forceinline__ unsigned expand_bits2(unsigned v)   // 15 bits -> every 2nd bit
{
    v &= 0x7fffu;
    v = (v | (v << 8)) & 0x00FF00FFu;
    v = (v | (v << 4)) & 0x0F0F0F0Fu;
    v = (v | (v << 2)) & 0x33333333u;
    v = (v | (v << 1)) & 0x55555555u;
    return v;
}

template <int DIM>
__device__ __forceinline__ void write_child(Node *nodes, int parent, bool right, const Box2T<DIM> &b, bool act)
{
    Node *nd = nodes + parent;
    pack_child<DIM>(right ? nd->r : nd->l, b);
    reinterpret_cast<unsigned char *>(&nd->d.y)[right ? 2 : 1] = act ? 1 : 0;
}

// Refit arrival at a node: one acquire-release add on its visit counter.  The
// first child's thread releases its box (written to the node before the add)
// and stops; the second acquires that box and climbs on.
__device__ __forceinline__ bool refit_second_arrival(int *counter)
{
    int prev;
    asm volatile("atom.acq_rel.gpu.global.add.s32 %0, [%1], 1;" : "=r"(prev) : "l"(counter) : "memory");
    return prev != 0;
}

// The second child to arrive at a node during the refit: merge the sibling's
// box (written by the first) into this child's box and activity.
template <int DIM>
__device__ __forceinline__ void merge_sibling(const Node *nd, bool right, Box2T<DIM> &box, bool &act)
{
    constexpr int S = DIM == 3 ? 3 : 2;
    float4 ss[S];
    const float4 *src = right ? nd->l : nd->r;
#pragma unroll
    for (int i = 0; i < S; ++i) ss[i] = __ldcg(src + i);
    const int meta = __ldcg(&nd->d.y);
    act = act || ((meta >> (right ? 8 : 16)) & 0xff);
    Box2T<DIM> b;
    unpack_child<DIM>(ss, b);
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
        box.t0lo[k] = fminf(box.t0lo[k], b.t0lo[k]); box.t0hi[k] = fmaxf(box.t0hi[k], b.t0hi[k]);
        box.t1lo[k] = fminf(box.t1lo[k], b.t1lo[k]); box.t1hi[k] = fmaxf(box.t1hi[k], b.t1hi[k]);
    }
}

// FP32 boxes that contain the FP64 ones (round min down, max up).
template <int DIM>
__device__ __forceinline__ Box2T<DIM> outward(const LeafBox<DIM> &b)
{
    Box2T<DIM> o;
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
        o.t0lo[k] = __double2float_rd(b.lo0[k]); o.t0hi[k] = __double2float_ru(b.hi0[k]);
        o.t1lo[k] = __double2float_rd(b.lo1[k]); o.t1hi[k] = __double2float_ru(b.hi1[k]);
    }
    return o;
}

// Three-valued leaf test.  Each stored FP32 bound brackets its FP64 value: a
// min rounded down (L) means the FP64 min lies in [L, next_up(L)], a max
// rounded up (H) means the FP64 max lies in [next_down(H), H].  The
// reference's predicate (BVHTree.cpp:411-423) is evaluated on those intervals:
// 1 = true for every FP64 value in the brackets, 0 = false for every one,
// 2 = cannot tell (then the FP64 boxes decide).  No FP64 data is touched for
// the clear cases, and the answer is never different from the FP64 test.
// Upper end of a min's bracket and lower end of a max's bracket:
// x + |x| 2^-22 (+ 2^-125 for tiny x) with directed rounding is at least one
// ulp away from x, so [x, up(x)] holds the FP64 min and [dn(x), x] the FP64 max.
__device__ __forceinline__ float up1(float x) { return __fadd_ru(__fmaf_ru(fabsf(x), 0x1p-22f, x), 0x1p-125f); }
__device__ __forceinline__ float dn1(float x) { return __fsub_rd(__fmaf_rd(-fabsf(x), 0x1p-22f, x), 0x1p-125f); }

template <int DIM>
__device__ __forceinline__ Box2T<DIM> inner(const Box2T<DIM> &b)
{
    Box2T<DIM> o;
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
        o.t0lo[k] = up1(b.t0lo[k]); o.t1lo[k] = up1(b.t1lo[k]);
        o.t0hi[k] = dn1(b.t0hi[k]); o.t1hi[k] = dn1(b.t1hi[k]);
    }
    return o;
}

// q, c: outward boxes; qi: inner(q).
template <int DIM>
__device__ __forceinline__ int leaf_test3(const Box2T<DIM> &q, const Box2T<DIM> &qi, const Box2T<DIM> &c)
{
    int res = 1;
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
        const float c0lo_u = up1(c.t0lo[k]), c1lo_u = up1(c.t1lo[k]);
        const float c0hi_d = dn1(c.t0hi[k]), c1hi_d = dn1(c.t1hi[k]);
        // overlap: min(lo0,lo1) <= max(hi0,hi1) both ways
        const float qmin_dn = fminf(q.t0lo[k], q.t1lo[k]), qmin_up = fminf(qi.t0lo[k], qi.t1lo[k]);
        const float qmax_up = fmaxf(q.t0hi[k], q.t1hi[k]), qmax_dn = fmaxf(qi.t0hi[k], qi.t1hi[k]);
        const float cmin_dn = fminf(c.t0lo[k], c.t1lo[k]), cmin_up = fminf(c0lo_u, c1lo_u);
        const float cmax_up = fmaxf(c.t0hi[k], c.t1hi[k]), cmax_dn = fmaxf(c0hi_d, c1hi_d);
        if (qmin_dn > cmax_up || cmin_dn > qmax_up) return 0;
        if (!(qmin_up <= cmax_dn && cmin_up <= qmax_dn)) res = 2;
        // separation on this axis at both times, on the same side:
        // (q.lo0 > c.hi0 && q.lo1 > c.hi1) || (q.hi0 < c.lo0 && q.hi1 < c.lo1)
        const bool a_true = q.t0lo[k] > c.t0hi[k] && q.t1lo[k] > c.t1hi[k];
        const bool a_false = qi.t0lo[k] <= c0hi_d || qi.t1lo[k] <= c1hi_d;
        const bool b_true = q.t0hi[k] < c.t0lo[k] && q.t1hi[k] < c.t1lo[k];
        const bool b_false = qi.t0hi[k] >= c0lo_u || qi.t1hi[k] >= c1lo_u;
        if (a_true || b_true) return 0;
        if (!(a_false && b_false)) res = 2;
    }
    return res;
}

// Candidate stencils of a leaf pair (faces fa, fb with representative flags
// ga, gb; get_candidates, BVHTree.cpp:305-398): bit i = VF (fa[i], fb),
// bit 3+i = VF (fb[i], fa), bit 6+3i+j = EE (fa edge i, fb edge j).
template <int DIM>
__device__ __forceinline__ unsigned stencil_bits(const int *fa, const int *fb, unsigned ga, unsigned gb)
{
    unsigned bits = 0;
#pragma unroll
    for (int i = 0; i < DIM; ++i) {
        bool sa = false, sb = false;
#pragma unroll
        for (int j = 0; j < DIM; ++j) { sa |= fa[i] == fb[j]; sb |= fb[i] == fa[j]; }
        if ((ga & (kFlagV0 << i)) && !sa) bits |= 1u << i;
        if ((gb & (kFlagV0 << i)) && !sb) bits |= 1u << (3 + i);
    }
    if constexpr (DIM == 3) {
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            if (!(ga & (kFlagE0 << i))) continue;
            const int a = fa[i], b = fa[(i + 1) % 3];
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                if (!(gb & (kFlagE0 << j))) continue;
                const int c = fb[j], d = fb[(j + 1) % 3];
                if (a == c || a == d || b == c || b == d) continue;
                bits |= 1u << (6 + 3 * i + j);
            }
        }
    }
    return bits;
}

} // namespace mclccd
