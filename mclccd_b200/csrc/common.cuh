// Shared device-side definitions for the B200 CCD path.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

// Pure arithmetic shared by device kernels and the host-side tests.
#ifndef MC_HD
#define MC_HD __host__ __device__ __forceinline__
#endif

namespace mclccd {

// ---------------------------------------------------------------------------
// Per-primitive flags (uint8).  Bits 0-2: vertex slot j is the representative
// occurrence of its vertex; bits 3-5: edge slot j is the representative
// occurrence of its edge (mclccd BVHTree.cpp:50-80); bit 6: primitive active.
// ---------------------------------------------------------------------------
constexpr unsigned kFlagV0 = 1u;
constexpr unsigned kFlagE0 = 1u << 3;
constexpr unsigned kFlagActive = 1u << 6;
constexpr unsigned kFlagAllRep = 0x3Fu;

// Error bits accumulated on the device (Counters::err).  None of them traps:
// the kernel records the bit and skips the offending access.
constexpr unsigned kErrBadIndex = 1u << 0;    // a P entry outside [0, nv)
constexpr unsigned kErrStack = 1u << 1;       // traversal stack overflow
constexpr unsigned kErrSortWait = 1u << 2;    // radix-sort look-back gave up
constexpr unsigned kErrHashFull = 1u << 3;    // edge hash table probe limit
constexpr unsigned kErrAccdIters = 1u << 4;   // ACCD loop hit its 1000 cap (reported, result kept)
constexpr unsigned kErrWave = 1u << 5;        // a batch wave could not fit its buffers

// Device counters of one traverse: counts are exact even when a buffer is
// too small (writes past capacity are skipped, the count keeps going).
struct Counters {
    unsigned long long n_pairs;
    unsigned long long n_vf;
    unsigned long long n_ee;
    unsigned long long n_hits;
    unsigned long long n_discrete;
    unsigned long long n_fp64[2];     // FP32 form: stencils queued for FP64 (VF / EE lists)
    unsigned long long n_bound_toi;   // FP32 form: hits reported with the certified toi bound
    unsigned int err;
    unsigned int pad;
};

// ---------------------------------------------------------------------------
// Hierarchy layout (LBVH, Karras 2012).  Internal node i has children
// split and split+1; each child is a leaf (sorted position) or an internal
// node.  Each child's FP32 t0 box and t1 box (outward-rounded; unions for
// inner nodes) live in the parent, so one 128-byte node read applies the
// reference's whole box predicate -- swept overlap and the t0/t1 same-side
// separation test -- to both children.
//   3D child (3 x float4): (t0lo.x t0lo.y t0lo.z t0hi.x) (t0hi.y t0hi.z t1lo.x t1lo.y)
//                          (t1lo.z t1hi.x t1hi.y t1hi.z)
//   2D child (2 x float4): (t0lo.x t0lo.y t0hi.x t0hi.y) (t1lo.x t1lo.y t1hi.x t1hi.y)
//   d = (split, meta, last, parent)
// meta byte 0: bit0 left child is a leaf, bit1 right child is a leaf;
// byte 1: left child active; byte 2: right child active.
// ---------------------------------------------------------------------------
struct __align__(16) Node {
    float4 l[3];
    float4 r[3];
    int4 d;
    int4 pad;
};

// FP32 t0/t1 boxes of one child or query.
template <int DIM>
struct Box2T {
    float t0lo[DIM], t0hi[DIM], t1lo[DIM], t1hi[DIM];
};

template <int DIM>
__device__ __forceinline__ void unpack_child(const float4 *s, Box2T<DIM> &b)
{
    if constexpr (DIM == 3) {
        b.t0lo[0] = s[0].x; b.t0lo[1] = s[0].y; b.t0lo[2] = s[0].z; b.t0hi[0] = s[0].w;
        b.t0hi[1] = s[1].x; b.t0hi[2] = s[1].y; b.t1lo[0] = s[1].z; b.t1lo[1] = s[1].w;
        b.t1lo[2] = s[2].x; b.t1hi[0] = s[2].y; b.t1hi[1] = s[2].z; b.t1hi[2] = s[2].w;
    } else {
        b.t0lo[0] = s[0].x; b.t0lo[1] = s[0].y; b.t0hi[0] = s[0].z; b.t0hi[1] = s[0].w;
        b.t1lo[0] = s[1].x; b.t1lo[1] = s[1].y; b.t1hi[0] = s[1].z; b.t1hi[1] = s[1].w;
    }
}

template <int DIM>
__device__ __forceinline__ void pack_child(float4 *s, const Box2T<DIM> &b)
{
    if constexpr (DIM == 3) {
        s[0] = make_float4(b.t0lo[0], b.t0lo[1], b.t0lo[2], b.t0hi[0]);
        s[1] = make_float4(b.t0hi[1], b.t0hi[2], b.t1lo[0], b.t1lo[1]);
        s[2] = make_float4(b.t1lo[2], b.t1hi[0], b.t1hi[1], b.t1hi[2]);
    } else {
        s[0] = make_float4(b.t0lo[0], b.t0lo[1], b.t0hi[0], b.t0hi[1]);
        s[1] = make_float4(b.t1lo[0], b.t1lo[1], b.t1hi[0], b.t1hi[1]);
    }
}

// The reference's box predicate (BVHTree.cpp:401-426, without the active
// test) on FP32 boxes.  With outward-rounded leaf boxes and exact unions it
// never rejects a pair the FP64 predicate accepts.
template <int DIM>
__device__ __forceinline__ bool boxes_may_intersect(const Box2T<DIM> &q, const Box2T<DIM> &c)
{
    bool ok = true;
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
        const float qlo = fminf(q.t0lo[k], q.t1lo[k]), qhi = fmaxf(q.t0hi[k], q.t1hi[k]);
        const float clo = fminf(c.t0lo[k], c.t1lo[k]), chi = fmaxf(c.t0hi[k], c.t1hi[k]);
        ok = ok && clo <= qhi && qlo <= chi;
        ok = ok && !((c.t0lo[k] > q.t0hi[k] && c.t1lo[k] > q.t1hi[k]) ||
                     (c.t0hi[k] < q.t0lo[k] && c.t1hi[k] < q.t1lo[k]));
    }
    return ok;
}
constexpr int kMetaLeftLeaf = 1;
constexpr int kMetaRightLeaf = 2;

// FP64 leaf record in sorted order: t0 box then t1 box, each (min, max).
// 3D: 12 doubles; 2D: 8 doubles.  The swept box is min/max of the two: the
// reference pads the swept box, t0 and t1 boxes by the same eta, and
// fl(min(a,b) - eta) == min(fl(a - eta), fl(b - eta)) for round-to-nearest.
template <int DIM>
struct LeafBox {
    double lo0[DIM], hi0[DIM], lo1[DIM], hi1[DIM];
};

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ unsigned lanemask_lt() { return (1u << lane_id()) - 1u; }

// Warp-aggregated append: every lane that calls this together (the active
// lanes at this point) gets a distinct slot; one atomic per warp.
__device__ __forceinline__ unsigned long long warp_append(unsigned long long *counter)
{
    unsigned mask = __activemask();
    int leader = __ffs(mask) - 1;
    unsigned rank = __popc(mask & lanemask_lt());
    unsigned long long base = 0;
    if ((int)lane_id() == leader) base = atomicAdd(counter, (unsigned long long)__popc(mask));
    base = __shfl_sync(mask, base, leader);
    return base + rank;
}

// Warp-wide (all 32 lanes must call) reservation of k slots per lane.
__device__ __forceinline__ unsigned long long warp_reserve(unsigned long long *counter, unsigned k)
{
    unsigned incl = k;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        unsigned v = __shfl_up_sync(0xffffffffu, incl, o);
        if ((int)lane_id() >= o) incl += v;
    }
    unsigned total = __shfl_sync(0xffffffffu, incl, 31);
    unsigned long long base = 0;
    if (lane_id() == 31 && total) base = atomicAdd(counter, (unsigned long long)total);
    base = __shfl_sync(0xffffffffu, base, 31);
    return base + (incl - k);
}

// Block-wide (every thread of the block must call, blockDim.x == BLOCK)
// reservation of a slots on counter ca and b slots on counter cb per thread:
// one atomic per counter per block instead of one per warp, so a kernel whose
// warps all append to the same list does not queue on that counter in L2.
// a, b < 2^16 per thread and their block totals < 2^16.  Returns the
// thread's first slot on each counter.
template <int BLOCK>
__device__ __forceinline__ void block_reserve2(unsigned long long *ca, unsigned a, unsigned long long *cb, unsigned b,
                                               unsigned long long &sa, unsigned long long &sb)
{
    constexpr int W = BLOCK / 32;
    __shared__ unsigned s_warp[W];
    __shared__ unsigned long long s_base[2];
    const unsigned k = a | (b << 16);
    unsigned incl = k;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned v = __shfl_up_sync(0xffffffffu, incl, o);
        if ((int)lane_id() >= o) incl += v;
    }
    const int warp = threadIdx.x >> 5;
    if (lane_id() == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const unsigned tot = lane_id() < W ? s_warp[lane_id()] : 0u;
        unsigned sc = tot;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned v = __shfl_up_sync(0xffffffffu, sc, o);
            if ((int)lane_id() >= o) sc += v;
        }
        if (lane_id() < W) s_warp[lane_id()] = sc - tot;   // exclusive offsets of the warps
        if (lane_id() == 31) {
            s_base[0] = (sc & 0xffffu) ? atomicAdd(ca, (unsigned long long)(sc & 0xffffu)) : 0ull;
            s_base[1] = (sc >> 16) ? atomicAdd(cb, (unsigned long long)(sc >> 16)) : 0ull;
        }
    }
    __syncthreads();
    const unsigned off = s_warp[warp] + (incl - k);
    sa = s_base[0] + (off & 0xffffu);
    sb = s_base[1] + (off >> 16);
    __syncthreads();   // the next call may overwrite s_warp / s_base
}

// Monotone float <-> uint mapping for atomic min/max of floats.
__device__ __forceinline__ unsigned float_to_ordered(float f)
{
    unsigned u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__host__ __device__ __forceinline__ float ordered_to_float(unsigned u)
{
    unsigned v = (u & 0x80000000u) ? (u & 0x7fffffffu) : ~u;
#ifdef __CUDA_ARCH__
    return __uint_as_float(v);
#else
    float f; __builtin_memcpy(&f, &v, 4); return f;
#endif
}

} // namespace mclccd
