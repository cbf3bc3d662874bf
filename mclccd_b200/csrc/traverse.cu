// Self-traversal of the LBVH and leaf-pair expansion.
//
// Replaces BVHTree::traverse/collide/get_candidates/default_discrete_test
// (BVHTree.cpp:129-302, 305-398, 464-500).  The reference enumerates each
// unordered pair of distinct leaves whose boxes pass boxes_intersect exactly
// once (one frontlist seed per internal node, BVHTree.cpp:169-185); here each
// sorted leaf q walks the tree for leaves k > q, so every unordered pair is
// found once.  Inner nodes are tested with outward-rounded FP32 boxes (a
// superset), leaves with the exact FP64 predicate, so the leaf-pair set is
// exactly the reference's.  Pairs are emitted canonically (lower primitive
// index first).
#include "common.cuh"

#include <algorithm>
#include "geom.cuh"
#include "kernels.cuh"
#include "lbvh.cuh"

namespace mclccd {

// Traversal stack entries per thread (shared memory) and resident blocks per
// SM the walk is compiled for.  A Karras tree's depth is at most 30 key bits
// plus log2 of the largest run of equal keys; overflow is reported
// (kErrStack), never silent.
#ifndef MCLCCD_WALK_STACK
#define MCLCCD_WALK_STACK 64
#endif
#ifndef MCLCCD_WALK_MIN_BLOCKS
#define MCLCCD_WALK_MIN_BLOCKS 5
#endif
#ifndef MCLCCD_WALK_BUF_MIN_BLOCKS
#define MCLCCD_WALK_BUF_MIN_BLOCKS 4
#endif
constexpr int kStackDepth = MCLCCD_WALK_STACK;

template <int DIM>
__global__ void __launch_bounds__(128, MCLCCD_WALK_MIN_BLOCKS)
k_traverse(const Node *__restrict__ nodes, const LeafBox<DIM> *__restrict__ leaf_box,
           const unsigned char *__restrict__ leaf_active, const int *__restrict__ sorted, int n, int q_begin,
           int q_end, int2 *__restrict__ pairs, unsigned long long cap, Counters *cnt)
{
    constexpr int S = DIM == 3 ? 3 : 2;
    const int q = q_begin + blockIdx.x * blockDim.x + threadIdx.x;   // queries [q_begin, q_end), q_end <= n - 1
    if (q >= q_end) return;
    const bool qact = leaf_active[q] != 0;
    const int qprim = sorted[q];
    // Only the FP32 boxes stay in registers; the FP64 box is re-read for the
    // rare undecided leaf test and the inner bracket recomputed per test.
    Box2T<DIM> qbox;
    {
        const LeafBox<DIM> &qb = leaf_box[q];
#pragma unroll
        for (int k = 0; k < DIM; ++k) {
            qbox.t0lo[k] = __double2float_rd(qb.lo0[k]); qbox.t0hi[k] = __double2float_ru(qb.hi0[k]);
            qbox.t1lo[k] = __double2float_rd(qb.lo1[k]); qbox.t1hi[k] = __double2float_ru(qb.hi1[k]);
        }
    }

    // Leaf k passed the cheap filters: decide it from the FP32 brackets and
    // fall back to the FP64 boxes only when they cannot tell.
    auto leaf = [&](int k, const Box2T<DIM> &kbox) {
        int r = leaf_test3<DIM>(qbox, inner<DIM>(qbox), kbox);
        if (r == 2) r = leaf_boxes_intersect<DIM>(leaf_box[q], leaf_box[k]) ? 1 : 0;
        if (r == 1) {
            const int kprim = __ldg(sorted + k);
            unsigned long long slot = warp_append(&cnt->n_pairs);
            if (slot < cap) pairs[slot] = make_int2(min(qprim, kprim), max(qprim, kprim));
        }
    };

    // Per-thread stack in shared memory, [depth][thread]: conflict-free.
    __shared__ int stack[kStackDepth][128];
    const int tid = threadIdx.x;
    int sp = 0;
    int node = 0;
    // A query visits each internal node at most once: n - 1 steps bound it.
    for (int steps = 0;; ++steps) {
        if (steps >= n) { atomicOr(&cnt->err, kErrStack); break; }
        float4 ls[S], rs[S];
#pragma unroll
        for (int i = 0; i < S; ++i) { ls[i] = __ldg(&nodes[node].l[i]); rs[i] = __ldg(&nodes[node].r[i]); }
        const int4 d = __ldg(&nodes[node].d);
        const int split = d.x, meta = d.y, last = d.z;
        Box2T<DIM> lb, rb;
        unpack_child<DIM>(ls, lb);
        unpack_child<DIM>(rs, rb);
        const bool lact = ((meta >> 8) & 0xff) != 0, ract = ((meta >> 16) & 0xff) != 0;
        bool lok = split > q && (qact || lact);
        bool rok = last > q && (qact || ract);
        if (lok && (meta & kMetaLeftLeaf)) { leaf(split, lb); lok = false; }
        if (rok && (meta & kMetaRightLeaf)) { leaf(split + 1, rb); rok = false; }
        lok = lok && boxes_may_intersect<DIM>(qbox, lb);
        rok = rok && boxes_may_intersect<DIM>(qbox, rb);
        if (lok) {
            if (rok) {
                if (sp < kStackDepth) stack[sp++][tid] = split + 1;
                else atomicOr(&cnt->err, kErrStack);
            }
            node = split;
        } else if (rok) {
            node = split + 1;
        } else {
            if (sp == 0) break;
            node = stack[--sp][tid];
        }
    }
}

// ---------------------------------------------------------------------------
// Warp-cooperative ("packet") form of the same walk.  The 32 queries of a warp
// are consecutive in Morton order, so their boxes are close: the warp walks
// the tree once, every lane tests each visited node's children against its
// own box, and the warp descends into a child when any lane needs it.
// Control flow is warp-uniform (one stack per warp, in shared memory); each
// lane still applies exactly its own tests, so the pairs found are the same.
// ---------------------------------------------------------------------------
// Window form (MCLCCD_TUNE_WALK_WINDOW = W).  Most of a query's overlapping
// leaves are close to it in Morton order, where the tree walk is also most
// divergent.  So each block first stages the FP32 boxes (rounded outward) and
// active flags of the leaves after its 128 queries, (q0, q0 + 127 + W], in
// shared memory with coalesced loads; each query tests the W leaves after it
// from there, all lanes in step; then it walks the tree only into subtrees
// that hold leaves beyond q + W.  Every leaf k > q is tested exactly once, by
// the same three-valued FP32 test with the FP64 fallback, so the leaf-pair
// set is the one of k_traverse.
// 4 resident blocks per SM: the staged window and the walk state need 128
// registers to run without spills (at 96 the spills in the walk loop cost
// more than the window saves).
template <int DIM, int W>
__global__ void __launch_bounds__(128, 4)
k_traverse_window(const Node *__restrict__ nodes, const LeafBox<DIM> *__restrict__ leaf_box,
                  const unsigned char *__restrict__ leaf_active, const int *__restrict__ sorted, int n, int q_begin,
                  int q_end, int2 *__restrict__ pairs, unsigned long long cap, Counters *cnt)
{
    constexpr int S = DIM == 3 ? 3 : 2;
    constexpr int NB = 127 + W;
    __shared__ float s_box[NB][4 * DIM];   // t0lo, t0hi, t1lo, t1hi
    __shared__ unsigned char s_act[NB];
    __shared__ int stack[kStackDepth][128];
    const int tid = threadIdx.x;
    const int q0 = q_begin + blockIdx.x * 128;   // queries [q_begin, q_end), q_end <= n - 1
    if (q0 >= q_end) return;                      // whole block past the end
    for (int i = tid; i < NB; i += 128) {
        const int k = q0 + 1 + i;
        if (k < n) {
            const LeafBox<DIM> &kb = leaf_box[k];
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                s_box[i][d] = __double2float_rd(kb.lo0[d]);
                s_box[i][DIM + d] = __double2float_ru(kb.hi0[d]);
                s_box[i][2 * DIM + d] = __double2float_rd(kb.lo1[d]);
                s_box[i][3 * DIM + d] = __double2float_ru(kb.hi1[d]);
            }
            s_act[i] = leaf_active[k];
        }
    }
    __syncthreads();
    const int q = q0 + tid;
    if (q >= q_end) return;
    const bool qact = leaf_active[q] != 0;
    const int qprim = sorted[q];
    Box2T<DIM> qbox;
    {
        const LeafBox<DIM> &qb = leaf_box[q];
#pragma unroll
        for (int k = 0; k < DIM; ++k) {
            qbox.t0lo[k] = __double2float_rd(qb.lo0[k]); qbox.t0hi[k] = __double2float_ru(qb.hi0[k]);
            qbox.t1lo[k] = __double2float_rd(qb.lo1[k]); qbox.t1hi[k] = __double2float_ru(qb.hi1[k]);
        }
    }
    auto leaf = [&](int k, const Box2T<DIM> &kbox) {
        int r = leaf_test3<DIM>(qbox, inner<DIM>(qbox), kbox);
        if (r == 2) r = leaf_boxes_intersect<DIM>(leaf_box[q], leaf_box[k]) ? 1 : 0;
        if (r == 1) {
            const int kprim = __ldg(sorted + k);
            unsigned long long slot = warp_append(&cnt->n_pairs);
            if (slot < cap) pairs[slot] = make_int2(min(qprim, kprim), max(qprim, kprim));
        }
    };
    // 1. the window: leaves q + 1 .. q + W from shared memory
    const int qw = min(q + W, n - 1);
    for (int k = q + 1; k <= qw; ++k) {
        const int i = k - q0 - 1;
        if (!(qact || s_act[i])) continue;
        Box2T<DIM> kb;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            kb.t0lo[d] = s_box[i][d]; kb.t0hi[d] = s_box[i][DIM + d];
            kb.t1lo[d] = s_box[i][2 * DIM + d]; kb.t1hi[d] = s_box[i][3 * DIM + d];
        }
        leaf(k, kb);
    }
    // 2. the tree, for leaves beyond the window
    int sp = 0, node = 0;
    for (int steps = 0;; ++steps) {
        if (steps >= n) { atomicOr(&cnt->err, kErrStack); break; }
        float4 ls[S], rs[S];
#pragma unroll
        for (int i = 0; i < S; ++i) { ls[i] = __ldg(&nodes[node].l[i]); rs[i] = __ldg(&nodes[node].r[i]); }
        const int4 d = __ldg(&nodes[node].d);
        const int split = d.x, meta = d.y, last = d.z;
        Box2T<DIM> lb, rb;
        unpack_child<DIM>(ls, lb);
        unpack_child<DIM>(rs, rb);
        const bool lact = ((meta >> 8) & 0xff) != 0, ract = ((meta >> 16) & 0xff) != 0;
        bool lok = split > qw && (qact || lact);
        bool rok = last > qw && (qact || ract);
        if (lok && (meta & kMetaLeftLeaf)) { leaf(split, lb); lok = false; }
        if (rok && (meta & kMetaRightLeaf)) { leaf(split + 1, rb); rok = false; }
        lok = lok && boxes_may_intersect<DIM>(qbox, lb);
        rok = rok && boxes_may_intersect<DIM>(qbox, rb);
        if (lok) {
            if (rok) {
                if (sp < kStackDepth) stack[sp++][tid] = split + 1;
                else atomicOr(&cnt->err, kErrStack);
            }
            node = split;
        } else if (rok) {
            node = split + 1;
        } else {
            if (sp == 0) break;
            node = stack[--sp][tid];
        }
    }
}

// ---------------------------------------------------------------------------
// Refill form (MCLCCD_TUNE_WALK_REFILL): the window walk with idle lanes
// refilled.  In the plain walk a warp runs until its slowest query is done,
// so most lanes idle through the long walks (about a third of the lanes are
// active per instruction).  Here each warp is persistent: it takes chunks of
// 32 consecutive queries from a global cursor, runs their window part (the
// W leaves after each query, staged per warp in shared memory: coherent) and
// queues them for the tree part in a per-warp pool; lanes whose tree walk is
// done take the next query from the pool, and the warp fetches a new chunk
// when the pool runs dry while a lane is idle.  Every query tests the same
// leaves with the same three-valued test and FP64 fallback as the window
// form, so the leaf-pair set is the same; only the order of the pairs in the
// list differs.
// ---------------------------------------------------------------------------
template <int DIM, int W>
__global__ void __launch_bounds__(128, 4)
k_traverse_refill(const Node *__restrict__ nodes, const LeafBox<DIM> *__restrict__ leaf_box,
                  const unsigned char *__restrict__ leaf_active, const int *__restrict__ sorted, int n, int q_begin,
                  int q_end, int2 *__restrict__ pairs, unsigned long long cap, Counters *cnt,
                  unsigned *__restrict__ cursor)
{
    constexpr int S = DIM == 3 ? 3 : 2;
    constexpr int NB = 32 + W;     // staged leaves per chunk: base + 1 .. base + 32 + W
    constexpr int POOL = 64;       // queries waiting for their tree part (< 32 left + one chunk)
    __shared__ float s_box[4][NB][4 * DIM];   // t0lo, t0hi, t1lo, t1hi (outward FP32)
    __shared__ unsigned char s_act[4][NB];
    __shared__ int s_pool[4][POOL];
    __shared__ int stack[kStackDepth][128];
    const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
    const unsigned full = 0xffffffffu;

    // leaf k against query qi (box qb, primitive qp): three-valued FP32 test,
    // FP64 boxes when it cannot tell
    auto leaf = [&](int qi, const Box2T<DIM> &qb, int qp, int k, const Box2T<DIM> &kb) {
        int r = leaf_test3<DIM>(qb, inner<DIM>(qb), kb);
        if (r == 2) r = leaf_boxes_intersect<DIM>(leaf_box[qi], leaf_box[k]) ? 1 : 0;
        if (r == 1) {
            const int kp = __ldg(sorted + k);
            const unsigned long long slot = warp_append(&cnt->n_pairs);
            if (slot < cap) pairs[slot] = make_int2(min(qp, kp), max(qp, kp));
        }
    };

    int npool = 0;            // warp-uniform
    bool exhausted = false;   // warp-uniform
    int q = -1, qw = 0, qprim = 0, node = 0, sp = 0, steps = 0;
    bool qact = false;
    Box2T<DIM> qbox;
    for (;;) {
        const unsigned idle = __ballot_sync(full, q < 0);
        if (idle && npool == 0 && !exhausted) {
            // next chunk: its window part, then into the pool
            unsigned b = 0;
            if (lane == 0) b = atomicAdd(cursor, 32u);
            b = __shfl_sync(full, b, 0);
            const long long base = (long long)q_begin + b;
            if (base >= q_end) {
                exhausted = true;
                continue;
            }
            for (int i = lane; i < NB; i += 32) {
                const long long k = base + 1 + i;
                if (k < n) {
                    const Box2T<DIM> kb = outward<DIM>(leaf_box[k]);
#pragma unroll
                    for (int d = 0; d < DIM; ++d) {
                        s_box[w][i][d] = kb.t0lo[d];
                        s_box[w][i][DIM + d] = kb.t0hi[d];
                        s_box[w][i][2 * DIM + d] = kb.t1lo[d];
                        s_box[w][i][3 * DIM + d] = kb.t1hi[d];
                    }
                    s_act[w][i] = leaf_active[k];
                }
            }
            __syncwarp();
            const int cq = (int)base + lane;
            const bool valid = base + lane < q_end;
            if (valid) {
                const Box2T<DIM> cb = outward<DIM>(leaf_box[cq]);
                const bool cact = leaf_active[cq] != 0;
                const int cp = sorted[cq];
                const int cw = min(cq + W, n - 1);
                for (int k = cq + 1; k <= cw; ++k) {
                    const int i = k - (int)base - 1;
                    if (!(cact || s_act[w][i])) continue;
                    Box2T<DIM> kb;
#pragma unroll
                    for (int d = 0; d < DIM; ++d) {
                        kb.t0lo[d] = s_box[w][i][d]; kb.t0hi[d] = s_box[w][i][DIM + d];
                        kb.t1lo[d] = s_box[w][i][2 * DIM + d]; kb.t1hi[d] = s_box[w][i][3 * DIM + d];
                    }
                    leaf(cq, cb, cp, k, kb);
                }
            }
            const unsigned vm = __ballot_sync(full, valid);
            if (valid) s_pool[w][npool + __popc(vm & lanemask_lt())] = cq;
            npool += __popc(vm);
            __syncwarp();
            continue;
        }
        if (idle && npool > 0) {   // idle lanes take queries from the pool
            const int take = min(__popc(idle), npool);
            const int rank = __popc(idle & lanemask_lt());
            if (q < 0 && rank < take) {
                q = s_pool[w][npool - 1 - rank];
                qbox = outward<DIM>(leaf_box[q]);
                qact = leaf_active[q] != 0;
                qprim = sorted[q];
                qw = min(q + W, n - 1);
                node = 0;
                sp = 0;
                steps = 0;
            }
            npool -= take;
            __syncwarp();
        }
        if (__ballot_sync(full, q >= 0) == 0) {
            if (exhausted && npool == 0) break;
            continue;
        }
        if (q < 0) continue;
        // one node of this lane's tree walk (leaves beyond its window)
        if (++steps > n) {
            atomicOr(&cnt->err, kErrStack);
            q = -1;
            continue;
        }
        float4 ls[S], rs[S];
#pragma unroll
        for (int i = 0; i < S; ++i) { ls[i] = __ldg(&nodes[node].l[i]); rs[i] = __ldg(&nodes[node].r[i]); }
        const int4 d = __ldg(&nodes[node].d);
        const int split = d.x, meta = d.y, last = d.z;
        Box2T<DIM> lb, rb;
        unpack_child<DIM>(ls, lb);
        unpack_child<DIM>(rs, rb);
        const bool lact = ((meta >> 8) & 0xff) != 0, ract = ((meta >> 16) & 0xff) != 0;
        bool lok = split > qw && (qact || lact);
        bool rok = last > qw && (qact || ract);
        if (lok && (meta & kMetaLeftLeaf)) { leaf(q, qbox, qprim, split, lb); lok = false; }
        if (rok && (meta & kMetaRightLeaf)) { leaf(q, qbox, qprim, split + 1, rb); rok = false; }
        lok = lok && boxes_may_intersect<DIM>(qbox, lb);
        rok = rok && boxes_may_intersect<DIM>(qbox, rb);
        if (lok) {
            if (rok) {
                if (sp < kStackDepth) stack[sp++][tid] = split + 1;
                else atomicOr(&cnt->err, kErrStack);
            }
            node = split;
        } else if (rok) {
            node = split + 1;
        } else if (sp == 0) {
            q = -1;
        } else {
            node = stack[--sp][tid];
        }
    }
}

// Buffered form of the window walk (MCLCCD_TUNE_WALK_BUFFER): the same tests
// in the same order, with the pairs a warp finds collected in a per-warp
// shared-memory buffer and written out 32 at a time with one atomic on the
// pair counter, instead of one atomic per leaf test that hits.  The warp's
// loops run in step (a lane that is done idles until the whole warp is), so
// every flush is a whole-warp operation.
// RUN: pairs are written in whole runs of RUN (32 or 64), which keeps the
// pairs of neighbouring queries together in the list for the kernels that
// read it.
template <int DIM, int W, int RUN = 32>
__global__ void __launch_bounds__(128, MCLCCD_WALK_BUF_MIN_BLOCKS)
k_traverse_window_buf(const Node *__restrict__ nodes, const LeafBox<DIM> *__restrict__ leaf_box,
                      const unsigned char *__restrict__ leaf_active, const int *__restrict__ sorted, int n,
                      int q_begin, int q_end, int2 *__restrict__ pairs, unsigned long long cap, Counters *cnt)
{
    constexpr int S = DIM == 3 ? 3 : 2;
    constexpr int NB = 127 + W;
    constexpr int OUT = RUN + 64;   // < RUN left after a flush + at most 64 per step
    __shared__ float s_box[NB][4 * DIM];
    __shared__ unsigned char s_act[NB];
    __shared__ int stack[kStackDepth][128];
    __shared__ int2 s_out[4][OUT];
    __shared__ int s_nout[4];
    const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
    const unsigned full = 0xffffffffu;
    const int q0 = q_begin + blockIdx.x * 128;
    if (q0 >= q_end) return;   // whole block past the end
    for (int i = tid; i < NB; i += 128) {
        const int k = q0 + 1 + i;
        if (k < n) {
            const Box2T<DIM> kb = outward<DIM>(leaf_box[k]);
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                s_box[i][d] = kb.t0lo[d];
                s_box[i][DIM + d] = kb.t0hi[d];
                s_box[i][2 * DIM + d] = kb.t1lo[d];
                s_box[i][3 * DIM + d] = kb.t1hi[d];
            }
            s_act[i] = leaf_active[k];
        }
    }
    if (lane == 0) s_nout[w] = 0;
    __syncthreads();
    const int q = q0 + tid;
    const bool valid = q < q_end;
    const int qq = valid ? q : q_end - 1;
    const bool qact = leaf_active[qq] != 0;
    const int qprim = sorted[qq];
    const Box2T<DIM> qbox = outward<DIM>(leaf_box[qq]);

    // whole warp: write out the buffered pairs, all of them or whole 32s
    auto flush = [&](bool all) {
        __syncwarp();
        const int c = s_nout[w];
        const int take = all ? c : (c / RUN) * RUN;
        if (take == 0) return;
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(&cnt->n_pairs, (unsigned long long)take);
        base = __shfl_sync(full, base, 0);
        for (int i = lane; i < take; i += 32)
            if (base + i < cap) pairs[base + i] = s_out[w][i];
        __syncwarp();
        const int rest = c - take;   // < RUN <= take: source and destination do not overlap
        for (int i = lane; i < rest; i += 32) s_out[w][i] = s_out[w][take + i];
        __syncwarp();
        if (lane == 0) s_nout[w] = rest;
        __syncwarp();
    };
    auto leaf = [&](int k, const Box2T<DIM> &kbox) {
        int r = leaf_test3<DIM>(qbox, inner<DIM>(qbox), kbox);
        if (r == 2) r = leaf_boxes_intersect<DIM>(leaf_box[qq], leaf_box[k]) ? 1 : 0;
        if (r == 1) {
            const int kprim = __ldg(sorted + k);
            const unsigned m = __activemask();
            const int leader = __ffs(m) - 1;
            int pos = 0;
            if (lane == leader) pos = atomicAdd(&s_nout[w], __popc(m));
            pos = __shfl_sync(m, pos, leader) + __popc(m & lanemask_lt());
            s_out[w][pos] = make_int2(min(qprim, kprim), max(qprim, kprim));
        }
    };
    // 1. the window: leaves q + 1 .. q + W from shared memory, in step
    const int qw = min(qq + W, n - 1);
    for (int j = 1; j <= W; ++j) {
        flush(false);
        const int k = qq + j;
        if (!valid || k > qw) continue;
        const int i = k - q0 - 1;
        if (!(qact || s_act[i])) continue;
        Box2T<DIM> kb;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            kb.t0lo[d] = s_box[i][d]; kb.t0hi[d] = s_box[i][DIM + d];
            kb.t1lo[d] = s_box[i][2 * DIM + d]; kb.t1hi[d] = s_box[i][3 * DIM + d];
        }
        leaf(k, kb);
    }
    // 2. the tree beyond the window, one node per lane per step, in step
    int sp = 0, node = 0, steps = 0;
    bool done = !valid;
    while (__any_sync(full, !done)) {
        flush(false);
        if (done) continue;
        if (++steps > n) { atomicOr(&cnt->err, kErrStack); done = true; continue; }
        float4 ls[S], rs[S];
#pragma unroll
        for (int i = 0; i < S; ++i) { ls[i] = __ldg(&nodes[node].l[i]); rs[i] = __ldg(&nodes[node].r[i]); }
        const int4 d = __ldg(&nodes[node].d);
        const int split = d.x, meta = d.y, last = d.z;
        Box2T<DIM> lb, rb;
        unpack_child<DIM>(ls, lb);
        unpack_child<DIM>(rs, rb);
        const bool lact = ((meta >> 8) & 0xff) != 0, ract = ((meta >> 16) & 0xff) != 0;
        bool lok = split > qw && (qact || lact);
        bool rok = last > qw && (qact || ract);
        if (lok && (meta & kMetaLeftLeaf)) { leaf(split, lb); lok = false; }
        if (rok && (meta & kMetaRightLeaf)) { leaf(split + 1, rb); rok = false; }
        lok = lok && boxes_may_intersect<DIM>(qbox, lb);
        rok = rok && boxes_may_intersect<DIM>(qbox, rb);
        if (lok) {
            if (rok) {
                if (sp < kStackDepth) stack[sp++][tid] = split + 1;
                else atomicOr(&cnt->err, kErrStack);
            }
            node = split;
        } else if (rok) {
            node = split + 1;
        } else if (sp == 0) {
            done = true;
        } else {
            node = stack[--sp][tid];
        }
    }
    flush(true);
}

template <int DIM>
__global__ void __launch_bounds__(128)
k_traverse_packet(const Node *__restrict__ nodes, const LeafBox<DIM> *__restrict__ leaf_box,
                  const unsigned char *__restrict__ leaf_active, const int *__restrict__ sorted, int n,
                  int2 *__restrict__ pairs, unsigned long long cap, Counters *cnt)
{
    constexpr int S = DIM == 3 ? 3 : 2;
    __shared__ int wstack[4][kStackDepth];
    const int warp = threadIdx.x >> 5;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (__all_sync(0xffffffffu, q >= n - 1)) return;   // whole warp past the end
    const bool valid = q < n - 1;
    const int qq = valid ? q : n - 1;
    bool qact = false;
    int qprim = 0;
    Box2T<DIM> qbox;
    {
        const LeafBox<DIM> qb = leaf_box[qq];
        qact = leaf_active[qq] != 0;
        qprim = sorted[qq];
#pragma unroll
        for (int k = 0; k < DIM; ++k) {
            qbox.t0lo[k] = __double2float_rd(qb.lo0[k]); qbox.t0hi[k] = __double2float_ru(qb.hi0[k]);
            qbox.t1lo[k] = __double2float_rd(qb.lo1[k]); qbox.t1hi[k] = __double2float_ru(qb.hi1[k]);
        }
    }
    const Box2T<DIM> qin = inner<DIM>(qbox);

    auto leaf = [&](int k, const Box2T<DIM> &kbox) {
        int r = leaf_test3<DIM>(qbox, qin, kbox);
        if (r == 2) r = leaf_boxes_intersect<DIM>(leaf_box[qq], leaf_box[k]) ? 1 : 0;
        if (r == 1) {
            const int kprim = __ldg(sorted + k);
            unsigned long long slot = warp_append(&cnt->n_pairs);
            if (slot < cap) pairs[slot] = make_int2(min(qprim, kprim), max(qprim, kprim));
        }
    };

    int sp = 0;      // warp-uniform
    int node = 0;    // warp-uniform
    for (int steps = 0;; ++steps) {
        if (steps >= n) { if ((threadIdx.x & 31) == 0) atomicOr(&cnt->err, kErrStack); break; }
        float4 ls[S], rs[S];
#pragma unroll
        for (int i = 0; i < S; ++i) { ls[i] = __ldg(&nodes[node].l[i]); rs[i] = __ldg(&nodes[node].r[i]); }
        const int4 d = __ldg(&nodes[node].d);
        const int split = d.x, meta = d.y, last = d.z;
        Box2T<DIM> lb, rb;
        unpack_child<DIM>(ls, lb);
        unpack_child<DIM>(rs, rb);
        const bool lact = ((meta >> 8) & 0xff) != 0, ract = ((meta >> 16) & 0xff) != 0;
        bool lok = valid && split > q && (qact || lact);
        bool rok = valid && last > q && (qact || ract);
        if (meta & kMetaLeftLeaf) { if (lok) leaf(split, lb); lok = false; }
        if (meta & kMetaRightLeaf) { if (rok) leaf(split + 1, rb); rok = false; }
        lok = lok && boxes_may_intersect<DIM>(qbox, lb);
        rok = rok && boxes_may_intersect<DIM>(qbox, rb);
        const bool anyl = __any_sync(0xffffffffu, lok), anyr = __any_sync(0xffffffffu, rok);
        if (anyl) {
            if (anyr) {
                if (sp < kStackDepth) {
                    if ((threadIdx.x & 31) == 0) wstack[warp][sp] = split + 1;
                    ++sp;
                } else if ((threadIdx.x & 31) == 0) {
                    atomicOr(&cnt->err, kErrStack);
                }
            }
            node = split;
        } else if (anyr) {
            node = split + 1;
        } else {
            if (sp == 0) break;
            __syncwarp();
            node = wstack[warp][--sp];
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// Leaf pairs -> VF/EE stencils (get_candidates, BVHTree.cpp:305-398, with the
// lower primitive as "left") and the discrete test at V1
// (default_discrete_test, BVHTree.cpp:464-500).
// Stencil bits: VF a->b slot i = bit i, VF b->a slot i = bit 3+i,
// EE (i,j) = bit 6 + 3i + j.
// ---------------------------------------------------------------------------
// DISC = false: stencils only (the discrete test runs in k_discrete_pairs),
// so the kernel keeps few registers and many warps in flight for its gathers.
template <int DIM, bool DISC = true>
__global__ void __launch_bounds__(256)
k_expand_pairs(const int2 *__restrict__ pairs, unsigned long long pair_cap, const int *__restrict__ P,
               const unsigned char *__restrict__ flags, const double *__restrict__ V1, int nv,
               int4 *__restrict__ vf, unsigned long long vf_cap, int4 *__restrict__ ee, unsigned long long ee_cap,
               int2 *__restrict__ disc, unsigned long long disc_cap, int continuous, int discrete, Counters *cnt,
               const unsigned long long *lo_ptr, const unsigned long long *hi_ptr)
{
    if constexpr (!DISC) discrete = 0;
    // pairs [lo, hi): the whole list, or one query chunk's part of it
    unsigned long long n = *(volatile const unsigned long long *)hi_ptr;
    if (n > pair_cap) n = pair_cap;
    unsigned long long lo = lo_ptr ? *(volatile const unsigned long long *)lo_ptr : 0ull;
    if (lo > n) lo = n;
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long base = lo + (unsigned long long)blockIdx.x * blockDim.x; base < n; base += stride) {
        const unsigned long long idx = base + threadIdx.x;
        const bool valid = idx < n;
        int2 pr = make_int2(0, 0);
        int fa[DIM], fb[DIM];
        unsigned bits = 0;
        if (valid) {
            pr = pairs[idx];
#pragma unroll
            for (int k = 0; k < DIM; ++k) { fa[k] = __ldg(P + (size_t)pr.x * DIM + k); fb[k] = __ldg(P + (size_t)pr.y * DIM + k); }
            if (continuous) bits = stencil_bits<DIM>(fa, fb, __ldg(flags + pr.x), __ldg(flags + pr.y));
        }
        if (continuous) {
            const unsigned nvf = __popc(bits & 0x3fu), nee = DIM == 3 ? __popc(bits >> 6) : 0u;
            unsigned long long bvf, bee;
            block_reserve2<256>(&cnt->n_vf, nvf, &cnt->n_ee, nee, bvf, bee);
            for (unsigned m = bits & 0x3fu; m; m &= m - 1) {
                const int b = __ffs(m) - 1;
                const int *vs = b < 3 ? fa : fb;
                const int *fs = b < 3 ? fb : fa;
                if (bvf < vf_cap) vf[bvf] = make_int4(vs[b % 3], fs[0], fs[1], DIM == 3 ? fs[DIM - 1] : -1);
                ++bvf;
            }
            if constexpr (DIM == 3) {
                for (unsigned m = bits >> 6; m; m &= m - 1) {
                    const int b = __ffs(m) - 1, i = b / 3, j = b % 3;
                    if (bee < ee_cap) ee[bee] = make_int4(fa[i], fa[(i + 1) % 3], fb[j], fb[(j + 1) % 3]);
                    ++bee;
                }
            }
        }
        if (discrete && valid) {
            bool shared = false;
#pragma unroll
            for (int i = 0; i < DIM; ++i)
#pragma unroll
                for (int j = 0; j < DIM; ++j) shared |= fa[i] == fb[j];
            bool inb = true;
#pragma unroll
            for (int i = 0; i < DIM; ++i) inb = inb && fa[i] >= 0 && fa[i] < nv && fb[i] >= 0 && fb[i] < nv;
            if (!inb) atomicOr(&cnt->err, kErrBadIndex);
            int hit = 0;
            if (!shared && inb) {
                double A[DIM][DIM], B[DIM][DIM];
#pragma unroll
                for (int i = 0; i < DIM; ++i)
#pragma unroll
                    for (int k = 0; k < DIM; ++k) {
                        A[i][k] = __ldg(V1 + (size_t)fa[i] * DIM + k);
                        B[i][k] = __ldg(V1 + (size_t)fb[i] * DIM + k);
                    }
                if constexpr (DIM == 3) hit = tri_tri(A[0], A[1], A[2], B[0], B[1], B[2]);
                else hit = seg_seg(A[0], A[1], B[0], B[1]);
            }
            if (hit) {
                unsigned long long slot = warp_append(&cnt->n_discrete);
                if (slot < disc_cap) disc[slot] = pr;
            }
        }
    }
}

// Discrete test of leaf pairs [lo, hi) alone (default_discrete_test,
// BVHTree.cpp:464-500): the half of k_expand_pairs that gathers V1.
template <int DIM>
__global__ void __launch_bounds__(128)
k_discrete_pairs(const int2 *__restrict__ pairs, unsigned long long pair_cap, const int *__restrict__ P,
                 const double *__restrict__ V1, int nv, int2 *__restrict__ disc, unsigned long long disc_cap,
                 Counters *cnt, const unsigned long long *lo_ptr, const unsigned long long *hi_ptr)
{
    unsigned long long n = *(volatile const unsigned long long *)hi_ptr;
    if (n > pair_cap) n = pair_cap;
    unsigned long long lo = lo_ptr ? *(volatile const unsigned long long *)lo_ptr : 0ull;
    if (lo > n) lo = n;
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long idx = lo + (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n;
         idx += stride) {
        const int2 pr = pairs[idx];
        int fa[DIM], fb[DIM];
        bool inb = true;
#pragma unroll
        for (int k = 0; k < DIM; ++k) {
            fa[k] = __ldg(P + (size_t)pr.x * DIM + k);
            fb[k] = __ldg(P + (size_t)pr.y * DIM + k);
            inb = inb && fa[k] >= 0 && fa[k] < nv && fb[k] >= 0 && fb[k] < nv;
        }
        bool shared = false;
#pragma unroll
        for (int i = 0; i < DIM; ++i)
#pragma unroll
            for (int j = 0; j < DIM; ++j) shared |= fa[i] == fb[j];
        if (!inb) atomicOr(&cnt->err, kErrBadIndex);
        if (shared || !inb) continue;
        double A[DIM][DIM], B[DIM][DIM];
#pragma unroll
        for (int i = 0; i < DIM; ++i)
#pragma unroll
            for (int k = 0; k < DIM; ++k) {
                A[i][k] = __ldg(V1 + (size_t)fa[i] * DIM + k);
                B[i][k] = __ldg(V1 + (size_t)fb[i] * DIM + k);
            }
        int hit;
        if constexpr (DIM == 3) hit = tri_tri(A[0], A[1], A[2], B[0], B[1], B[2]);
        else hit = seg_seg(A[0], A[1], B[0], B[1]);
        if (hit) {
            const unsigned long long slot = warp_append(&cnt->n_discrete);
            if (slot < disc_cap) disc[slot] = pr;
        }
    }
}

// The same test with the lanes compacted: each warp reads 32 pairs per step,
// drops those that share a vertex (most leaf pairs of a mesh are neighbours)
// and queues the rest in shared memory; whenever 32 are queued the whole warp
// runs the test on them, so the V1 gathers and the test run on full warps.
template <int DIM>
__global__ void __launch_bounds__(128)
k_discrete_pairs_compact(const int2 *__restrict__ pairs, unsigned long long pair_cap, const int *__restrict__ P,
                         const double *__restrict__ V1, int nv, int2 *__restrict__ disc, unsigned long long disc_cap,
                         Counters *cnt, const unsigned long long *lo_ptr, const unsigned long long *hi_ptr)
{
    __shared__ int2 s_pr[4][64];
    __shared__ int s_v[4][64][2 * DIM];
    unsigned long long n = *(volatile const unsigned long long *)hi_ptr;
    if (n > pair_cap) n = pair_cap;
    unsigned long long lo = lo_ptr ? *(volatile const unsigned long long *)lo_ptr : 0ull;
    if (lo > n) lo = n;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned full = 0xffffffffu;
    auto test = [&](int slot) {
        double A[DIM][DIM], B[DIM][DIM];
#pragma unroll
        for (int i = 0; i < DIM; ++i) {
            const int a = s_v[w][slot][i], b = s_v[w][slot][DIM + i];
#pragma unroll
            for (int k = 0; k < DIM; ++k) {
                A[i][k] = __ldg(V1 + (size_t)a * DIM + k);
                B[i][k] = __ldg(V1 + (size_t)b * DIM + k);
            }
        }
        int hit;
        if constexpr (DIM == 3) hit = tri_tri(A[0], A[1], A[2], B[0], B[1], B[2]);
        else hit = seg_seg(A[0], A[1], B[0], B[1]);
        if (hit) {
            const unsigned long long slot_out = warp_append(&cnt->n_discrete);
            if (slot_out < disc_cap) disc[slot_out] = s_pr[w][slot];
        }
    };
    int queued = 0;   // warp-uniform
    const unsigned long long wstride = (unsigned long long)gridDim.x * 4 * 32;
    for (unsigned long long base = lo + ((unsigned long long)blockIdx.x * 4 + w) * 32; base < n; base += wstride) {
        const unsigned long long idx = base + lane;
        bool keep = idx < n;
        int2 pr = make_int2(0, 0);
        int fa[DIM], fb[DIM];
        if (keep) {
            pr = pairs[idx];
            bool inb = true;
#pragma unroll
            for (int k = 0; k < DIM; ++k) {
                fa[k] = __ldg(P + (size_t)pr.x * DIM + k);
                fb[k] = __ldg(P + (size_t)pr.y * DIM + k);
                inb = inb && fa[k] >= 0 && fa[k] < nv && fb[k] >= 0 && fb[k] < nv;
            }
            bool shared = false;
#pragma unroll
            for (int i = 0; i < DIM; ++i)
#pragma unroll
                for (int j = 0; j < DIM; ++j) shared |= fa[i] == fb[j];
            if (!inb) atomicOr(&cnt->err, kErrBadIndex);
            keep = inb && !shared;
        }
        const unsigned m = __ballot_sync(full, keep);
        if (keep) {
            const int pos = queued + __popc(m & lanemask_lt());   // < 31 + 32 = 63
            s_pr[w][pos] = pr;
#pragma unroll
            for (int k = 0; k < DIM; ++k) { s_v[w][pos][k] = fa[k]; s_v[w][pos][DIM + k] = fb[k]; }
        }
        queued += __popc(m);
        __syncwarp();
        if (queued >= 32) {
            test(lane);
            __syncwarp();
            queued -= 32;   // move entries 32 .. 32 + queued - 1 to the front
            if (lane < queued) {
                s_pr[w][lane] = s_pr[w][32 + lane];
#pragma unroll
                for (int k = 0; k < 2 * DIM; ++k) s_v[w][lane][k] = s_v[w][32 + lane][k];
            }
            __syncwarp();
        }
    }
    if (lane < queued) test(lane);
}

void launch_discrete_pairs(int dim, const int2 *pairs, unsigned long long pair_cap, const int *P, const double *V1,
                           int nv, int2 *disc, unsigned long long disc_cap, Counters *cnt, int grid, cudaStream_t st,
                           const unsigned long long *lo_ptr, const unsigned long long *hi_ptr, bool compact)
{
    if (!hi_ptr) hi_ptr = &cnt->n_pairs;
    if (compact) {
        if (dim == 3)
            k_discrete_pairs_compact<3><<<grid, 128, 0, st>>>(pairs, pair_cap, P, V1, nv, disc, disc_cap, cnt, lo_ptr,
                                                              hi_ptr);
        else
            k_discrete_pairs_compact<2><<<grid, 128, 0, st>>>(pairs, pair_cap, P, V1, nv, disc, disc_cap, cnt, lo_ptr,
                                                              hi_ptr);
        return;
    }
    if (dim == 3)
        k_discrete_pairs<3><<<grid, 128, 0, st>>>(pairs, pair_cap, P, V1, nv, disc, disc_cap, cnt, lo_ptr, hi_ptr);
    else
        k_discrete_pairs<2><<<grid, 128, 0, st>>>(pairs, pair_cap, P, V1, nv, disc, disc_cap, cnt, lo_ptr, hi_ptr);
}

void launch_traverse_refill(int dim, int window, const Node *nodes, const void *leaf_box,
                            const unsigned char *leaf_active, const int *sorted, int n, int2 *pairs,
                            unsigned long long cap, Counters *cnt, unsigned *cursor, cudaStream_t st, int q_begin,
                            int q_end)
{
    if (n < 2) return;
    if (q_end < 0 || q_end > n - 1) q_end = n - 1;
    if (q_begin >= q_end) return;
    // persistent: one wave of resident blocks, fewer for short ranges
    const long long warps_needed = ((long long)(q_end - q_begin) + 31) / 32;
    const int g = (int)std::max<long long>(1, std::min<long long>(148 * 4, (warps_needed + 3) / 4));
    cudaMemsetAsync(cursor, 0, sizeof(unsigned), st);
    const auto *lb3 = reinterpret_cast<const LeafBox<3> *>(leaf_box);
    const auto *lb2 = reinterpret_cast<const LeafBox<2> *>(leaf_box);
#define MCLCCD_REFILL_CASE(Wv)                                                                                     \
    case Wv:                                                                                                       \
        if (dim == 3)                                                                                              \
            k_traverse_refill<3, Wv><<<g, 128, 0, st>>>(nodes, lb3, leaf_active, sorted, n, q_begin, q_end, pairs,  \
                                                         cap, cnt, cursor);                                         \
        else                                                                                                       \
            k_traverse_refill<2, Wv><<<g, 128, 0, st>>>(nodes, lb2, leaf_active, sorted, n, q_begin, q_end, pairs,  \
                                                         cap, cnt, cursor);                                         \
        return;
    // (the per-warp staging of 32 + W boxes keeps W <= 32 within static shared memory)
    switch (window) {
        MCLCCD_REFILL_CASE(8)
        MCLCCD_REFILL_CASE(32)
    default:
        MCLCCD_REFILL_CASE(16)
    }
#undef MCLCCD_REFILL_CASE
}

void launch_traverse_buffered(int dim, int window, int run, const Node *nodes, const void *leaf_box,
                              const unsigned char *leaf_active, const int *sorted, int n, int2 *pairs,
                              unsigned long long cap, Counters *cnt, cudaStream_t st, int q_begin, int q_end)
{
    if (n < 2) return;
    if (q_end < 0 || q_end > n - 1) q_end = n - 1;
    if (q_begin >= q_end) return;
    const int g = (q_end - q_begin + 127) / 128;
    const auto *lb3 = reinterpret_cast<const LeafBox<3> *>(leaf_box);
    const auto *lb2 = reinterpret_cast<const LeafBox<2> *>(leaf_box);
#define MCLCCD_BUF_CASE(Wv)                                                                                        \
    case Wv:                                                                                                       \
        if (run >= 64) {                                                                                           \
            if (dim == 3)                                                                                          \
                k_traverse_window_buf<3, Wv, 64><<<g, 128, 0, st>>>(nodes, lb3, leaf_active, sorted, n, q_begin,    \
                                                                     q_end, pairs, cap, cnt);                       \
            else                                                                                                   \
                k_traverse_window_buf<2, Wv, 64><<<g, 128, 0, st>>>(nodes, lb2, leaf_active, sorted, n, q_begin,    \
                                                                     q_end, pairs, cap, cnt);                       \
        } else if (dim == 3) {                                                                                     \
            k_traverse_window_buf<3, Wv><<<g, 128, 0, st>>>(nodes, lb3, leaf_active, sorted, n, q_begin, q_end,     \
                                                             pairs, cap, cnt);                                      \
        } else {                                                                                                   \
            k_traverse_window_buf<2, Wv><<<g, 128, 0, st>>>(nodes, lb2, leaf_active, sorted, n, q_begin, q_end,     \
                                                             pairs, cap, cnt);                                      \
        }                                                                                                          \
        return;
    switch (window) {
        MCLCCD_BUF_CASE(8)
        MCLCCD_BUF_CASE(32)
    default:
        MCLCCD_BUF_CASE(16)
    }
#undef MCLCCD_BUF_CASE
}

void launch_traverse(int dim, int packet, int window, const Node *nodes, const void *leaf_box,
                     const unsigned char *leaf_active, const int *sorted, int n, int2 *pairs, unsigned long long cap,
                     Counters *cnt, cudaStream_t st, int q_begin, int q_end)
{
    if (n < 2) return;
    if (q_end < 0 || q_end > n - 1) q_end = n - 1;
    if (q_begin >= q_end) return;
    const int g = (q_end - q_begin + 127) / 128;
    const auto *lb3 = reinterpret_cast<const LeafBox<3> *>(leaf_box);
    const auto *lb2 = reinterpret_cast<const LeafBox<2> *>(leaf_box);
    if (window) {
#define MCLCCD_WINDOW_CASE(Wv)                                                                                     \
    case Wv:                                                                                                       \
        cudaFuncSetAttribute(k_traverse_window<3, Wv>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);        \
        cudaFuncSetAttribute(k_traverse_window<2, Wv>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);        \
        if (dim == 3)                                                                                              \
            k_traverse_window<3, Wv><<<g, 128, 0, st>>>(nodes, lb3, leaf_active, sorted, n, q_begin, q_end, pairs,  \
                                                         cap, cnt);                                                 \
        else                                                                                                       \
            k_traverse_window<2, Wv><<<g, 128, 0, st>>>(nodes, lb2, leaf_active, sorted, n, q_begin, q_end, pairs,  \
                                                         cap, cnt);                                                 \
        return;
        switch (window) {
            MCLCCD_WINDOW_CASE(8)
            MCLCCD_WINDOW_CASE(16)
            MCLCCD_WINDOW_CASE(32)
            MCLCCD_WINDOW_CASE(64)
            MCLCCD_WINDOW_CASE(128)
        }
#undef MCLCCD_WINDOW_CASE
    }
    if (packet) {
        if (dim == 3) k_traverse_packet<3><<<g, 128, 0, st>>>(nodes, lb3, leaf_active, sorted, n, pairs, cap, cnt);
        else k_traverse_packet<2><<<g, 128, 0, st>>>(nodes, lb2, leaf_active, sorted, n, pairs, cap, cnt);
    } else {
        if (dim == 3) k_traverse<3><<<g, 128, 0, st>>>(nodes, lb3, leaf_active, sorted, n, q_begin, q_end, pairs, cap, cnt);
        else k_traverse<2><<<g, 128, 0, st>>>(nodes, lb2, leaf_active, sorted, n, q_begin, q_end, pairs, cap, cnt);
    }
}

void launch_expand_pairs(int dim, const int2 *pairs, unsigned long long pair_cap, const int *P,
                         const unsigned char *flags, const double *V1, int nv, int4 *vf, unsigned long long vf_cap,
                         int4 *ee, unsigned long long ee_cap, int2 *disc, unsigned long long disc_cap, int continuous,
                         int discrete, Counters *cnt, int grid, cudaStream_t st, const unsigned long long *lo_ptr,
                         const unsigned long long *hi_ptr)
{
    if (!hi_ptr) hi_ptr = &cnt->n_pairs;
    if (!discrete) {   // stencils only: the lean instantiation
        if (dim == 3)
            k_expand_pairs<3, false><<<grid, 256, 0, st>>>(pairs, pair_cap, P, flags, V1, nv, vf, vf_cap, ee, ee_cap,
                                                           disc, disc_cap, continuous, 0, cnt, lo_ptr, hi_ptr);
        else
            k_expand_pairs<2, false><<<grid, 256, 0, st>>>(pairs, pair_cap, P, flags, V1, nv, vf, vf_cap, ee, ee_cap,
                                                           disc, disc_cap, continuous, 0, cnt, lo_ptr, hi_ptr);
        return;
    }
    if (dim == 3)
        k_expand_pairs<3><<<grid, 256, 0, st>>>(pairs, pair_cap, P, flags, V1, nv, vf, vf_cap, ee, ee_cap, disc,
                                                disc_cap, continuous, discrete, cnt, lo_ptr, hi_ptr);
    else
        k_expand_pairs<2><<<grid, 256, 0, st>>>(pairs, pair_cap, P, flags, V1, nv, vf, vf_cap, ee, ee_cap, disc,
                                                disc_cap, continuous, discrete, cnt, lo_ptr, hi_ptr);
}

// dst[i] = *src[i]: a snapshot of running counters between two launches.
__global__ void k_snapshot(const unsigned long long *a, unsigned long long *da, const unsigned long long *b,
                           unsigned long long *db)
{
    *da = *(volatile const unsigned long long *)a;
    if (b) *db = *(volatile const unsigned long long *)b;
}

void launch_snapshot(const unsigned long long *a, unsigned long long *da, const unsigned long long *b,
                     unsigned long long *db, cudaStream_t st)
{
    k_snapshot<<<1, 1, 0, st>>>(a, da, b, db);
}

} // namespace mclccd
