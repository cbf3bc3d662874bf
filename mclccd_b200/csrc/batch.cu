// Batched CCD: many independent scenes of uneven sizes per step.
//
// Per dimension group (3D triangle meshes, 2D edge meshes), all scenes'
// primitives live in one array, scene by scene.  The hierarchy is a
// segmented LBVH: Morton codes against each scene's own centroid bounds, a
// stable two-stage radix sort (Morton code, then scene id) that leaves every
// scene's leaves contiguous in Morton order, and one Karras tree per scene
// built by a single launch over all internal nodes (node indices are local to
// the scene, offset by the scene's base).  Refit is the usual bottom-up pass
// with per-scene thickness.
//
// Traversal and narrow phase run in waves over the query leaves, all inside
// one CUDA graph: a conditional WHILE node repeats one wave -- the walk of a
// range of queries through their scenes' trees (the single-scene walk with
// scene offsets; pairs k > q only, so each unordered pair once) into a
// leaf-pair buffer, the single-scene stencil expansion (with the discrete
// test), and ACCD over the VF and EE lists -- until every query is done.  A
// device-side controller sizes the waves: a wave whose pairs or stencils
// overflow their buffers is voided and redone with half the queries, and
// waves that use under a quarter of the buffers double.  No hit list is
// materialised: per scene the ACCD and discrete kernels accumulate candidate,
// hit and discrete counts, the earliest hit (a 128-bit compare-and-swap on
// its (toi, kind, v0, v1) key plus a log of ties), and the time the scene's
// last work finished.
//
// Per-pair and per-stencil results are those of the single-scene path: same
// leaf predicate, same canonical pair orientation, same stencil expansion and
// the same ACCD (FP64, or FP32-certified with FP64 fallback inline).
#include <algorithm>
#include <cstring>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "common.cuh"
#include "geom.cuh"
#include "kernels.cuh"
#include "lbvh.cuh"
#include "cert.cuh"
#include "mclccd_b200.h"

namespace mclccd {

// Scene's earliest hit key: toi bits, then k1 = (EE flag, v0, v1).
struct __align__(16) BestKey {
    unsigned long long toi, k1;
};

struct BatchRecord {
    int4 sten;
    double toi;
    int scene;    // group-local scene index, | kRecGroup3 for the 3D group
    int is_vf;
};
constexpr int kRecGroup3 = 1 << 28;

// Device view of one dimension group.
struct BatchGroupDev {
    int np, nv, n_scenes;
    const double *V0, *V1;
    const int *P;                   // np x DIM, group vertex ids
    const unsigned char *flags;     // representative flags per primitive
    const int *prim_scene;          // group scene of each primitive
    const int *sorted;              // sorted leaf -> primitive
    const int *leaf_off, *node_off, *scene_np;
    const double *eta;
    const Node *nodes;
    const void *leaf_box;
    const unsigned char *leaf_active;
    unsigned long long *queue;      // persistent form: next query to hand out
    unsigned long long *n_hits, *n_disc, *n_sten, *done_ns;
    BestKey *best;
    BatchRecord *rec;
    unsigned long long *n_rec;
    unsigned long long rec_cap;
    unsigned *err;
    int chunk, leaf_size;
};

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// ---------------------------------------------------------------------------
// Build kernels.
// ---------------------------------------------------------------------------
__global__ void k_b_stamp(unsigned long long *t) { *t = global_ns(); }

template <int DIM>
__global__ void k_b_init_bounds_dim(unsigned *bounds, int n_scenes)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_scenes * 2 * DIM; i += gridDim.x * blockDim.x)
        bounds[i] = (i % (2 * DIM)) < DIM ? 0xff800000u : 0x007fffffu;   // ordered(+inf) / ordered(-inf)
}

template <int DIM>
__global__ void k_b_centroids(const double *__restrict__ V0, const double *__restrict__ V1, const int *__restrict__ P,
                              int np, int nv, const int *__restrict__ prim_scene, float *__restrict__ cent,
                              unsigned *bounds, unsigned *err)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += gridDim.x * blockDim.x) {
        LeafBox<DIM> b;
        bool act;
        if (!compute_leaf_box<DIM>(V0, V1, P, DIM, nv, i, 0.0, nullptr, b, act)) atomicOr(err, kErrBadIndex);
        const int s = prim_scene[i];
        float c[DIM];
#pragma unroll
        for (int k = 0; k < DIM; ++k) {
            double mn = b.lo0[k] < b.lo1[k] ? b.lo0[k] : b.lo1[k];
            double mx = b.hi0[k] < b.hi1[k] ? b.hi1[k] : b.hi0[k];
            c[k] = (float)(0.5 * (mn + mx));
            if (!(c[k] == c[k]) || fabsf(c[k]) > 3.0e38f) c[k] = 0.f;
            cent[(size_t)i * DIM + k] = c[k];
        }
        // lanes of one scene reduce first (primitives are grouped by scene)
        const unsigned peers = __match_any_sync(__activemask(), s);
        const int leader = __ffs(peers) - 1;
#pragma unroll
        for (int k = 0; k < DIM; ++k) {
            float lo = c[k], hi = c[k];
            for (unsigned m = peers; m; m &= m - 1) {
                const int src = __ffs(m) - 1;
                lo = fminf(lo, __shfl_sync(peers, c[k], src));
                hi = fmaxf(hi, __shfl_sync(peers, c[k], src));
            }
            if ((int)lane_id() == leader) {
                atomicMin(bounds + (size_t)s * 2 * DIM + k, float_to_ordered(lo));
                atomicMax(bounds + (size_t)s * 2 * DIM + DIM + k, float_to_ordered(hi));
            }
        }
    }
}

template <int DIM>
__global__ void k_b_morton(const float *__restrict__ cent, int np, const int *__restrict__ prim_scene,
                           const unsigned *__restrict__ bounds, unsigned *__restrict__ mort,
                           unsigned *__restrict__ keys, int *__restrict__ vals)
{
    constexpr float kCells = DIM == 3 ? 1024.f : 32768.f;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += gridDim.x * blockDim.x) {
        const unsigned *b = bounds + (size_t)prim_scene[i] * 2 * DIM;
        unsigned code = 0;
#pragma unroll
        for (int k = 0; k < DIM; ++k) {
            const float lo = ordered_to_float(b[k]);
            const float ext = ordered_to_float(b[DIM + k]) - lo;
            const float inv = ext > 0.f ? kCells / ext : 0.f;
            const float q = (cent[(size_t)i * DIM + k] - lo) * inv;
            const unsigned u = (unsigned)fminf(fmaxf(q, 0.f), kCells - 1.f);
            code |= (DIM == 3 ? expand_bits3(u) : expand_bits2(u)) << (DIM == 3 ? 2 - k : 1 - k);
        }
        mort[i] = code;
        keys[i] = code;
        vals[i] = i;
    }
}

// keys[i] = table[vals[i]]
__global__ void k_b_gather_keys(const int *__restrict__ vals, const unsigned *__restrict__ table, int n,
                                unsigned *__restrict__ keys)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) keys[i] = table[vals[i]];
}

__device__ __forceinline__ int kdelta_l(const unsigned *__restrict__ keys, int n, int i, int j)
{
    if (j < 0 || j >= n) return -1;
    const unsigned a = keys[i], b = keys[j];
    return a == b ? 32 + __clz(i ^ j) : __clz(a ^ b);
}

// One Karras tree per scene (HPG 2012), over all scenes' internal nodes in
// one launch.  Indices stored in the nodes are local to the scene; pad.x
// holds the node's first leaf (the range is [first, last]).
__global__ void k_b_karras(const unsigned *__restrict__ keys, int n_int, const int *__restrict__ node_scene,
                           const int *__restrict__ leaf_off, const int *__restrict__ node_off,
                           const int *__restrict__ scene_np, Node *__restrict__ nodes, int *__restrict__ leaf_parent)
{
    for (int gi = blockIdx.x * blockDim.x + threadIdx.x; gi < n_int; gi += gridDim.x * blockDim.x) {
        const int s = node_scene[gi];
        const int n = scene_np[s], i = gi - node_off[s];
        const unsigned *kl = keys + leaf_off[s];
        Node *nl = nodes + node_off[s];
        int *lp = leaf_parent + leaf_off[s];
        const int d = (kdelta_l(kl, n, i, i + 1) - kdelta_l(kl, n, i, i - 1)) >= 0 ? 1 : -1;
        const int dmin = kdelta_l(kl, n, i, i - d);
        int lmax = 2;
        while (kdelta_l(kl, n, i, i + lmax * d) > dmin) lmax <<= 1;
        int l = 0;
        for (int t = lmax >> 1; t >= 1; t >>= 1)
            if (kdelta_l(kl, n, i, i + (l + t) * d) > dmin) l += t;
        const int j = i + l * d;
        const int dnode = kdelta_l(kl, n, i, j);
        int sp = 0, t = l;
        for (;;) {
            t = (t + 1) >> 1;
            if (kdelta_l(kl, n, i, i + (sp + t) * d) > dnode) sp += t;
            if (t <= 1) break;
        }
        const int gamma = i + sp * d + (d < 0 ? -1 : 0);
        const int first = min(i, j), last = max(i, j);
        if (gamma < first || gamma >= last) continue;   // cannot happen for sorted keys
        const bool lleaf = first == gamma, rleaf = last == gamma + 1;
        Node &nd = nl[i];
        nd.d.x = gamma;
        nd.d.y = (lleaf ? kMetaLeftLeaf : 0) | (rleaf ? kMetaRightLeaf : 0);
        nd.d.z = last;
        nd.pad.x = first;
        if (i == 0) nd.d.w = -1;
        if (lleaf) lp[gamma] = i; else nl[gamma].d.w = i;
        if (rleaf) lp[gamma + 1] = i; else nl[gamma + 1].d.w = i;
    }
}

template <int DIM>
__global__ void k_b_refit(const double *__restrict__ V0, const double *__restrict__ V1, const int *__restrict__ P,
                          int np, int nv, const int *__restrict__ prim_scene, const int *__restrict__ sorted,
                          const int *__restrict__ leaf_off, const int *__restrict__ node_off,
                          const int *__restrict__ scene_np, const double *__restrict__ eta,
                          const int *__restrict__ leaf_parent, Node *nodes, int *__restrict__ visits,
                          LeafBox<DIM> *__restrict__ leaf_box, unsigned char *__restrict__ leaf_active, unsigned *err)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= np) return;
    const int prim = sorted[k];
    const int s = prim_scene[prim];
    LeafBox<DIM> b;
    bool act;
    if (!compute_leaf_box<DIM>(V0, V1, P, DIM, nv, prim, eta[s], nullptr, b, act)) atomicOr(err, kErrBadIndex);
    leaf_box[k] = b;
    leaf_active[k] = 1;
    if (scene_np[s] < 2) return;
    const int lk = k - leaf_off[s];
    Node *nl = nodes + node_off[s];
    int *vis = visits + node_off[s];
    Box2T<DIM> box = outward<DIM>(b);
    int parent = leaf_parent[k];
    bool right = __ldg(&nl[parent].d.x) != lk;
    write_child<DIM>(nl, parent, right, box, act);
    for (int level = 0; level < 256; ++level) {
        if (!refit_second_arrival(vis + parent)) return;
        const int node = parent;
        merge_sibling<DIM>(nl + node, right, box, act);
        parent = __ldcg(&nl[node].d.w);
        if (parent < 0) return;
        const int psplit = __ldg(&nl[parent].d.x);
        const int pmeta = __ldg(&nl[parent].d.y) & 0xff;
        right = !(psplit == node && !(pmeta & kMetaLeftLeaf));
        write_child<DIM>(nl, parent, right, box, act);
    }
    atomicOr(err, kErrStack);
}

// Scatter of the caller's per-scene vertex arrays into the group arrays:
// dst[dst_off[s] + i] = src[src_off[s] + i] for the scene owning each slot.
__global__ void k_b_scatter(const double *__restrict__ src, double *__restrict__ dst, long long n,
                            const long long *__restrict__ dst_off, const long long *__restrict__ src_off, int n_scenes)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        int lo = 0, hi = n_scenes - 1;   // last scene with dst_off <= i
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (dst_off[mid] <= i) lo = mid; else hi = mid - 1;
        }
        dst[i] = src[src_off[lo] + (i - dst_off[lo])];
    }
}

// ---------------------------------------------------------------------------
// Waves: segmented walk -> stencil expansion -> ACCD with per-scene
// reductions, repeated over the queries by a device-driven loop.
// ---------------------------------------------------------------------------
constexpr unsigned kFull = 0xffffffffu;
constexpr int kScanFlag = 1 << 30;

// Per-scene sums over the lanes of a warp that share a scene: one atomic per
// scene.  All 32 lanes must call; scene < 0 contributes nothing.
__device__ __forceinline__ void scene_add(unsigned long long *arr, int scene, unsigned v)
{
    const unsigned peers = __match_any_sync(kFull, scene);
    const unsigned sum = __reduce_add_sync(peers, v);
    if (scene >= 0 && sum && (int)lane_id() == __ffs(peers) - 1) atomicAdd(arr + scene, (unsigned long long)sum);
}

__device__ __forceinline__ void scene_touch(unsigned long long *done_ns, int scene)
{
    const unsigned peers = __match_any_sync(kFull, scene);
    if (scene >= 0 && (int)lane_id() == __ffs(peers) - 1) atomicMax(done_ns + scene, global_ns());
}

template <int DIM, bool CERT>
__device__ __forceinline__ int batch_accd(const int (&s)[4], bool vf, const BatchGroupDev &g, double eta, double &toi)
{
    double x0[DIM + 1][DIM], x1[DIM + 1][DIM];
    if (!gather_c<DIM>(s, g.V0, g.V1, g.nv, x0, x1)) { atomicOr(g.err, kErrBadIndex); return 0; }
    toi = -1.0;
    int iters = 0, hit;
    if constexpr (CERT) {
        bool bound;
        const int c = (DIM == 3 && !vf) ? accd_certified<DIM, false>(x0, x1, eta, toi, bound)
                                         : accd_certified<DIM, true>(x0, x1, eta, toi, bound);
        if (c != kCertFallback) return c == kCertHit;
    }
    if (DIM == 3 && !vf) hit = accd<DIM, false>(x0, x1, eta, toi, iters);
    else hit = accd<DIM, true>(x0, x1, eta, toi, iters);
    if (iters >= 1000) atomicOr(g.err, kErrAccdIters);
    return hit;
}

// The scene's earliest hit under the order (toi, VF before EE, v0, v1, v2,
// v3): the lanes of one scene reduce to their smallest key, whose leader
// merges it into the scene's 16-byte (toi, k1) minimum with a
// compare-and-swap loop; hits that install or tie that minimum are logged
// with v2, v3 for the final choice among equal (toi, k1).  All lanes call;
// hs = the hit's scene or -1.
template <int DIM>
__device__ __forceinline__ void scene_best(const BatchGroupDev &g, int hs, double toi, const int (&s4)[4], bool vf)
{
    const int lane = lane_id();
    const unsigned long long kt = hs >= 0 ? (unsigned long long)__double_as_longlong(toi) : ~0ull;
    // cheap filter: only hits at or below the scene's current minimum contend
    const bool cand = hs >= 0 && kt <= *(volatile const unsigned long long *)&g.best[hs].toi;
    if (!__any_sync(kFull, cand)) return;
    const int cs = cand ? hs : -1;
    const unsigned long long k1 = cand ? ((unsigned long long)(vf ? 0 : 1) << 63) |
                                             ((unsigned long long)(unsigned)s4[0] << 32) | (unsigned)s4[1]
                                       : ~0ull;
    const unsigned long long k2 = ((unsigned long long)(unsigned)s4[2] << 32) | (unsigned)s4[3];
    const unsigned long long kc = cand ? kt : ~0ull;
    const unsigned peers = __match_any_sync(kFull, cs);
    unsigned long long bt = kc, b1 = k1, b2 = k2;
    for (unsigned m = peers; m; m &= m - 1) {
        const int src = __ffs(m) - 1;
        const unsigned long long ot = __shfl_sync(peers, kc, src), o1 = __shfl_sync(peers, k1, src),
                                 o2 = __shfl_sync(peers, k2, src);
        if (ot < bt || (ot == bt && (o1 < b1 || (o1 == b1 && o2 < b2)))) { bt = ot; b1 = o1; b2 = o2; }
    }
    if (cs < 0 || lane != __ffs(peers) - 1) return;
    BestKey mine{bt, b1};
    BestKey cur = atomicCAS(g.best + cs, BestKey{0ull, 0ull}, BestKey{0ull, 0ull});   // atomic read
    bool keep = false;
    for (int it = 0; it < 1024; ++it) {
        if (cur.toi < mine.toi || (cur.toi == mine.toi && cur.k1 <= mine.k1)) {
            keep = cur.toi == mine.toi && cur.k1 == mine.k1;   // tie with the stored minimum
            break;
        }
        const BestKey prev = atomicCAS(g.best + cs, cur, mine);
        if (prev.toi == cur.toi && prev.k1 == cur.k1) { keep = true; break; }
        cur = prev;
    }
    if (keep) {
        const unsigned long long r = atomicAdd(g.n_rec, 1ull);
        if (r < g.rec_cap) {
            const double t = __longlong_as_double((long long)bt);
            const int v0 = (int)((b1 >> 32) & 0x7fffffffu), v1 = (int)(unsigned)b1;
            g.rec[r] = BatchRecord{make_int4(v0, v1, (int)(unsigned)(b2 >> 32), (int)(unsigned)b2), t,
                                   cs | (DIM == 3 ? kRecGroup3 : 0), (b1 >> 63) ? 0 : 1};
        }
    }
}

// Device state of a group's wave loop.
struct WaveState {
    unsigned long long cursor;        // first query not yet done
    unsigned long long q0, q1;        // this wave's queries
    unsigned long long wave_q;        // queries per wave (adapted, kept across runs)
    unsigned long long waves, redos;
    unsigned long long used_pairs, used_vf, used_ee;
    int redo, stop;
};

__global__ void k_wave_init(WaveState *ws, unsigned long long initial_q)
{
    ws->cursor = 0;
    if (ws->wave_q == 0) ws->wave_q = initial_q;
    ws->waves = ws->redos = 0;
    ws->stop = 0;
}

__global__ void k_wave_begin(WaveState *ws, Counters *wc, unsigned long long n_total)
{
    wc->n_pairs = wc->n_vf = wc->n_ee = wc->n_discrete = 0;
    ws->q0 = ws->cursor;
    const unsigned long long q1 = ws->cursor + ws->wave_q;
    ws->q1 = q1 < n_total ? q1 : n_total;
    ws->redo = 0;
}

// Overflowed buffers void the wave (the next kernels then see zero work).
__global__ void k_wave_check_pairs(WaveState *ws, Counters *wc, unsigned long long cap_pairs)
{
    ws->used_pairs = wc->n_pairs;
    if (wc->n_pairs > cap_pairs) { ws->redo = 1; wc->n_pairs = 0; }
}

__global__ void k_wave_check_sten(WaveState *ws, Counters *wc, unsigned long long cap_vf, unsigned long long cap_ee,
                                  unsigned long long cap_disc)
{
    ws->used_vf = wc->n_vf;
    ws->used_ee = wc->n_ee;
    if (ws->redo || wc->n_vf > cap_vf || wc->n_ee > cap_ee || wc->n_discrete > cap_disc) {
        ws->redo = 1;
        wc->n_vf = wc->n_ee = wc->n_discrete = 0;
    }
}

// Advances the loop and sizes the next wave from this one's demand: the
// fullest buffer (pairs, VF or EE stencils; the counters keep counting past
// capacity) should come to about 60% full: pair density grows along the
// small-first scene order, and a redo costs a wasted walk.  A voided wave is
// redone with at most half its queries; a done wave moves the cursor and may
// grow the next one up to 2x.  Sets the loop condition.  A single query that cannot fit,
// or a runaway loop, stops it with an error.
__global__ void k_wave_end(WaveState *ws, unsigned long long n_total, unsigned long long cap_pairs,
                           unsigned long long cap_vf, unsigned long long cap_ee, cudaGraphConditionalHandle handle,
                           unsigned *err)
{
    const unsigned long long nq = ws->q1 - ws->q0;
    double fill = (double)ws->used_pairs / (double)cap_pairs;
    fill = fmax(fill, (double)ws->used_vf / (double)cap_vf);
    if (cap_ee) fill = fmax(fill, (double)ws->used_ee / (double)cap_ee);
    if (ws->redo) {
        ++ws->redos;
        if (nq <= 1) { atomicOr(err, kErrWave); ws->stop = 1; }
        else {
            double q = fill > 1.0 ? (double)nq * (0.6 / fill) : 0.5 * (double)nq;
            q = fmin(q, 0.5 * (double)nq);
            ws->wave_q = q < 1.0 ? 1ull : (unsigned long long)q;
        }
    } else {
        ws->cursor = ws->q1;
        ++ws->waves;
        const double grow = fill > 0.3 ? 0.6 / fill : 2.0;
        const double q = (double)nq * grow;
        ws->wave_q = q < 1.0 ? 1ull : q > (double)n_total ? n_total : (unsigned long long)q;
    }
    if (ws->waves + ws->redos > (1ull << 24)) { atomicOr(err, kErrWave); ws->stop = 1; }
    cudaGraphSetConditional(handle, (!ws->stop && ws->cursor < n_total) ? 1u : 0u);
}

// Walk of this wave's queries (one per thread, grid-stride), each in its
// scene's tree: the single-scene walk with scene offsets, plus scanning
// subtrees of at most leaf_size leaves instead of descending them.
template <int DIM, int STACK>
__global__ void __launch_bounds__(256)
k_b_walk(BatchGroupDev g, const WaveState *ws, int2 *__restrict__ pairs, unsigned long long cap, Counters *wc)
{
    constexpr int S = DIM == 3 ? 3 : 2;
    extern __shared__ int s_stack[];   // [STACK][blockDim.x]
    const LeafBox<DIM> *lbox = reinterpret_cast<const LeafBox<DIM> *>(g.leaf_box);
    const unsigned long long q0 = ws->q0, q1 = ws->q1;
    const int tid = threadIdx.x, bs = blockDim.x;
    for (unsigned long long qi = q0 + (unsigned long long)blockIdx.x * bs + tid; qi < q1;
         qi += (unsigned long long)gridDim.x * bs) {
        const int q = (int)qi;
        const int qprim = g.sorted[q];
        const int sc = g.prim_scene[qprim];
        const int lb = g.leaf_off[sc], nb = g.node_off[sc], ns = g.scene_np[sc];
        const int lq = q - lb;
        if (ns < 2 || lq >= ns - 1) continue;
        Box2T<DIM> qbox;
        {
            const LeafBox<DIM> &qb = lbox[q];
#pragma unroll
            for (int k = 0; k < DIM; ++k) {
                qbox.t0lo[k] = __double2float_rd(qb.lo0[k]); qbox.t0hi[k] = __double2float_ru(qb.hi0[k]);
                qbox.t1lo[k] = __double2float_rd(qb.lo1[k]); qbox.t1hi[k] = __double2float_ru(qb.hi1[k]);
            }
        }
        auto emit = [&](int k, int r) {   // local leaf k, three-valued test result r
            if (r == 2) r = leaf_boxes_intersect<DIM>(lbox[q], lbox[lb + k]) ? 1 : 0;
            if (r == 1) {
                const int kprim = __ldg(g.sorted + lb + k);
                const unsigned long long slot = warp_append(&wc->n_pairs);
                if (slot < cap) pairs[slot] = make_int2(min(qprim, kprim), max(qprim, kprim));
            }
        };
        auto test_leaf = [&](int k) {
            const LeafBox<DIM> &kb = lbox[lb + k];
            Box2T<DIM> kbox;
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                kbox.t0lo[d] = __double2float_rd(kb.lo0[d]); kbox.t0hi[d] = __double2float_ru(kb.hi0[d]);
                kbox.t1lo[d] = __double2float_rd(kb.lo1[d]); kbox.t1hi[d] = __double2float_ru(kb.hi1[d]);
            }
            emit(k, leaf_test3<DIM>(qbox, inner<DIM>(qbox), kbox));
        };
        int sp = 0, node = 0, scan_k = 1, scan_end = 0;
        bool have_node = true;
        for (long long steps = 0;; ++steps) {
            if (steps > 4ll * ns + 64) { atomicOr(g.err, kErrStack); break; }
            if (scan_k <= scan_end) { test_leaf(scan_k++); continue; }
            if (!have_node) {
                if (sp == 0) break;
                const int e = s_stack[(--sp) * bs + tid];
                if (e & kScanFlag) {
                    const int c = e & ~kScanFlag;
                    scan_k = max(__ldg(&g.nodes[nb + c].pad.x), lq + 1);
                    scan_end = __ldg(&g.nodes[nb + c].d.z);
                } else {
                    node = e;
                    have_node = true;
                }
                continue;
            }
            const Node *nd = g.nodes + nb + node;
            float4 ls[S], rs[S];
#pragma unroll
            for (int i = 0; i < S; ++i) { ls[i] = __ldg(&nd->l[i]); rs[i] = __ldg(&nd->r[i]); }
            const int4 d = __ldg(&nd->d);
            const int first = __ldg(&nd->pad.x);
            const int split = d.x, meta = d.y, last = d.z;
            Box2T<DIM> lbx, rbx;
            unpack_child<DIM>(ls, lbx);
            unpack_child<DIM>(rs, rbx);
            bool lok = split > lq, rok = last > lq;   // every batch leaf is active
            if (lok && (meta & kMetaLeftLeaf)) { emit(split, leaf_test3<DIM>(qbox, inner<DIM>(qbox), lbx)); lok = false; }
            if (rok && (meta & kMetaRightLeaf)) { emit(split + 1, leaf_test3<DIM>(qbox, inner<DIM>(qbox), rbx)); rok = false; }
            lok = lok && boxes_may_intersect<DIM>(qbox, lbx);
            rok = rok && boxes_may_intersect<DIM>(qbox, rbx);
            const bool lscan = lok && split - first + 1 <= g.leaf_size;
            const bool rscan = rok && last - split <= g.leaf_size;
            have_node = false;
            if (lok && rok) {
                if (sp < STACK) s_stack[(sp++) * bs + tid] = rscan ? ((split + 1) | kScanFlag) : split + 1;
                else { atomicOr(g.err, kErrStack); break; }
            }
            if (lok) {
                if (lscan) { scan_k = max(first, lq + 1); scan_end = split; }
                else { node = split; have_node = true; }
            } else if (rok) {
                if (rscan) { scan_k = max(split + 1, lq + 1); scan_end = last; }
                else { node = split + 1; have_node = true; }
            }
        }
    }
}

// Per-lane running sums for one scene, flushed (warp-aggregated) whenever a
// lane's scene changes: the lists are scene-major, so flushes are rare.
struct SceneSums {
    int scene = -1;
    unsigned a = 0, b = 0;
    __device__ __forceinline__ void add(int sc, unsigned da, unsigned db, unsigned long long *A, unsigned long long *B,
                                        unsigned long long *done_ns)
    {
        if (__any_sync(kFull, sc >= 0 && sc != scene)) flush(A, B, done_ns);
        if (sc >= 0) { scene = sc; a += da; b += db; }
    }
    __device__ __forceinline__ void flush(unsigned long long *A, unsigned long long *B, unsigned long long *done_ns)
    {
        scene_add(A, scene, a);
        if (B) scene_add(B, scene, b);
        scene_touch(done_ns, scene);
        a = b = 0;
    }
};

// ACCD over one stencil list of the wave, per-scene reductions.
template <int DIM, bool VF, bool CERT>
__global__ void __launch_bounds__(128, 4)
k_b_accd(BatchGroupDev g, const int4 *__restrict__ sten, const unsigned long long *n_ptr, unsigned long long cap,
         const int *__restrict__ vert_scene)
{
    unsigned long long n = *(volatile const unsigned long long *)n_ptr;
    if (n > cap) n = cap;
    const int lane = lane_id();
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    SceneSums sums;
    for (unsigned long long base = (unsigned long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < n;
         base += stride) {
        const unsigned long long i = base + lane;
        int s4[4] = {-1, -1, -1, -1};
        int sc = -1;
        bool hit = false;
        double toi = -1.0;
        if (i < n) {
            const int4 v = sten[i];
            s4[0] = v.x; s4[1] = v.y; s4[2] = v.z; s4[3] = v.w;
            sc = (v.x >= 0 && v.x < g.nv) ? vert_scene[v.x] : -1;
            if (sc < 0) atomicOr(g.err, kErrBadIndex);
            else hit = batch_accd<DIM, CERT>(s4, VF, g, g.eta[sc], toi) && toi >= 0.0;
        }
        sums.add(sc, sc >= 0 ? 1u : 0u, hit ? 1u : 0u, g.n_sten, g.n_hits, g.done_ns);
        scene_best<DIM>(g, hit ? sc : -1, toi, s4, VF);
    }
    sums.flush(g.n_sten, g.n_hits, g.done_ns);
}

// Discrete pairs of the wave -> per-scene counts.
__global__ void __launch_bounds__(256)
k_b_disc(BatchGroupDev g, const int2 *__restrict__ disc, const unsigned long long *n_ptr, unsigned long long cap)
{
    unsigned long long n = *(volatile const unsigned long long *)n_ptr;
    if (n > cap) n = cap;
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    SceneSums sums;
    for (unsigned long long base = (unsigned long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < n;
         base += stride) {
        const unsigned long long i = base + lane_id();
        const int sc = i < n ? g.prim_scene[disc[i].x] : -1;
        sums.add(sc, sc >= 0 ? 1u : 0u, 0u, g.n_disc, nullptr, g.done_ns);
    }
    sums.flush(g.n_disc, nullptr, g.done_ns);
}

// ---------------------------------------------------------------------------
// Persistent form: one kernel per group walks, expands and scores.  Warps
// take chunks of queries from a global work queue; each lane walks its
// query's scene tree one node (or scanned leaf) per step, found pairs go to a
// per-warp shared-memory buffer, and every 32 buffered pairs the warp runs
// the discrete tests, expands the stencils (VF first, then EE) and scores
// them 32 at a time.  Nothing but per-scene results leaves the chip.
// ---------------------------------------------------------------------------
constexpr int kPairBuf = 96;   // per warp: < 32 left over + up to 2 per lane per step

// Expands and evaluates the first m (<= 32) buffered pairs of this warp.
template <int DIM, bool CERT>
__device__ void batch_process(const BatchGroupDev &g, int m, const int2 *pairs, int (*face)[2 * DIM], int *scn_of,
                              unsigned short *codes)
{
    const int lane = lane_id();
    int fa[DIM], fb[DIM];
    unsigned bits = 0;
    int scene = -1;
    bool disc = false;
    if (lane < m) {
        const int2 pr = pairs[lane];
        scene = g.prim_scene[pr.x];
#pragma unroll
        for (int k = 0; k < DIM; ++k) { fa[k] = __ldg(g.P + (size_t)pr.x * DIM + k); fb[k] = __ldg(g.P + (size_t)pr.y * DIM + k); }
        bits = stencil_bits<DIM>(fa, fb, __ldg(g.flags + pr.x), __ldg(g.flags + pr.y));
        bool shared = false, inb = true;
#pragma unroll
        for (int i = 0; i < DIM; ++i) {
            inb = inb && fa[i] >= 0 && fa[i] < g.nv && fb[i] >= 0 && fb[i] < g.nv;
#pragma unroll
            for (int j = 0; j < DIM; ++j) shared |= fa[i] == fb[j];
        }
        if (!inb) atomicOr(g.err, kErrBadIndex);
        if (!shared && inb) {
            double A[DIM][DIM], B[DIM][DIM];
#pragma unroll
            for (int i = 0; i < DIM; ++i)
#pragma unroll
                for (int k = 0; k < DIM; ++k) {
                    A[i][k] = __ldg(g.V1 + (size_t)fa[i] * DIM + k);
                    B[i][k] = __ldg(g.V1 + (size_t)fb[i] * DIM + k);
                }
            if constexpr (DIM == 3) disc = tri_tri(A[0], A[1], A[2], B[0], B[1], B[2]);
            else disc = seg_seg(A[0], A[1], B[0], B[1]);
        }
        if (!inb) bits = 0;
#pragma unroll
        for (int k = 0; k < DIM; ++k) { face[lane][k] = fa[k]; face[lane][DIM + k] = fb[k]; }
        scn_of[lane] = scene;
    }
    scene_add(g.n_sten, scene, __popc(bits));
    scene_add(g.n_disc, scene, disc ? 1u : 0u);
    // stencil codes (source lane << 4 | bit), VF first then EE
    const unsigned nvf = __popc(bits & 0x3fu), nee = __popc(bits >> 6);
    unsigned ivf = nvf, iee = nee;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned a = __shfl_up_sync(kFull, ivf, o), b = __shfl_up_sync(kFull, iee, o);
        if (lane >= o) { ivf += a; iee += b; }
    }
    const unsigned tvf = __shfl_sync(kFull, ivf, 31), tee = __shfl_sync(kFull, iee, 31);
    unsigned pv = ivf - nvf, pe = tvf + iee - nee;
    for (unsigned mm = bits & 0x3fu; mm; mm &= mm - 1) codes[pv++] = (unsigned short)((lane << 4) | (__ffs(mm) - 1));
    for (unsigned mm = bits >> 6; mm; mm &= mm - 1) codes[pe++] = (unsigned short)((lane << 4) | (6 + __ffs(mm) - 1));
    __syncwarp();
    const unsigned total = tvf + tee;
    for (unsigned base = 0; base < total; base += 32) {
        const unsigned idx = base + lane;
        int sc = -1;
        bool hit = false;
        double toi = -1.0;
        int s4[4] = {-1, -1, -1, -1};
        bool vf = true;
        if (idx < total) {
            const unsigned code = codes[idx];
            const int pl = code >> 4, b = code & 15;
            const int *A = face[pl], *B = face[pl] + DIM;
            sc = scn_of[pl];
            if (b < 6) {
                const int *vs = b < 3 ? A : B, *fs = b < 3 ? B : A;
                s4[0] = vs[b % 3]; s4[1] = fs[0]; s4[2] = fs[1]; s4[3] = DIM == 3 ? fs[DIM - 1] : -1;
            } else {
                const int i = (b - 6) / 3, j = (b - 6) % 3;
                s4[0] = A[i]; s4[1] = A[(i + 1) % 3]; s4[2] = B[j]; s4[3] = B[(j + 1) % 3];
                vf = false;
            }
            hit = batch_accd<DIM, CERT>(s4, vf, g, g.eta[sc], toi) && toi >= 0.0;
        }
        const int hs = hit ? sc : -1;
        scene_add(g.n_hits, hs, hit ? 1u : 0u);
        scene_best<DIM>(g, hs, toi, s4, vf);
    }
    scene_touch(g.done_ns, scene);
    __syncwarp();
}

// Drops the first m = 32 (or all) entries of a warp's pair buffer of n < kPairBuf.
__device__ __forceinline__ void shift_pairs(int2 *buf, int m, int n)
{
    const int lane = lane_id(), rem = n - m;
    int2 a = make_int2(0, 0), b = make_int2(0, 0);
    if (lane < rem) a = buf[m + lane];
    if (lane + 32 < rem) b = buf[m + 32 + lane];
    __syncwarp();
    if (lane < rem) buf[lane] = a;
    if (lane + 32 < rem) buf[32 + lane] = b;
    __syncwarp();
}

// Dynamic shared memory of the persistent kernel: per-thread traversal
// stacks, then per warp the pair buffer, the faces and scenes of the pairs
// being expanded and their stencil codes.
template <int DIM, int BLOCK, int STACK>
struct FusedSmem {
    static constexpr int W = BLOCK / 32;
    static constexpr int kCodes = 32 * (DIM == 3 ? 15 : 6);
    int stack[STACK][BLOCK];
    int2 pairs[W][kPairBuf];
    int face[W][32][2 * DIM];
    int scene[W][32];
    unsigned short code[W][kCodes];
};

template <int DIM, bool CERT, int BLOCK, int STACK>
__global__ void __launch_bounds__(BLOCK, 512 / BLOCK)
k_batch_fused(BatchGroupDev g)
{
    constexpr int S = DIM == 3 ? 3 : 2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    auto &sm = *reinterpret_cast<FusedSmem<DIM, BLOCK, STACK> *>(smem_raw);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const LeafBox<DIM> *lbox = reinterpret_cast<const LeafBox<DIM> *>(g.leaf_box);
    const unsigned long long total = (unsigned long long)g.np;

    int npairs = 0;
    // query state of this lane
    int q = -1, sc = 0, lq = 0, lb = 0, nb = 0, ns = 0, qprim = 0, node = 0, sp = 0, scan_k = 1, scan_end = 0;
    bool have_node = false;
    long long steps = 0;
    Box2T<DIM> qbox;   // the query's FP32 boxes; its FP64 box is re-read on the rare undecided test
    unsigned long long next = 0, end = 0;
    bool drained = false;

    auto start_query = [&](int qi) {
        qprim = g.sorted[qi];
        sc = g.prim_scene[qprim];
        lb = g.leaf_off[sc];
        nb = g.node_off[sc];
        ns = g.scene_np[sc];
        lq = qi - lb;
        if (ns < 2 || lq >= ns - 1) return;   // nothing after it in its scene
        q = qi;
        const LeafBox<DIM> &qb = lbox[qi];
#pragma unroll
        for (int k = 0; k < DIM; ++k) {
            qbox.t0lo[k] = __double2float_rd(qb.lo0[k]); qbox.t0hi[k] = __double2float_ru(qb.hi0[k]);
            qbox.t1lo[k] = __double2float_rd(qb.lo1[k]); qbox.t1hi[k] = __double2float_ru(qb.hi1[k]);
        }
        node = 0; sp = 0; have_node = true; scan_k = 1; scan_end = 0; steps = 0;
    };

    for (;;) {
        // 1. idle lanes take the next queries of the warp's chunk
        bool need = q < 0;
        unsigned needm = __ballot_sync(kFull, need);
        while (needm && !drained) {
            if (next >= end) {
                unsigned long long b0 = 0;
                if (lane == 0) b0 = atomicAdd(g.queue, 32ull * (unsigned long long)g.chunk);
                b0 = __shfl_sync(kFull, b0, 0);
                if (b0 >= total) { drained = true; break; }
                next = b0;
                end = b0 + 32ull * (unsigned long long)g.chunk;
                if (end > total) end = total;
            }
            const unsigned rank = __popc(needm & lanemask_lt());
            const unsigned long long left = end - next, want = (unsigned long long)__popc(needm);
            const unsigned take = (unsigned)(left < want ? left : want);
            if (need && rank < take) { start_query((int)(next + rank)); need = false; }
            next += take;
            needm = __ballot_sync(kFull, need);
        }
        if (!__any_sync(kFull, q >= 0)) {
            if (drained) break;
            continue;   // every new query was trivial: take more
        }
        // 2. one unit of work per active lane: a scanned leaf or a node visit
        int2 f[2];
        int nf = 0;
        int finished = -1;   // scene of a query that ends in this step
        if (q >= 0) {
            auto found = [&](int k, int r) {   // local leaf k, three-valued test result r
                if (r == 2) r = leaf_boxes_intersect<DIM>(lbox[q], lbox[lb + k]) ? 1 : 0;
                if (r == 1) {
                    const int kprim = __ldg(g.sorted + lb + k);
                    f[nf++] = make_int2(min(qprim, kprim), max(qprim, kprim));
                }
            };
            if (++steps > 4ll * ns + 64) {
                atomicOr(g.err, kErrStack);
                q = -1;
            } else if (scan_k <= scan_end) {
                const int k = scan_k++;
                const LeafBox<DIM> &kb = lbox[lb + k];
                Box2T<DIM> kbox;
#pragma unroll
                for (int d = 0; d < DIM; ++d) {
                    kbox.t0lo[d] = __double2float_rd(kb.lo0[d]); kbox.t0hi[d] = __double2float_ru(kb.hi0[d]);
                    kbox.t1lo[d] = __double2float_rd(kb.lo1[d]); kbox.t1hi[d] = __double2float_ru(kb.hi1[d]);
                }
                found(k, leaf_test3<DIM>(qbox, inner<DIM>(qbox), kbox));
            } else if (!have_node) {
                if (sp == 0) {
                    q = -1;   // query done
                } else {
                    const int e = sm.stack[--sp][tid];
                    if (e & kScanFlag) {
                        const int c = e & ~kScanFlag;
                        scan_k = max(__ldg(&g.nodes[nb + c].pad.x), lq + 1);
                        scan_end = __ldg(&g.nodes[nb + c].d.z);
                    } else {
                        node = e;
                        have_node = true;
                    }
                }
            } else {
                const Node *nd = g.nodes + nb + node;
                float4 ls[S], rs[S];
#pragma unroll
                for (int i = 0; i < S; ++i) { ls[i] = __ldg(&nd->l[i]); rs[i] = __ldg(&nd->r[i]); }
                const int4 d = __ldg(&nd->d);
                const int first = __ldg(&nd->pad.x);
                const int split = d.x, meta = d.y, last = d.z;
                Box2T<DIM> lbx, rbx;
                unpack_child<DIM>(ls, lbx);
                unpack_child<DIM>(rs, rbx);
                bool lok = split > lq, rok = last > lq;   // every batch leaf is active
                if (lok && (meta & kMetaLeftLeaf)) { found(split, leaf_test3<DIM>(qbox, inner<DIM>(qbox), lbx)); lok = false; }
                if (rok && (meta & kMetaRightLeaf)) { found(split + 1, leaf_test3<DIM>(qbox, inner<DIM>(qbox), rbx)); rok = false; }
                lok = lok && boxes_may_intersect<DIM>(qbox, lbx);
                rok = rok && boxes_may_intersect<DIM>(qbox, rbx);
                // small subtrees are scanned leaf by leaf instead of descended
                const bool lscan = lok && split - first + 1 <= g.leaf_size;
                const bool rscan = rok && last - split <= g.leaf_size;
                have_node = false;
                if (lok && rok) {
                    if (sp < STACK) sm.stack[sp++][tid] = rscan ? ((split + 1) | kScanFlag) : split + 1;
                    else { atomicOr(g.err, kErrStack); q = -1; }
                }
                if (q >= 0) {
                    if (lok) {
                        if (lscan) { scan_k = max(first, lq + 1); scan_end = split; }
                        else { node = split; have_node = true; }
                    } else if (rok) {
                        if (rscan) { scan_k = max(split + 1, lq + 1); scan_end = last; }
                        else { node = split + 1; have_node = true; }
                    }
                }
            }
            if (q < 0) finished = sc;
        }
        scene_touch(g.done_ns, finished);
        // 3. buffer the found pairs: < 32 held before the step, <= 64 added
        unsigned incl = nf;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned v = __shfl_up_sync(kFull, incl, o);
            if (lane >= o) incl += v;
        }
        const int tot = (int)__shfl_sync(kFull, incl, 31);
        for (int j = 0; j < nf; ++j) sm.pairs[warp][npairs + (int)(incl - nf) + j] = f[j];
        npairs += tot;
        __syncwarp();
        while (npairs >= 32) {
            batch_process<DIM, CERT>(g, 32, sm.pairs[warp], sm.face[warp], sm.scene[warp], sm.code[warp]);
            shift_pairs(sm.pairs[warp], 32, npairs);
            npairs -= 32;
        }
    }
    while (npairs > 0) {
        const int m = npairs < 32 ? npairs : 32;
        batch_process<DIM, CERT>(g, m, sm.pairs[warp], sm.face[warp], sm.scene[warp], sm.code[warp]);
        shift_pairs(sm.pairs[warp], m, npairs);
        npairs -= m;
    }
}

// Per-scene results: counts 0, earliest-hit key (+inf, max).
__global__ void k_b_init_results(unsigned long long *res, BestKey *best, int n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 5 * n; i += gridDim.x * blockDim.x) {
        res[i] = 0ull;
        if (i < n) best[i] = BestKey{0x7ff0000000000000ull, ~0ull};
    }
}

// ---------------------------------------------------------------------------
// Host side.
// ---------------------------------------------------------------------------
namespace {

struct GroupHost {
    int dim = 0, n_scenes = 0, np = 0, nv = 0, n_int = 0;
    std::vector<int> scene_user;         // group scene -> caller's scene index
    std::vector<long long> v_dst_off;    // doubles, per group scene (+1 total)
    std::vector<long long> v_src_off;    // doubles, offset in the caller's V arrays
    std::vector<int> vbase;              // group vertex id of each scene's vertex 0
    double *V0 = nullptr, *V1 = nullptr, *eta = nullptr;
    int *P = nullptr, *prim_scene = nullptr, *leaf_off = nullptr, *node_off = nullptr, *scene_np = nullptr;
    int *node_scene = nullptr, *vals = nullptr, *vals_alt = nullptr, *leaf_parent = nullptr, *visits = nullptr;
    unsigned char *flags = nullptr, *leaf_active = nullptr;
    long long *dst_off = nullptr, *src_off = nullptr;
    float *cent = nullptr;
    unsigned *bounds = nullptr, *mort = nullptr, *keys = nullptr, *keys_alt = nullptr;
    void *sort_scratch = nullptr, *leaf_box = nullptr;
    Node *nodes = nullptr;
    unsigned long long *res = nullptr;   // [5][n_scenes]: hits, (unused), discrete, stencils, done ns
    BestKey *best = nullptr;             // per scene: earliest-hit key
    int *vert_scene = nullptr;           // group scene of each group vertex
    // wave buffers (sized by the wave-buffer tuning) and loop state
    unsigned long long cap_pairs = 0, cap_vf = 0, cap_ee = 0, cap_disc = 0;
    int2 *w_pairs = nullptr, *w_disc = nullptr;
    int4 *w_vf = nullptr, *w_ee = nullptr;
    Counters *w_cnt = nullptr;
    WaveState *ws = nullptr;
    unsigned long long *queue = nullptr;   // persistent form's work queue
    int fused_grid = 0;                    // persistent form's grid (resident blocks x SMs)
    cudaGraphConditionalHandle handle = 0;
};

int bits_for(int n)
{
    int b = 1;
    while ((1 << b) < n) ++b;
    return b;
}

} // namespace

} // namespace mclccd

using namespace mclccd;

struct mclccd_batch {
    int device = 0;
    int precision = MCLCCD_PREC_FP64;
    // block size, stack depth, queue chunk, leaf-scan size, form (0 waves,
    // 1 persistent), wave buffer (2^16 leaf pairs)
    int tune[MCLCCD_BATCH_TUNE_COUNT] = {128, 64, 4, 1, MCLCCD_BATCH_FORM_WAVES, 2048};
    int wave_chunk = 0;              // wave-buffer size the wave buffers were allocated for
    int n_scenes = 0;
    long long total_doubles = 0;
    std::vector<int> scene_dim;
    GroupHost grp[2];   // [0] 2D, [1] 3D (2D first: small scenes finish early)
    std::vector<void *> allocs;
    Counters *cnt = nullptr;
    BatchRecord *rec = nullptr;
    unsigned long long *n_rec = nullptr, *t_start = nullptr;
    unsigned long long rec_cap = 1ull << 22;
    double *stage0 = nullptr, *stage1 = nullptr;
    cudaStream_t stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool dirty = true, ran = false;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::string err;
};

namespace {

template <typename T>
cudaError_t balloc(mclccd_batch *b, T *&p, size_t count)
{
    void *q = nullptr;
    cudaError_t e = cudaMalloc(&q, std::max<size_t>(count * sizeof(T), 16));
    if (e != cudaSuccess) { cudaGetLastError(); return e; }
    b->allocs.push_back(q);
    p = static_cast<T *>(q);
    return cudaSuccess;
}

void free_all(mclccd_batch *b)
{
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    for (void *p : b->allocs) cudaFree(p);
    b->allocs.clear();
    for (auto &g : b->grp) g = GroupHost();
    b->cnt = nullptr;
    b->rec = nullptr;
    b->n_rec = b->t_start = nullptr;
    b->stage0 = b->stage1 = nullptr;
    b->n_scenes = 0;
    b->ran = false;
    b->wave_chunk = 0;
}

int bfail(mclccd_batch *b, int code, const std::string &msg)
{
    b->err = msg;
    return code;
}

#define MB_CUDA(b, x)                                                                              \
    do {                                                                                           \
        cudaError_t e_ = (x);                                                                      \
        if (e_ != cudaSuccess)                                                                     \
            return bfail(b, e_ == cudaErrorMemoryAllocation ? MCLCCD_ERR_NOMEM : MCLCCD_ERR_CUDA, \
                         std::string(#x) + ": " + cudaGetErrorString(e_));                        \
    } while (0)

int grid_of(long long n, int block, int cap)
{
    long long g = (n + block - 1) / block;
    return (int)std::max<long long>(1, std::min<long long>(g, cap));
}

template <int DIM, int STACK>
cudaError_t walk_attr(int block)
{
    return cudaFuncSetAttribute(k_b_walk<DIM, STACK>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                STACK * block * (int)sizeof(int));
}

cudaError_t prepare_walk(int dim, int block, int stack)
{
    if (dim == 3) return stack == 32 ? walk_attr<3, 32>(block) : walk_attr<3, 64>(block);
    return stack == 32 ? walk_attr<2, 32>(block) : walk_attr<2, 64>(block);
}

BatchGroupDev group_view(mclccd_batch *b, GroupHost &G)
{
    BatchGroupDev g{};
    g.np = G.np; g.nv = G.nv; g.n_scenes = G.n_scenes;
    g.V0 = G.V0; g.V1 = G.V1; g.P = G.P; g.flags = G.flags; g.prim_scene = G.prim_scene; g.sorted = G.vals;
    g.leaf_off = G.leaf_off; g.node_off = G.node_off; g.scene_np = G.scene_np; g.eta = G.eta;
    g.nodes = G.nodes; g.leaf_box = G.leaf_box; g.leaf_active = G.leaf_active;
    g.n_hits = G.res; g.n_disc = G.res + 2 * G.n_scenes;
    g.n_sten = G.res + 3 * G.n_scenes; g.done_ns = G.res + 4 * G.n_scenes; g.best = G.best;
    g.rec = b->rec; g.n_rec = b->n_rec; g.rec_cap = b->rec_cap; g.err = &b->cnt->err;
    g.queue = G.queue;
    g.chunk = b->tune[MCLCCD_BATCH_TUNE_CHUNK];
    g.leaf_size = b->tune[MCLCCD_BATCH_TUNE_LEAF];
    return g;
}

// Segmented LBVH build of group G (before its wave loop).
void enqueue_build(mclccd_batch *b, GroupHost &G, cudaStream_t st)
{
    const int dim = G.dim;
    unsigned *err = &b->cnt->err;
    const int gsz = grid_of(G.np, 256, 148 * 16);
    if (dim == 3) {
        k_b_init_bounds_dim<3><<<grid_of(G.n_scenes * 6, 256, 1024), 256, 0, st>>>(G.bounds, G.n_scenes);
        k_b_centroids<3><<<gsz, 256, 0, st>>>(G.V0, G.V1, G.P, G.np, G.nv, G.prim_scene, G.cent, G.bounds, err);
        k_b_morton<3><<<gsz, 256, 0, st>>>(G.cent, G.np, G.prim_scene, G.bounds, G.mort, G.keys, G.vals);
    } else {
        k_b_init_bounds_dim<2><<<grid_of(G.n_scenes * 4, 256, 1024), 256, 0, st>>>(G.bounds, G.n_scenes);
        k_b_centroids<2><<<gsz, 256, 0, st>>>(G.V0, G.V1, G.P, G.np, G.nv, G.prim_scene, G.cent, G.bounds, err);
        k_b_morton<2><<<gsz, 256, 0, st>>>(G.cent, G.np, G.prim_scene, G.bounds, G.mort, G.keys, G.vals);
    }
    // (scene, Morton) order: Morton passes, then a stable pass on the scene id
    launch_sort_pairs(G.keys, G.vals, G.keys_alt, G.vals_alt, G.np, 30, G.sort_scratch, b->cnt, st);
    k_b_gather_keys<<<gsz, 256, 0, st>>>(G.vals, reinterpret_cast<const unsigned *>(G.prim_scene), G.np, G.keys);
    launch_sort_pairs(G.keys, G.vals, G.keys_alt, G.vals_alt, G.np, (unsigned)bits_for(G.n_scenes), G.sort_scratch,
                      b->cnt, st);
    k_b_gather_keys<<<gsz, 256, 0, st>>>(G.vals, G.mort, G.np, G.keys);
    if (G.n_int > 0) {
        cudaMemsetAsync(G.visits, 0, sizeof(int) * (size_t)G.n_int, st);
        k_b_karras<<<grid_of(G.n_int, 256, 148 * 16), 256, 0, st>>>(G.keys, G.n_int, G.node_scene, G.leaf_off,
                                                                    G.node_off, G.scene_np, G.nodes, G.leaf_parent);
    }
    if (dim == 3)
        k_b_refit<3><<<(G.np + 255) / 256, 256, 0, st>>>(G.V0, G.V1, G.P, G.np, G.nv, G.prim_scene, G.vals, G.leaf_off,
                                                         G.node_off, G.scene_np, G.eta, G.leaf_parent, G.nodes,
                                                         G.visits, reinterpret_cast<LeafBox<3> *>(G.leaf_box),
                                                         G.leaf_active, err);
    else
        k_b_refit<2><<<(G.np + 255) / 256, 256, 0, st>>>(G.V0, G.V1, G.P, G.np, G.nv, G.prim_scene, G.vals, G.leaf_off,
                                                         G.node_off, G.scene_np, G.eta, G.leaf_parent, G.nodes,
                                                         G.visits, reinterpret_cast<LeafBox<2> *>(G.leaf_box),
                                                         G.leaf_active, err);
}

template <int DIM, bool CERT>
void enqueue_accd(const BatchGroupDev &g, GroupHost &G, cudaStream_t st)
{
    const int grid = 148 * 128;   // as the single-scene ACCD grid
    k_b_accd<DIM, true, CERT><<<grid, 128, 0, st>>>(g, G.w_vf, &G.w_cnt->n_vf, G.cap_vf, G.vert_scene);
    if constexpr (DIM == 3)
        k_b_accd<DIM, false, CERT><<<grid, 128, 0, st>>>(g, G.w_ee, &G.w_cnt->n_ee, G.cap_ee, G.vert_scene);
}

// One wave: walk, expansion, ACCD, discrete counts, loop control.
void enqueue_wave(mclccd_batch *b, GroupHost &G, cudaStream_t st)
{
    const BatchGroupDev g = group_view(b, G);
    const int block = b->tune[MCLCCD_BATCH_TUNE_BLOCK], stack = b->tune[MCLCCD_BATCH_TUNE_STACK];
    const unsigned long long nq = (unsigned long long)G.np;
    k_wave_begin<<<1, 1, 0, st>>>(G.ws, G.w_cnt, nq);
    const size_t smem = (size_t)stack * block * sizeof(int);
    const int wgrid = 148 * (2048 / block);
    if (G.dim == 3) {
        if (stack == 32) k_b_walk<3, 32><<<wgrid, block, smem, st>>>(g, G.ws, G.w_pairs, G.cap_pairs, G.w_cnt);
        else k_b_walk<3, 64><<<wgrid, block, smem, st>>>(g, G.ws, G.w_pairs, G.cap_pairs, G.w_cnt);
    } else {
        if (stack == 32) k_b_walk<2, 32><<<wgrid, block, smem, st>>>(g, G.ws, G.w_pairs, G.cap_pairs, G.w_cnt);
        else k_b_walk<2, 64><<<wgrid, block, smem, st>>>(g, G.ws, G.w_pairs, G.cap_pairs, G.w_cnt);
    }
    k_wave_check_pairs<<<1, 1, 0, st>>>(G.ws, G.w_cnt, G.cap_pairs);
    launch_expand_pairs(G.dim, G.w_pairs, G.cap_pairs, G.P, G.flags, G.V1, G.nv, G.w_vf, G.cap_vf, G.w_ee, G.cap_ee,
                        G.w_disc, G.cap_disc, 1, 1, G.w_cnt, 148 * 16, st);
    k_wave_check_sten<<<1, 1, 0, st>>>(G.ws, G.w_cnt, G.cap_vf, G.cap_ee, G.cap_disc);
    const bool cert = b->precision == MCLCCD_PREC_FP32_CERTIFIED;
    if (G.dim == 3) { if (cert) enqueue_accd<3, true>(g, G, st); else enqueue_accd<3, false>(g, G, st); }
    else { if (cert) enqueue_accd<2, true>(g, G, st); else enqueue_accd<2, false>(g, G, st); }
    k_b_disc<<<148 * 4, 256, 0, st>>>(g, G.w_disc, &G.w_cnt->n_discrete, G.cap_disc);
    k_wave_end<<<1, 1, 0, st>>>(G.ws, nq, G.cap_pairs, G.cap_vf, G.cap_ee, G.handle, &b->cnt->err);
}

// Persistent form.  prepare = true (outside capture): set the shared-memory
// limit and compute the grid (every block resident); false: launch it.
template <int DIM, bool CERT, int BLOCK, int STACK>
cudaError_t fused_t(const BatchGroupDev &g, cudaStream_t st, bool prepare, int &grid)
{
    const size_t bytes = sizeof(FusedSmem<DIM, BLOCK, STACK>);
    auto kern = k_batch_fused<DIM, CERT, BLOCK, STACK>;
    if (prepare) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        if (e != cudaSuccess) return e;
        int per_sm = 0, sms = 0, dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, BLOCK, bytes);
        if (e != cudaSuccess) return e;
        grid = std::max(1, per_sm) * std::max(1, sms);
        return cudaSuccess;
    }
    kern<<<grid, BLOCK, bytes, st>>>(g);
    return cudaGetLastError();
}

template <int DIM, bool CERT>
cudaError_t fused_d(const BatchGroupDev &g, int block, int stack, cudaStream_t st, bool prepare, int &grid)
{
    if (block == 256)
        return stack == 32 ? fused_t<DIM, CERT, 256, 32>(g, st, prepare, grid)
                           : fused_t<DIM, CERT, 256, 64>(g, st, prepare, grid);
    return stack == 32 ? fused_t<DIM, CERT, 128, 32>(g, st, prepare, grid)
                       : fused_t<DIM, CERT, 128, 64>(g, st, prepare, grid);
}

cudaError_t fused(mclccd_batch *b, GroupHost &G, cudaStream_t st, bool prepare)
{
    const bool cert = b->precision == MCLCCD_PREC_FP32_CERTIFIED;
    const int block = b->tune[MCLCCD_BATCH_TUNE_BLOCK], stack = b->tune[MCLCCD_BATCH_TUNE_STACK];
    const BatchGroupDev g = group_view(b, G);
    if (G.dim == 3)
        return cert ? fused_d<3, true>(g, block, stack, st, prepare, G.fused_grid)
                    : fused_d<3, false>(g, block, stack, st, prepare, G.fused_grid);
    return cert ? fused_d<2, true>(g, block, stack, st, prepare, G.fused_grid)
                : fused_d<2, false>(g, block, stack, st, prepare, G.fused_grid);
}

// Whole step as a graph: build of each group, then either its wave loop as
// a conditional WHILE node whose body is one wave, or the persistent kernel.
cudaError_t capture_step(mclccd_batch *b, cudaGraph_t *out)
{
    cudaStream_t st = nullptr, body_st = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&body_st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        k_b_stamp<<<1, 1, 0, st>>>(b->t_start);
        cudaMemsetAsync(b->cnt, 0, sizeof(Counters), st);
        cudaMemsetAsync(b->n_rec, 0, sizeof(unsigned long long), st);
        for (auto &G : b->grp) {
            if (G.n_scenes == 0) continue;
            k_b_init_results<<<grid_of(5ll * G.n_scenes, 256, 64), 256, 0, st>>>(G.res, G.best, G.n_scenes);
        }
        for (auto &G : b->grp) {
            if (G.np == 0 || e != cudaSuccess) continue;
            enqueue_build(b, G, st);
            if (b->tune[MCLCCD_BATCH_TUNE_FORM] == MCLCCD_BATCH_FORM_PERSISTENT) {
                cudaMemsetAsync(G.queue, 0, sizeof(unsigned long long), st);
                e = fused(b, G, st, false);
                continue;
            }
            k_wave_init<<<1, 1, 0, st>>>(G.ws, 1ull << 16);
            cudaStreamCaptureStatus cs;
            cudaGraph_t graph = nullptr;
            const cudaGraphNode_t *deps = nullptr;
            size_t ndeps = 0;
            e = cudaStreamGetCaptureInfo(st, &cs, nullptr, &graph, &deps, &ndeps);
            if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&G.handle, graph, 1, cudaGraphCondAssignDefault);
            cudaGraphNodeParams cp = {};
            cudaGraphNode_t node = nullptr;
            if (e == cudaSuccess) {
                cp.type = cudaGraphNodeTypeConditional;
                cp.conditional.handle = G.handle;
                cp.conditional.type = cudaGraphCondTypeWhile;
                cp.conditional.size = 1;
                e = cudaGraphAddNode(&node, graph, deps, ndeps, &cp);
            }
            if (e == cudaSuccess) e = cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies);
            if (e == cudaSuccess)
                e = cudaStreamBeginCaptureToGraph(body_st, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                                  cudaStreamCaptureModeThreadLocal);
            if (e == cudaSuccess) {
                enqueue_wave(b, G, body_st);
                cudaGraph_t body = nullptr;
                e = cudaStreamEndCapture(body_st, &body);
            }
        }
        if (e == cudaSuccess) e = cudaGetLastError();
        cudaGraph_t g = nullptr;
        const cudaError_t e2 = cudaStreamEndCapture(st, &g);
        if (e == cudaSuccess) e = e2;
        if (e == cudaSuccess) *out = g;
        else if (g) cudaGraphDestroy(g);
    }
    if (body_st) cudaStreamDestroy(body_st);
    if (st) cudaStreamDestroy(st);
    return e;
}

// Wave buffers for the current wave-buffer tuning.
cudaError_t ensure_wave_buffers(mclccd_batch *b)
{
    const int chunk = b->tune[MCLCCD_BATCH_TUNE_WAVE];
    if (b->wave_chunk == chunk) return cudaSuccess;
    for (auto &G : b->grp) {
        for (void *p : {(void *)G.w_pairs, (void *)G.w_disc, (void *)G.w_vf, (void *)G.w_ee}) {
            if (!p) continue;
            cudaFree(p);
            b->allocs.erase(std::remove(b->allocs.begin(), b->allocs.end(), p), b->allocs.end());
        }
        G.w_pairs = G.w_disc = nullptr;
        G.w_vf = G.w_ee = nullptr;
        if (G.np == 0) continue;
        G.cap_pairs = (unsigned long long)chunk << 16;
        G.cap_vf = 2 * G.cap_pairs;
        G.cap_ee = G.dim == 3 ? 4 * G.cap_pairs : 0;
        G.cap_disc = G.cap_pairs;
        cudaError_t e = balloc(b, G.w_pairs, G.cap_pairs);
        if (e == cudaSuccess) e = balloc(b, G.w_disc, G.cap_disc);
        if (e == cudaSuccess) e = balloc(b, G.w_vf, G.cap_vf);
        if (e == cudaSuccess && G.cap_ee) e = balloc(b, G.w_ee, G.cap_ee);
        if (e != cudaSuccess) return e;
    }
    b->wave_chunk = chunk;
    return cudaSuccess;
}

} // namespace

extern "C" {

int mclccd_batch_create(mclccd_batch **out)
{
    if (!out) return MCLCCD_ERR_INVALID;
    *out = nullptr;
    auto *b = new (std::nothrow) mclccd_batch();
    if (!b) return MCLCCD_ERR_NOMEM;
    cudaGetDevice(&b->device);
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&b->ev0) != cudaSuccess || cudaEventCreate(&b->ev1) != cudaSuccess) {
        cudaGetLastError();
        delete b;
        return MCLCCD_ERR_CUDA;
    }
    *out = b;
    return MCLCCD_OK;
}

int mclccd_batch_destroy(mclccd_batch *b)
{
    if (!b) return MCLCCD_OK;
    cudaSetDevice(b->device);
    cudaStreamSynchronize(b->stream);
    free_all(b);
    cudaEventDestroy(b->ev0);
    cudaEventDestroy(b->ev1);
    cudaStreamDestroy(b->stream);
    delete b;
    return MCLCCD_OK;
}

int mclccd_batch_set_scenes(mclccd_batch *b, int n_scenes, const int *scene_dim, const int *scene_nv,
                            const int *scene_np, const double *V0, const double *V1, const int *P, const double *eta,
                            int mem_kind)
{
    if (!b) return MCLCCD_ERR_INVALID;
    if (n_scenes <= 0 || !scene_dim || !scene_nv || !scene_np || !V0 || !V1 || !P || !eta)
        return bfail(b, MCLCCD_ERR_INVALID, "bad arguments");
    if (mem_kind != MCLCCD_MEM_HOST && mem_kind != MCLCCD_MEM_DEVICE) return bfail(b, MCLCCD_ERR_INVALID, "bad mem_kind");
    cudaSetDevice(b->device);
    cudaStreamSynchronize(b->stream);
    free_all(b);
    cudaStream_t st = b->stream;
    // scene table and the caller's offsets
    std::vector<long long> voff(n_scenes + 1, 0), poff(n_scenes + 1, 0);
    for (int s = 0; s < n_scenes; ++s) {
        if ((scene_dim[s] != 2 && scene_dim[s] != 3) || scene_nv[s] < 0 || scene_np[s] < 0 || !(eta[s] >= 0))
            return bfail(b, MCLCCD_ERR_INVALID, "bad scene " + std::to_string(s));
        voff[s + 1] = voff[s] + (long long)scene_nv[s] * scene_dim[s];
        poff[s + 1] = poff[s] + (long long)scene_np[s] * scene_dim[s];
    }
    std::vector<int> hP((size_t)poff[n_scenes]);
    if (mem_kind == MCLCCD_MEM_HOST) std::memcpy(hP.data(), P, sizeof(int) * hP.size());
    else MB_CUDA(b, cudaMemcpy(hP.data(), P, sizeof(int) * hP.size(), cudaMemcpyDeviceToHost));
    b->n_scenes = n_scenes;
    b->scene_dim.assign(scene_dim, scene_dim + n_scenes);
    b->total_doubles = voff[n_scenes];
    MB_CUDA(b, balloc(b, b->cnt, 1));
    MB_CUDA(b, balloc(b, b->rec, b->rec_cap));
    MB_CUDA(b, balloc(b, b->n_rec, 1));
    MB_CUDA(b, balloc(b, b->t_start, 1));
    for (int gi = 0; gi < 2; ++gi) {
        GroupHost &G = b->grp[gi];
        G.dim = gi == 0 ? 2 : 3;
        for (int s = 0; s < n_scenes; ++s)
            if (scene_dim[s] == G.dim) G.scene_user.push_back(s);
        // smaller scenes first: they finish early instead of waiting behind large ones
        std::stable_sort(G.scene_user.begin(), G.scene_user.end(),
                         [&](int a, int c) { return scene_np[a] < scene_np[c]; });
        G.n_scenes = (int)G.scene_user.size();
        if (G.n_scenes == 0) continue;
        const int dim = G.dim;
        std::vector<int> leaf_off(G.n_scenes + 1, 0), node_off(G.n_scenes + 1, 0), snp(G.n_scenes);
        std::vector<double> heta(G.n_scenes);
        G.v_dst_off.assign(G.n_scenes + 1, 0);
        G.v_src_off.assign(G.n_scenes, 0);
        G.vbase.assign(G.n_scenes, 0);
        long long np_tot = 0, nv_tot = 0, nint = 0;
        for (int k = 0; k < G.n_scenes; ++k) {
            const int s = G.scene_user[k];
            snp[k] = scene_np[s];
            heta[k] = eta[s];
            G.vbase[k] = (int)nv_tot;
            G.v_src_off[k] = voff[s];
            G.v_dst_off[k] = nv_tot * dim;
            leaf_off[k] = (int)np_tot;
            node_off[k] = (int)nint;
            np_tot += scene_np[s];
            nv_tot += scene_nv[s];
            nint += scene_np[s] > 1 ? scene_np[s] - 1 : 0;
        }
        G.v_dst_off[G.n_scenes] = nv_tot * dim;
        leaf_off[G.n_scenes] = (int)np_tot;
        node_off[G.n_scenes] = (int)nint;
        if (np_tot >= (1ll << 30) || nv_tot >= (1ll << 31) / 3)
            return bfail(b, MCLCCD_ERR_INVALID, "batch group too large");
        G.np = (int)np_tot;
        G.nv = (int)nv_tot;
        G.n_int = (int)nint;
        std::vector<int> gP((size_t)np_tot * dim), pscene((size_t)np_tot), nscene((size_t)std::max<long long>(nint, 1));
        for (int k = 0; k < G.n_scenes; ++k) {
            const int s = G.scene_user[k];
            const int *src = hP.data() + poff[s];
            for (long long i = 0; i < (long long)scene_np[s] * dim; ++i) {
                const int v = src[i];
                if (v < 0 || v >= scene_nv[s]) return bfail(b, MCLCCD_ERR_INVALID, "P index out of range in scene " + std::to_string(s));
                gP[(size_t)leaf_off[k] * dim + i] = v + G.vbase[k];
            }
            for (int i = 0; i < scene_np[s]; ++i) pscene[(size_t)leaf_off[k] + i] = k;
            for (int i = node_off[k]; i < node_off[k + 1]; ++i) nscene[(size_t)i] = k;
        }
        const size_t np = (size_t)np_tot, nv = (size_t)nv_tot, ni = (size_t)std::max<long long>(nint, 1);
        std::vector<int> vscene(std::max<size_t>(nv, 1), 0);
        for (int k = 0; k < G.n_scenes; ++k)
            for (int i = 0; i < scene_nv[G.scene_user[k]]; ++i) vscene[(size_t)G.vbase[k] + i] = k;
        MB_CUDA(b, balloc(b, G.V0, nv * dim));
        MB_CUDA(b, balloc(b, G.V1, nv * dim));
        MB_CUDA(b, balloc(b, G.eta, G.n_scenes));
        MB_CUDA(b, balloc(b, G.P, np * dim));
        MB_CUDA(b, balloc(b, G.prim_scene, np));
        MB_CUDA(b, balloc(b, G.leaf_off, G.n_scenes + 1));
        MB_CUDA(b, balloc(b, G.node_off, G.n_scenes + 1));
        MB_CUDA(b, balloc(b, G.scene_np, G.n_scenes));
        MB_CUDA(b, balloc(b, G.node_scene, ni));
        MB_CUDA(b, balloc(b, G.vals, np));
        MB_CUDA(b, balloc(b, G.vals_alt, np));
        MB_CUDA(b, balloc(b, G.keys, np));
        MB_CUDA(b, balloc(b, G.keys_alt, np));
        MB_CUDA(b, balloc(b, G.mort, np));
        MB_CUDA(b, balloc(b, G.cent, np * dim));
        MB_CUDA(b, balloc(b, G.bounds, (size_t)G.n_scenes * 2 * dim));
        MB_CUDA(b, balloc(b, G.leaf_parent, np));
        MB_CUDA(b, balloc(b, G.visits, ni));
        MB_CUDA(b, balloc(b, G.nodes, ni));
        MB_CUDA(b, balloc(b, G.leaf_active, np));
        MB_CUDA(b, balloc(b, G.flags, np));
        MB_CUDA(b, balloc(b, G.res, (size_t)G.n_scenes * 5));
        MB_CUDA(b, balloc(b, G.best, (size_t)G.n_scenes));
        MB_CUDA(b, balloc(b, G.vert_scene, std::max<size_t>(nv, 1)));
        MB_CUDA(b, balloc(b, G.w_cnt, 1));
        MB_CUDA(b, balloc(b, G.ws, 1));
        MB_CUDA(b, balloc(b, G.queue, 1));
        MB_CUDA(b, cudaMemsetAsync(G.ws, 0, sizeof(WaveState), st));
        MB_CUDA(b, balloc(b, G.dst_off, G.n_scenes + 1));
        MB_CUDA(b, balloc(b, G.src_off, G.n_scenes));
        unsigned char *lb = nullptr;
        MB_CUDA(b, balloc(b, lb, np * (dim == 3 ? sizeof(LeafBox<3>) : sizeof(LeafBox<2>))));
        G.leaf_box = lb;
        unsigned char *ss = nullptr;
        const int passes = std::max(sort_num_passes(30), sort_num_passes((unsigned)bits_for(G.n_scenes)));
        MB_CUDA(b, balloc(b, ss, sort_scratch_bytes(G.np, passes)));
        G.sort_scratch = ss;
        MB_CUDA(b, cudaMemcpyAsync(G.eta, heta.data(), sizeof(double) * G.n_scenes, cudaMemcpyHostToDevice, st));
        MB_CUDA(b, cudaMemcpyAsync(G.P, gP.data(), sizeof(int) * gP.size(), cudaMemcpyHostToDevice, st));
        MB_CUDA(b, cudaMemcpyAsync(G.prim_scene, pscene.data(), sizeof(int) * np, cudaMemcpyHostToDevice, st));
        MB_CUDA(b, cudaMemcpyAsync(G.vert_scene, vscene.data(), sizeof(int) * vscene.size(), cudaMemcpyHostToDevice, st));
        MB_CUDA(b, cudaMemcpyAsync(G.leaf_off, leaf_off.data(), sizeof(int) * leaf_off.size(), cudaMemcpyHostToDevice, st));
        MB_CUDA(b, cudaMemcpyAsync(G.node_off, node_off.data(), sizeof(int) * node_off.size(), cudaMemcpyHostToDevice, st));
        MB_CUDA(b, cudaMemcpyAsync(G.scene_np, snp.data(), sizeof(int) * snp.size(), cudaMemcpyHostToDevice, st));
        MB_CUDA(b, cudaMemcpyAsync(G.node_scene, nscene.data(), sizeof(int) * nscene.size(), cudaMemcpyHostToDevice, st));
        MB_CUDA(b, cudaMemcpyAsync(G.dst_off, G.v_dst_off.data(), sizeof(long long) * G.v_dst_off.size(),
                                   cudaMemcpyHostToDevice, st));
        MB_CUDA(b, cudaMemcpyAsync(G.src_off, G.v_src_off.data(), sizeof(long long) * G.v_src_off.size(),
                                   cudaMemcpyHostToDevice, st));
        // representative flags (topology only), as the single-scene update computes them
        unsigned long long ecap = 1024;
        while (ecap < np * 6) ecap <<= 1;
        int *vowner = nullptr, *eowner = nullptr;
        unsigned long long *ekeys = nullptr;
        MB_CUDA(b, cudaMalloc(&vowner, sizeof(int) * std::max<size_t>(nv, 1)));
        MB_CUDA(b, cudaMalloc(&eowner, sizeof(int) * ecap));
        MB_CUDA(b, cudaMalloc(&ekeys, sizeof(unsigned long long) * ecap));
        MB_CUDA(b, cudaMemsetAsync(b->cnt, 0, sizeof(Counters), st));
        launch_owner_flags(G.P, G.np, dim, G.nv, vowner, ekeys, eowner, ecap, G.flags, b->cnt, st);
        MB_CUDA(b, cudaStreamSynchronize(st));
        cudaFree(vowner);
        cudaFree(eowner);
        cudaFree(ekeys);
        Counters hc{};
        MB_CUDA(b, cudaMemcpy(&hc, b->cnt, sizeof(Counters), cudaMemcpyDeviceToHost));
        if (hc.err) return bfail(b, MCLCCD_ERR_DEVICE, "representative flags failed");
    }
    b->dirty = true;
    return mclccd_batch_set_positions(b, V0, V1, mem_kind);
}

int mclccd_batch_set_positions(mclccd_batch *b, const double *V0, const double *V1, int mem_kind)
{
    if (!b || !V0 || !V1) return MCLCCD_ERR_INVALID;
    if (b->n_scenes == 0) return bfail(b, MCLCCD_ERR_STATE, "no scenes");
    if (mem_kind != MCLCCD_MEM_HOST && mem_kind != MCLCCD_MEM_DEVICE) return MCLCCD_ERR_INVALID;
    cudaSetDevice(b->device);
    cudaStream_t st = b->stream;
    const double *s0 = V0, *s1 = V1;
    if (mem_kind == MCLCCD_MEM_HOST) {
        if (!b->stage0) {
            MB_CUDA(b, balloc(b, b->stage0, (size_t)b->total_doubles));
            MB_CUDA(b, balloc(b, b->stage1, (size_t)b->total_doubles));
        }
        MB_CUDA(b, cudaMemcpyAsync(b->stage0, V0, sizeof(double) * b->total_doubles, cudaMemcpyHostToDevice, st));
        MB_CUDA(b, cudaMemcpyAsync(b->stage1, V1, sizeof(double) * b->total_doubles, cudaMemcpyHostToDevice, st));
        s0 = b->stage0;
        s1 = b->stage1;
    }
    for (auto &G : b->grp) {
        const long long n = G.n_scenes ? G.v_dst_off[G.n_scenes] : 0;
        if (n == 0) continue;
        k_b_scatter<<<grid_of(n, 256, 148 * 16), 256, 0, st>>>(s0, G.V0, n, G.dst_off, G.src_off, G.n_scenes);
        k_b_scatter<<<grid_of(n, 256, 148 * 16), 256, 0, st>>>(s1, G.V1, n, G.dst_off, G.src_off, G.n_scenes);
    }
    MB_CUDA(b, cudaGetLastError());
    if (mem_kind == MCLCCD_MEM_HOST) MB_CUDA(b, cudaStreamSynchronize(st));   // host buffers may be reused
    return MCLCCD_OK;
}

int mclccd_batch_set_precision(mclccd_batch *b, int precision)
{
    if (!b || (precision != MCLCCD_PREC_FP64 && precision != MCLCCD_PREC_FP32_CERTIFIED)) return MCLCCD_ERR_INVALID;
    if (b->precision != precision) b->dirty = true;
    b->precision = precision;
    return MCLCCD_OK;
}

int mclccd_batch_set_tuning(mclccd_batch *b, int key, int value)
{
    if (!b || key < 0 || key >= MCLCCD_BATCH_TUNE_COUNT) return MCLCCD_ERR_INVALID;
    const bool ok = (key == MCLCCD_BATCH_TUNE_BLOCK && (value == 128 || value == 256)) ||
                    (key == MCLCCD_BATCH_TUNE_STACK && (value == 32 || value == 64)) ||
                    (key == MCLCCD_BATCH_TUNE_CHUNK && value >= 1 && value <= 64) ||
                    (key == MCLCCD_BATCH_TUNE_LEAF && value >= 1 && value <= 16) ||
                    (key == MCLCCD_BATCH_TUNE_FORM &&
                     (value == MCLCCD_BATCH_FORM_WAVES || value == MCLCCD_BATCH_FORM_PERSISTENT)) ||
                    (key == MCLCCD_BATCH_TUNE_WAVE && value >= 1 && value <= 4096);
    if (!ok) return MCLCCD_ERR_INVALID;
    if (b->tune[key] != value) b->dirty = true;
    b->tune[key] = value;
    return MCLCCD_OK;
}

int mclccd_batch_get_tuning(const mclccd_batch *b, int key, int *value)
{
    if (!b || !value || key < 0 || key >= MCLCCD_BATCH_TUNE_COUNT) return MCLCCD_ERR_INVALID;
    *value = b->tune[key];
    return MCLCCD_OK;
}

int mclccd_batch_wave_stats(mclccd_batch *b, long long *waves, long long *redos)
{
    if (!b || !waves || !redos) return MCLCCD_ERR_INVALID;
    *waves = *redos = 0;
    if (!b->ran || b->tune[MCLCCD_BATCH_TUNE_FORM] != MCLCCD_BATCH_FORM_WAVES) return MCLCCD_OK;
    cudaSetDevice(b->device);
    for (auto &G : b->grp) {
        if (G.np == 0 || !G.ws) continue;
        WaveState h{};
        MB_CUDA(b, cudaMemcpyAsync(&h, G.ws, sizeof(h), cudaMemcpyDeviceToHost, b->stream));
        MB_CUDA(b, cudaStreamSynchronize(b->stream));
        *waves += (long long)h.waves;
        *redos += (long long)h.redos;
    }
    return MCLCCD_OK;
}

int mclccd_batch_run(mclccd_batch *b, void *stream)
{
    if (!b) return MCLCCD_ERR_INVALID;
    if (b->n_scenes == 0) return bfail(b, MCLCCD_ERR_STATE, "no scenes");
    cudaSetDevice(b->device);
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : b->stream;
    if (st != b->stream) {   // order after pending position updates on the batch's own stream
        cudaEvent_t e;
        MB_CUDA(b, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        cudaEventRecord(e, b->stream);
        cudaStreamWaitEvent(st, e, 0);
        cudaEventDestroy(e);
    }
    if (b->dirty) {
        MB_CUDA(b, cudaStreamSynchronize(st));
        const bool persistent = b->tune[MCLCCD_BATCH_TUNE_FORM] == MCLCCD_BATCH_FORM_PERSISTENT;
        if (!persistent) MB_CUDA(b, ensure_wave_buffers(b));
        for (auto &G : b->grp) {
            if (G.np == 0) continue;
            if (persistent) MB_CUDA(b, fused(b, G, st, true));
            else MB_CUDA(b, prepare_walk(G.dim, b->tune[MCLCCD_BATCH_TUNE_BLOCK], b->tune[MCLCCD_BATCH_TUNE_STACK]));
        }
        if (b->exec) cudaGraphExecDestroy(b->exec);
        if (b->graph) cudaGraphDestroy(b->graph);
        b->exec = nullptr;
        b->graph = nullptr;
        cudaError_t e = capture_step(b, &b->graph);
        if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, b->graph, 0);
        if (e != cudaSuccess) { cudaGetLastError(); return bfail(b, MCLCCD_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e)); }
        b->dirty = false;
    }
    MB_CUDA(b, cudaEventRecord(b->ev0, st));
    MB_CUDA(b, cudaGraphLaunch(b->exec, st));
    MB_CUDA(b, cudaEventRecord(b->ev1, st));
    if (st != b->stream) {
        cudaEvent_t e;
        MB_CUDA(b, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        cudaEventRecord(e, st);
        cudaStreamWaitEvent(b->stream, e, 0);
        cudaEventDestroy(e);
    }
    b->ran = true;
    return MCLCCD_OK;
}

int mclccd_batch_results(mclccd_batch *b, long long *n_hits, double *min_toi, int *min_sten,
                         unsigned char *min_is_vf, long long *n_discrete, long long *n_stencils, double *done_ms,
                         double *batch_ms)
{
    if (!b) return MCLCCD_ERR_INVALID;
    if (!b->ran) return bfail(b, MCLCCD_ERR_STATE, "no batch run");
    cudaSetDevice(b->device);
    MB_CUDA(b, cudaStreamSynchronize(b->stream));
    MB_CUDA(b, cudaEventSynchronize(b->ev1));
    Counters hc{};
    unsigned long long nrec = 0, t0 = 0;
    MB_CUDA(b, cudaMemcpy(&hc, b->cnt, sizeof(Counters), cudaMemcpyDeviceToHost));
    MB_CUDA(b, cudaMemcpy(&nrec, b->n_rec, sizeof(nrec), cudaMemcpyDeviceToHost));
    MB_CUDA(b, cudaMemcpy(&t0, b->t_start, sizeof(t0), cudaMemcpyDeviceToHost));
    std::vector<BatchRecord> rec((size_t)std::min(nrec, b->rec_cap));
    if (!rec.empty()) MB_CUDA(b, cudaMemcpy(rec.data(), b->rec, sizeof(BatchRecord) * rec.size(), cudaMemcpyDeviceToHost));
    if (batch_ms) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, b->ev0, b->ev1);
        *batch_ms = ms;
    }
    for (int gi = 0; gi < 2; ++gi) {
        GroupHost &G = b->grp[gi];
        if (G.n_scenes == 0) continue;
        std::vector<unsigned long long> res((size_t)G.n_scenes * 5);
        std::vector<BestKey> bk((size_t)G.n_scenes);
        MB_CUDA(b, cudaMemcpy(res.data(), G.res, sizeof(unsigned long long) * res.size(), cudaMemcpyDeviceToHost));
        MB_CUDA(b, cudaMemcpy(bk.data(), G.best, sizeof(BestKey) * bk.size(), cudaMemcpyDeviceToHost));
        // argmin: the logged hit with the scene's final (toi, k1) and the
        // smallest (v2, v3)
        std::vector<long long> best((size_t)G.n_scenes, -1);
        auto k1_of = [](const BatchRecord &r) {
            return ((unsigned long long)(r.is_vf ? 0 : 1) << 63) | ((unsigned long long)(unsigned)r.sten.x << 32) |
                   (unsigned)r.sten.y;
        };
        auto k2_of = [](const BatchRecord &r) {
            return ((unsigned long long)(unsigned)r.sten.z << 32) | (unsigned)r.sten.w;
        };
        for (size_t i = 0; i < rec.size(); ++i) {
            const BatchRecord &r = rec[i];
            if (((r.scene & kRecGroup3) != 0) != (gi == 1)) continue;
            const int rs = r.scene & (kRecGroup3 - 1);
            if (rs >= G.n_scenes) continue;
            unsigned long long bits;
            std::memcpy(&bits, &r.toi, 8);
            if (bits != bk[(size_t)rs].toi || k1_of(r) != bk[(size_t)rs].k1) continue;
            long long &cur = best[(size_t)rs];
            if (cur < 0 || k2_of(r) < k2_of(rec[(size_t)cur])) cur = (long long)i;
        }
        for (int k = 0; k < G.n_scenes; ++k) {
            const int s = G.scene_user[k];
            const unsigned long long mb = bk[(size_t)k].toi;
            double mt;
            std::memcpy(&mt, &mb, 8);
            if (n_hits) n_hits[s] = (long long)res[k];
            if (min_toi) min_toi[s] = res[k] ? mt : -1.0;
            if (n_discrete) n_discrete[s] = (long long)res[2 * (size_t)G.n_scenes + k];
            if (n_stencils) n_stencils[s] = (long long)res[3 * (size_t)G.n_scenes + k];
            if (done_ms) {
                const unsigned long long dn = res[4 * (size_t)G.n_scenes + k];
                done_ms[s] = dn > t0 ? (double)(dn - t0) * 1e-6 : 0.0;
            }
            const long long r = best[(size_t)k];
            if (min_sten) {
                int4 v = r >= 0 ? rec[(size_t)r].sten : make_int4(-1, -1, -1, -1);
                const int base = G.vbase[k];
                int *o = min_sten + 4 * (size_t)s;
                o[0] = v.x >= 0 ? v.x - base : -1;
                o[1] = v.y >= 0 ? v.y - base : -1;
                o[2] = v.z >= 0 ? v.z - base : -1;
                o[3] = v.w >= 0 ? v.w - base : -1;
            }
            if (min_is_vf) min_is_vf[s] = r >= 0 ? (unsigned char)rec[(size_t)r].is_vf : 0;
        }
    }
    const unsigned fatal = hc.err & ~kErrAccdIters;
    if (fatal & kErrBadIndex) return bfail(b, MCLCCD_ERR_INVALID, "primitive index out of range");
    if (fatal) return bfail(b, MCLCCD_ERR_DEVICE, "device error flags " + std::to_string(fatal));
    if (nrec > b->rec_cap) return bfail(b, MCLCCD_ERR_OVERFLOW, "earliest-hit log overflowed");
    return MCLCCD_OK;
}

const char *mclccd_batch_last_error(const mclccd_batch *b) { return b ? b->err.c_str() : ""; }

} // extern "C"
