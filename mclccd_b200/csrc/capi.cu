// C ABI of the B200 CCD path: handle state, device buffers and the
// update / traverse orchestration (see include/mclccd_b200.h).
#include "../../include/mclccd_b200.h"
#include "kernels.cuh"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

using namespace mclccd;

namespace {

struct DevBuf {
    void *p = nullptr;
    size_t cap = 0;
};

// Grid sizes (blocks) of the grid-stride expansion and ACCD kernels, from a
// sweep on the 2.1M-triangle step: ACCD 148 x {8, 16, 32, 64, 128, 256,
// 1024} -> 4.69, 4.59, 4.46, 4.35, 4.31, 4.32, 4.81 ms; expansion 148 x {4, 8,
// 16, 32} -> 2.43, 1.87, 1.81, 1.81 ms.
constexpr int kExpandGrid = 148 * 16;
constexpr int kAccdGrid = 148 * 128;
// The fused pairs -> ACCD kernel is grid-stride over warp batches: one wave
// of resident blocks (6 per SM).
constexpr int kFusedGrid = 148 * 6;
// the tree-quality sum runs after every full build and every 4th refit
constexpr int kQualityEvery = 4;
// The discrete test is grid-stride over the leaf pairs (128-thread blocks).
#ifndef MCLCCD_DISCRETE_GRID
#define MCLCCD_DISCRETE_GRID (148 * 128)
#endif
constexpr int kDiscreteGrid = MCLCCD_DISCRETE_GRID;
constexpr int kMaxAttempts = 6;

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev)
    {
        if (cudaGetDevice(&prev) == cudaSuccess && prev != dev) cudaSetDevice(dev);
        else prev = -1;
    }
    ~DeviceGuard() { if (prev >= 0) cudaSetDevice(prev); }
};

} // namespace

struct mclccd_tree {
    int dim = 3;
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    double box_eta = 1e-6, vf_eta = 1e-6, ee_eta = 1e-6;
    unsigned flags = MCLCCD_OPT_DEFAULT;
    int precision = MCLCCD_PREC_FP64;
    std::string err;

    bool built = false, traversed = false;
    int np = 0, pdim = 0, nv = 0, flags_np = 0;
    const double *upd_V0 = nullptr, *upd_V1 = nullptr;
    const double *tr_V0 = nullptr, *tr_V1 = nullptr;   // device V0/V1 of the last traverse
    int tr_nv = 0;
    long long launches = 0;
    float stage[7] = {0, 0, 0, 0, 0, 0, 0};
    unsigned long long n_pairs = 0, n_vf = 0, n_ee = 0, n_hits = 0, n_disc = 0, n_fp64 = 0, n_bound_toi = 0;
    unsigned long long cap_pairs = 0, cap_vf = 0, cap_ee = 0, cap_hits = 0, cap_disc = 0;

    DevBuf V0d, V1d, Pd, Pstage, actd, pflags, pflags_tmp, vowner, ekeys, eowner;
    DevBuf cent, bounds, keys, vals, keys_alt, vals_alt, sort_scratch;
    DevBuf nodes, leaf_parent, visits, leaf_box, leaf_active;
    DevBuf pairs, vf, ee, hit_sten, hit_toi, hit_isvf, disc, counters, diff, fp64_queue;
    DevBuf in_V, in_P, in_act, in_tmp;   // input conversion staging (mclccd_update_ex / mclccd_traverse_ex)
    DevBuf cand_cnt;                     // counters of the on-request candidate expansion
    DevBuf walk_cursor;                  // query cursor of the refill walk
    DevBuf quality;                      // summed box areas of the internal nodes and of the leaves
    double *h_quality = nullptr;         // pinned copy of the two sums
    double q_build = 0.0;                // tree quality (internal / leaf box areas) after the last build
    bool force_rebuild = false;          // the refit-only tree degraded: rebuild at the next update
    long long n_builds = 0, n_quality_rebuilds = 0, refits_since_check = 0;
    DevBuf tq_idx, tq_state, tq_count;   // continuing-stencil queue of the split ACCD form
    std::vector<DevBuf *> all()
    {
        return {&V0d, &V1d, &Pd, &Pstage, &actd, &pflags, &pflags_tmp, &vowner, &ekeys, &eowner, &cent, &bounds,
                &keys, &vals, &keys_alt, &vals_alt, &sort_scratch, &nodes, &leaf_parent, &visits, &leaf_box,
                &leaf_active, &pairs, &vf, &ee, &hit_sten, &hit_toi, &hit_isvf, &disc, &counters, &diff,
                &fp64_queue, &in_V, &in_P, &in_act, &in_tmp, &cand_cnt, &walk_cursor, &tq_idx, &tq_state, &tq_count, &quality};
    }
    Counters *h_cnt = nullptr;   // pinned mirror of the device counters
    int *h_diff = nullptr;
    cudaEvent_t ev[8] = {};
    // overlapped traverse (MCLCCD_TUNE_OVERLAP): walk and narrow-phase streams,
    // fork / chunk / join events, per-chunk list boundaries
    cudaStream_t s_walk = nullptr, s_narrow = nullptr;
    cudaEvent_t ov_ev[4] = {};
    DevBuf ovl;
    // streamed results (mclccd_traverse_out): copy stream, per-chunk events
    // and pinned hit-count snapshots
    cudaStream_t s_copy = nullptr;
    cudaEvent_t out_ev[16] = {};
    unsigned long long *h_snap = nullptr;
    unsigned long long out_done = 0;   // hits already copied out by the streamed path
    int tune[MCLCCD_TUNE_COUNT] = {kExpandGrid, kAccdGrid, 0, 0, 16, 0, 0, kFusedGrid, 0, 1, 150, 2};
    // The fused narrow phase counts the candidate lists without writing them;
    // mclccd_get_candidates rebuilds them from the leaf pairs and the P of the
    // last traverse.
    bool cand_lazy = false, cand_ready = false;
    const int *tr_P = nullptr;
};

namespace {

int fail(mclccd_tree *t, int code, const std::string &msg)
{
    if (t) t->err = msg;
    return code;
}

int cuda_fail(mclccd_tree *t, cudaError_t e, const char *what)
{
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    return fail(t, e == cudaErrorMemoryAllocation ? MCLCCD_ERR_NOMEM : MCLCCD_ERR_CUDA, m);
}

#define MC_CUDA(t, x)                                        \
    do {                                                     \
        cudaError_t e_ = (x);                                \
        if (e_ != cudaSuccess) return cuda_fail(t, e_, #x); \
    } while (0)

// Grow-only device buffer (contents are not preserved).
cudaError_t ensure(DevBuf &b, size_t bytes)
{
    if (bytes == 0) bytes = 16;
    if (bytes <= b.cap) return cudaSuccess;
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.cap = 0;
    size_t want = bytes + bytes / 8;
    cudaError_t e = cudaMalloc(&b.p, want);
    if (e != cudaSuccess) { cudaGetLastError(); return e; }
    b.cap = want;
    return cudaSuccess;
}

template <typename T> T *as(DevBuf &b) { return reinterpret_cast<T *>(b.p); }


int check_launch(mclccd_tree *t, const char *what)
{
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(t, e, what);
    return MCLCCD_OK;
}

int device_errors(mclccd_tree *t, unsigned err)
{
    if (err & kErrBadIndex) return fail(t, MCLCCD_ERR_INVALID, "a primitive or stencil references a vertex outside [0, nv)");
    if (err & kErrHashFull) return fail(t, MCLCCD_ERR_DEVICE, "edge table probe limit reached");
    if (err & kErrSortWait) return fail(t, MCLCCD_ERR_DEVICE, "radix sort look-back wait gave up");
    if (err & kErrStack) return fail(t, MCLCCD_ERR_DEVICE, "traversal stack overflow");
    return MCLCCD_OK;
}

} // namespace

// The tree walk over queries [qb, qe) (qe < 0: all): the refill form when
// tuned in (and not the packet walk), else launch_traverse's forms.
static int launch_walk(mclccd_tree *t, int dim, int packet, int np, Counters *cnt, cudaStream_t st, int qb = 0,
                       int qe = -1)
{
    if (!packet && t->tune[MCLCCD_TUNE_WALK_REFILL]) {
        MC_CUDA(t, ensure(t->walk_cursor, sizeof(unsigned)));
        launch_traverse_refill(dim, t->tune[MCLCCD_TUNE_WALK_WINDOW] ? t->tune[MCLCCD_TUNE_WALK_WINDOW] : 16,
                               as<Node>(t->nodes), t->leaf_box.p, as<unsigned char>(t->leaf_active), as<int>(t->vals),
                               np, as<int2>(t->pairs), t->cap_pairs, cnt, as<unsigned>(t->walk_cursor), st, qb, qe);
        return MCLCCD_OK;
    }
    const int win = t->tune[MCLCCD_TUNE_WALK_WINDOW];
    if (!packet && t->tune[MCLCCD_TUNE_WALK_BUFFER] && (win == 8 || win == 16 || win == 32)) {
        launch_traverse_buffered(dim, t->tune[MCLCCD_TUNE_WALK_WINDOW], t->tune[MCLCCD_TUNE_WALK_BUFFER] >= 2 ? 64 : 32,
                                 as<Node>(t->nodes), t->leaf_box.p,
                                 as<unsigned char>(t->leaf_active), as<int>(t->vals), np, as<int2>(t->pairs),
                                 t->cap_pairs, cnt, st, qb, qe);
        return MCLCCD_OK;
    }
    launch_traverse(dim, packet, t->tune[MCLCCD_TUNE_WALK_WINDOW], as<Node>(t->nodes), t->leaf_box.p,
                    as<unsigned char>(t->leaf_active), as<int>(t->vals), np, as<int2>(t->pairs), t->cap_pairs, cnt, st,
                    qb, qe);
    return MCLCCD_OK;
}

// Leaf pairs [*lo, *hi) -> stencil lists and discrete pairs: one kernel, or
// (MCLCCD_TUNE_EXPAND_SPLIT) the stencil expansion and the discrete test as
// two kernels.  Returns the launches made.
static int launch_expand(mclccd_tree *t, int dim, const int *dP, const double *dV1, int nv, int cont, bool discr,
                         Counters *cnt, cudaStream_t st, const unsigned long long *lo = nullptr,
                         const unsigned long long *hi = nullptr)
{
    if (t->tune[MCLCCD_TUNE_EXPAND_SPLIT] && discr && cont) {
        launch_expand_pairs(dim, as<int2>(t->pairs), t->cap_pairs, dP, as<unsigned char>(t->pflags), dV1, nv,
                            as<int4>(t->vf), t->cap_vf, as<int4>(t->ee), t->cap_ee, as<int2>(t->disc), t->cap_disc,
                            cont, 0, cnt, t->tune[MCLCCD_TUNE_EXPAND_GRID], st, lo, hi);
        launch_discrete_pairs(dim, as<int2>(t->pairs), t->cap_pairs, dP, dV1, nv, as<int2>(t->disc), t->cap_disc, cnt,
                              kDiscreteGrid, st, lo, hi, t->tune[MCLCCD_TUNE_EXPAND_SPLIT] == 2);
        return 2;
    }
    launch_expand_pairs(dim, as<int2>(t->pairs), t->cap_pairs, dP, as<unsigned char>(t->pflags), dV1, nv,
                        as<int4>(t->vf), t->cap_vf, as<int4>(t->ee), t->cap_ee, as<int2>(t->disc), t->cap_disc, cont,
                        discr, cnt, t->tune[MCLCCD_TUNE_EXPAND_GRID], st, lo, hi);
    return 1;
}

// Inputs in other forms than row-major double (float coordinates, column-
// major V or P): one pass converts them on the device into the row-major
// double / int arrays the path runs on.  Widening float -> double is exact.
template <typename T, bool COL>
__global__ void k_stage_positions(const T *__restrict__ a, const T *__restrict__ b, double *__restrict__ oa,
                                  double *__restrict__ ob, int nv, int dim)
{
    const long long n = (long long)nv * dim;
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n; s += (long long)gridDim.x * blockDim.x) {
        const long long d = COL ? (s % nv) * dim + s / nv : s;   // source index s -> row-major index d
        oa[d] = (double)a[s];
        ob[d] = (double)b[s];
    }
}

__global__ void k_stage_prims(const int *__restrict__ P, int *__restrict__ out, int np, int pdim)
{
    const long long n = (long long)np * pdim;
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n; s += (long long)gridDim.x * blockDim.x)
        out[(s % np) * pdim + s / np] = P[s];
}

static int stage_grid(long long n) { return (int)std::max<long long>(1, std::min<long long>((n + 255) / 256, 148 * 16)); }

// V0/V1 (in_flags form, mem_kind side) -> t->V0d/V1d (row-major double, device).
static int stage_positions(mclccd_tree *t, const void *V0, const void *V1, int nv, int mem_kind, unsigned in_flags)
{
    const int dim = t->dim;
    const long long n = (long long)nv * dim;
    const size_t esz = (in_flags & MCLCCD_IN_F32) ? sizeof(float) : sizeof(double);
    cudaStream_t st = t->stream;
    MC_CUDA(t, ensure(t->V0d, sizeof(double) * (size_t)n));
    MC_CUDA(t, ensure(t->V1d, sizeof(double) * (size_t)n));
    const void *a = V0, *b = V1;
    if (mem_kind == MCLCCD_MEM_HOST) {
        MC_CUDA(t, ensure(t->in_V, 2 * esz * (size_t)n));
        char *s = static_cast<char *>(t->in_V.p);
        MC_CUDA(t, cudaMemcpyAsync(s, V0, esz * (size_t)n, cudaMemcpyHostToDevice, st));
        MC_CUDA(t, cudaMemcpyAsync(s + esz * n, V1, esz * (size_t)n, cudaMemcpyHostToDevice, st));
        a = s;
        b = s + esz * n;
    }
    const bool col = (in_flags & MCLCCD_IN_V_COLMAJOR) != 0;
    double *oa = as<double>(t->V0d), *ob = as<double>(t->V1d);
    const int g = stage_grid(n);
    if (in_flags & MCLCCD_IN_F32) {
        if (col) k_stage_positions<float, true><<<g, 256, 0, st>>>((const float *)a, (const float *)b, oa, ob, nv, dim);
        else k_stage_positions<float, false><<<g, 256, 0, st>>>((const float *)a, (const float *)b, oa, ob, nv, dim);
    } else {
        k_stage_positions<double, true><<<g, 256, 0, st>>>((const double *)a, (const double *)b, oa, ob, nv, dim);
    }
    ++t->launches;
    MC_CUDA(t, cudaGetLastError());
    return MCLCCD_OK;
}

// An int array on the mem_kind side -> a device pointer; column-major P
// (slot j of primitive i at [j * np + i]) is transposed to row-major.
static int stage_ints(mclccd_tree *t, DevBuf &buf, DevBuf &tmp, const int *src, int rows, int cols, bool colmajor,
                      int mem_kind, const int *&out)
{
    out = src;
    if (!src) return MCLCCD_OK;
    const size_t count = (size_t)rows * cols;
    if (mem_kind == MCLCCD_MEM_HOST) {
        DevBuf &dst = colmajor ? tmp : buf;
        MC_CUDA(t, ensure(dst, sizeof(int) * std::max<size_t>(count, 1)));
        MC_CUDA(t, cudaMemcpyAsync(dst.p, src, sizeof(int) * count, cudaMemcpyHostToDevice, t->stream));
        out = as<int>(dst);
    }
    if (colmajor) {
        MC_CUDA(t, ensure(buf, sizeof(int) * std::max<size_t>(count, 1)));
        k_stage_prims<<<stage_grid((long long)count), 256, 0, t->stream>>>(out, as<int>(buf), rows, cols);
        ++t->launches;
        MC_CUDA(t, cudaGetLastError());
        out = as<int>(buf);
    }
    return MCLCCD_OK;
}

// Overlapped traverse: the queries in `chunks` ranges.  The walk of chunk
// c + 1 (high-priority stream) runs while chunk c's pairs are expanded and
// scored (low-priority stream), so the latency-bound walk and the FP64-bound
// narrow phase share the SMs.  Running counters are snapshotted between
// launches (ovl: pair, VF and EE list ends per chunk) to give each launch its
// range; the lists, hits and counts are the ones of the sequential order
// (only their order in the buffers differs).
template <typename Accd>
static int enqueue_overlapped(mclccd_tree *t, int chunks, int dim, int np, int nv, const int *dP, const double *dV0,
                              const double *dV1, bool discr, bool fused, Counters *cnt, Accd &accd)
{
    cudaStream_t st = t->stream;
    if (!t->s_walk) {
        int least = 0, greatest = 0;
        MC_CUDA(t, cudaDeviceGetStreamPriorityRange(&least, &greatest));
        MC_CUDA(t, cudaStreamCreateWithPriority(&t->s_walk, cudaStreamNonBlocking, greatest));
        MC_CUDA(t, cudaStreamCreateWithPriority(&t->s_narrow, cudaStreamNonBlocking, least));
        for (auto &e : t->ov_ev) MC_CUDA(t, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    MC_CUDA(t, ensure(t->ovl, sizeof(unsigned long long) * 3 * 17));
    unsigned long long *pe = as<unsigned long long>(t->ovl), *ve = pe + 17, *ee = ve + 17;
    MC_CUDA(t, cudaMemsetAsync(pe, 0, sizeof(unsigned long long) * 3 * 17, st));
    MC_CUDA(t, cudaEventRecord(t->ov_ev[0], st));   // fork
    MC_CUDA(t, cudaStreamWaitEvent(t->s_walk, t->ov_ev[0], 0));
    MC_CUDA(t, cudaStreamWaitEvent(t->s_narrow, t->ov_ev[0], 0));
    const int nq = np - 1;
    for (int c = 0; c < chunks; ++c) {
        const int qb = (int)((long long)nq * c / chunks), qe = (int)((long long)nq * (c + 1) / chunks);
        if (int rc = launch_walk(t, dim, 0, np, cnt, t->s_walk, qb, qe)) return rc;
        launch_snapshot(&cnt->n_pairs, pe + c + 1, nullptr, nullptr, t->s_walk);
        MC_CUDA(t, cudaEventRecord(t->ov_ev[1], t->s_walk));
        MC_CUDA(t, cudaStreamWaitEvent(t->s_narrow, t->ov_ev[1], 0));
        if (fused) {
            launch_narrow_fused(dim, as<int2>(t->pairs), t->cap_pairs, dP, as<unsigned char>(t->pflags), dV0, dV1, nv,
                                t->vf_eta, t->ee_eta, 1, discr, as<int2>(t->disc), t->cap_disc, as<int4>(t->hit_sten),
                                as<double>(t->hit_toi), as<unsigned char>(t->hit_isvf), t->cap_hits, cnt,
                                t->tune[MCLCCD_TUNE_FUSED_GRID], t->s_narrow, pe + c, pe + c + 1);
            t->launches += 2;
        } else {
            t->launches += launch_expand(t, dim, dP, dV1, nv, 1, discr, cnt, t->s_narrow, pe + c, pe + c + 1) - 1;
            launch_snapshot(&cnt->n_vf, ve + c + 1, &cnt->n_ee, ee + c + 1, t->s_narrow);
            accd(true, t->vf, ve + c + 1, t->cap_vf, t->vf_eta, ve + c, t->s_narrow);
            if (dim == 3) accd(false, t->ee, ee + c + 1, t->cap_ee, t->ee_eta, ee + c, t->s_narrow);
            t->launches += 4;
        }
    }
    MC_CUDA(t, cudaEventRecord(t->ov_ev[2], t->s_walk));   // join
    MC_CUDA(t, cudaEventRecord(t->ov_ev[3], t->s_narrow));
    MC_CUDA(t, cudaStreamWaitEvent(st, t->ov_ev[2], 0));
    MC_CUDA(t, cudaStreamWaitEvent(st, t->ov_ev[3], 0));
    if (t->flags & MCLCCD_OPT_PROFILE) {   // walk = all chunks' walks; expand = 0; narrow = the rest
        cudaEventRecord(t->ev[4], t->s_walk);
        cudaEventRecord(t->ev[5], t->s_walk);
    }
    return MCLCCD_OK;
}

// Caller buffers for the results of mclccd_traverse_out.
struct HostOut {
    int *sten;
    unsigned char *is_vf;
    double *toi;
    long long hit_cap;
    int *disc;
    long long disc_cap;
    int mem_kind;
};

// mclccd_traverse_out: the step in kOutChunks query chunks on the handle's
// stream; after each chunk's narrow phase its hits (appended after the
// previous chunks') are copied to the caller's host arrays on a copy stream
// while the next chunks compute.  The host waits on each chunk's event to
// learn its hit count (a pinned snapshot).  Copies stop at the caller's
// capacity; an overflow retry recomputes and copies again from the start.
constexpr int kOutChunks = 16;

template <typename Accd>
static int enqueue_streamed(mclccd_tree *t, int dim, int np, int nv, const int *dP, const double *dV0,
                            const double *dV1, bool discr, bool fused, Counters *cnt, Accd &accd, const HostOut &out)
{
    cudaStream_t st = t->stream;
    if (!t->s_copy) {
        MC_CUDA(t, cudaStreamCreateWithFlags(&t->s_copy, cudaStreamNonBlocking));
        for (auto &e : t->out_ev) MC_CUDA(t, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        MC_CUDA(t, cudaHostAlloc(reinterpret_cast<void **>(&t->h_snap), sizeof(unsigned long long) * 16, 0));
    }
    MC_CUDA(t, ensure(t->ovl, sizeof(unsigned long long) * 3 * 17));
    unsigned long long *pe = as<unsigned long long>(t->ovl), *ve = pe + 17, *ee = ve + 17;
    MC_CUDA(t, cudaMemsetAsync(pe, 0, sizeof(unsigned long long) * 3 * 17, st));
    const int nq = np - 1;
    for (int c = 0; c < kOutChunks; ++c) {
        const int qb = (int)((long long)nq * c / kOutChunks), qe = (int)((long long)nq * (c + 1) / kOutChunks);
        if (int rc = launch_walk(t, dim, 0, np, cnt, st, qb, qe)) return rc;
        launch_snapshot(&cnt->n_pairs, pe + c + 1, nullptr, nullptr, st);
        if (fused) {
            launch_narrow_fused(dim, as<int2>(t->pairs), t->cap_pairs, dP, as<unsigned char>(t->pflags), dV0, dV1, nv,
                                t->vf_eta, t->ee_eta, 1, discr, as<int2>(t->disc), t->cap_disc, as<int4>(t->hit_sten),
                                as<double>(t->hit_toi), as<unsigned char>(t->hit_isvf), t->cap_hits, cnt,
                                t->tune[MCLCCD_TUNE_FUSED_GRID], st, pe + c, pe + c + 1);
            t->launches += 3;
        } else {
            t->launches += launch_expand(t, dim, dP, dV1, nv, 1, discr, cnt, st, pe + c, pe + c + 1) - 1;
            launch_snapshot(&cnt->n_vf, ve + c + 1, &cnt->n_ee, ee + c + 1, st);
            accd(true, t->vf, ve + c + 1, t->cap_vf, t->vf_eta, ve + c, st);
            if (dim == 3) accd(false, t->ee, ee + c + 1, t->cap_ee, t->ee_eta, ee + c, st);
            t->launches += 4;
        }
        MC_CUDA(t, cudaMemcpyAsync(t->h_snap + c, &cnt->n_hits, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
        MC_CUDA(t, cudaEventRecord(t->out_ev[c], st));
    }
    if (t->flags & MCLCCD_OPT_PROFILE) {   // walk = the whole chunked step; expand, narrow = 0
        cudaEventRecord(t->ev[4], st);
        cudaEventRecord(t->ev[5], st);
    }
    if (int rc = check_launch(t, "traverse kernels")) return rc;
    // stream each chunk's hits out as soon as it is done
    unsigned long long done = 0;
    const unsigned long long lim = std::min<unsigned long long>((unsigned long long)std::max(out.hit_cap, 0ll),
                                                                t->cap_hits);
    for (int c = 0; c < kOutChunks; ++c) {
        MC_CUDA(t, cudaEventSynchronize(t->out_ev[c]));
        const unsigned long long upto = std::min<unsigned long long>(t->h_snap[c], lim);
        if (upto <= done) continue;
        const size_t n = (size_t)(upto - done);
        if (out.sten)
            MC_CUDA(t, cudaMemcpyAsync(out.sten + 4 * done, as<int4>(t->hit_sten) + done, sizeof(int4) * n,
                                       cudaMemcpyDeviceToHost, t->s_copy));
        if (out.is_vf)
            MC_CUDA(t, cudaMemcpyAsync(out.is_vf + done, as<unsigned char>(t->hit_isvf) + done, n,
                                       cudaMemcpyDeviceToHost, t->s_copy));
        if (out.toi)
            MC_CUDA(t, cudaMemcpyAsync(out.toi + done, as<double>(t->hit_toi) + done, sizeof(double) * n,
                                       cudaMemcpyDeviceToHost, t->s_copy));
        done = upto;
    }
    t->out_done = done;
    return MCLCCD_OK;
}

// The results of a successful traverse_out into the caller's buffers: the
// hits not streamed yet, then the discrete pairs.
static int deliver_out(mclccd_tree *t, const HostOut &out)
{
    cudaStream_t st = t->stream;
    const unsigned long long nh = std::min<unsigned long long>(t->n_hits, (unsigned long long)std::max(out.hit_cap, 0ll));
    const cudaMemcpyKind k = out.mem_kind == MCLCCD_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    const unsigned long long from = t->out_done < nh ? t->out_done : nh;
    if (nh > from) {
        const size_t n = (size_t)(nh - from);
        if (out.sten)
            MC_CUDA(t, cudaMemcpyAsync(out.sten + 4 * from, as<int4>(t->hit_sten) + from, sizeof(int4) * n, k, st));
        if (out.is_vf) MC_CUDA(t, cudaMemcpyAsync(out.is_vf + from, as<unsigned char>(t->hit_isvf) + from, n, k, st));
        if (out.toi)
            MC_CUDA(t, cudaMemcpyAsync(out.toi + from, as<double>(t->hit_toi) + from, sizeof(double) * n, k, st));
    }
    const unsigned long long nd = std::min<unsigned long long>(t->n_disc, (unsigned long long)std::max(out.disc_cap, 0ll));
    if (out.disc && nd) MC_CUDA(t, cudaMemcpyAsync(out.disc, t->disc.p, sizeof(int2) * nd, k, st));
    if (t->s_copy) MC_CUDA(t, cudaStreamSynchronize(t->s_copy));
    MC_CUDA(t, cudaStreamSynchronize(st));
    t->out_done = 0;
    return MCLCCD_OK;
}

extern "C" {

const char *mclccd_status_string(int s)
{
    switch (s) {
    case MCLCCD_OK: return "ok";
    case MCLCCD_ERR_INVALID: return "invalid argument";
    case MCLCCD_ERR_CUDA: return "CUDA error";
    case MCLCCD_ERR_NOMEM: return "out of device memory";
    case MCLCCD_ERR_OVERFLOW: return "output capacity too small";
    case MCLCCD_ERR_STATE: return "call out of order";
    case MCLCCD_ERR_DEVICE: return "device-side failure (bounded wait or stack)";
    case MCLCCD_ERR_UNSUPPORTED: return "unsupported option";
    case MCLCCD_ERR_SCRATCH_LIMIT: return "arrays exceed the fixed scratch of mclccd_narrow_phase_bulk_static";
    }
    return "unknown status";
}

const char *mclccd_last_error(const mclccd_tree *t) { return t ? t->err.c_str() : "null handle"; }

int mclccd_create(int dim, mclccd_tree **out)
{
    if (!out || (dim != 2 && dim != 3)) return MCLCCD_ERR_INVALID;
    *out = nullptr;
    mclccd_tree *t = new mclccd_tree();
    t->dim = dim;
    cudaError_t e = cudaGetDevice(&t->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&t->own_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMallocHost(&t->h_cnt, sizeof(Counters));
    if (e == cudaSuccess) e = cudaMallocHost(&t->h_diff, 2 * sizeof(int));
    if (e == cudaSuccess) e = cudaMallocHost(&t->h_quality, 2 * sizeof(double));
    for (int i = 0; i < 8 && e == cudaSuccess; ++i) e = cudaEventCreate(&t->ev[i]);
    if (e == cudaSuccess) e = ensure(t->counters, sizeof(Counters));
    if (e == cudaSuccess) e = ensure(t->diff, 2 * sizeof(int));
    if (e != cudaSuccess) {
        mclccd_destroy(t);
        return e == cudaErrorMemoryAllocation ? MCLCCD_ERR_NOMEM : MCLCCD_ERR_CUDA;
    }
    t->stream = t->own_stream;
    *out = t;
    return MCLCCD_OK;
}

int mclccd_destroy(mclccd_tree *t)
{
    if (!t) return MCLCCD_ERR_INVALID;
    DeviceGuard g(t->device);
    if (t->stream) cudaStreamSynchronize(t->stream);
    for (DevBuf *b : t->all())
        if (b->p) cudaFree(b->p);
    for (int i = 0; i < 8; ++i)
        if (t->ev[i]) cudaEventDestroy(t->ev[i]);
    for (int i = 0; i < 4; ++i)
        if (t->ov_ev[i]) cudaEventDestroy(t->ov_ev[i]);
    if (t->s_walk) cudaStreamDestroy(t->s_walk);
    if (t->s_copy) cudaStreamSynchronize(t->s_copy), cudaStreamDestroy(t->s_copy);
    for (auto e : t->out_ev)
        if (e) cudaEventDestroy(e);
    if (t->h_snap) cudaFreeHost(t->h_snap);
    if (t->s_narrow) cudaStreamDestroy(t->s_narrow);
    if (t->ovl.p) cudaFree(t->ovl.p);
    if (t->h_cnt) cudaFreeHost(t->h_cnt);
    if (t->h_diff) cudaFreeHost(t->h_diff);
    if (t->h_quality) cudaFreeHost(t->h_quality);
    if (t->own_stream) cudaStreamDestroy(t->own_stream);
    delete t;
    return MCLCCD_OK;
}

int mclccd_set_options(mclccd_tree *t, double box_eta, double vf, double ee, unsigned flags)
{
    if (!t) return MCLCCD_ERR_INVALID;
    if (!(box_eta >= 0) || !(vf >= 0) || !(ee >= 0)) return fail(t, MCLCCD_ERR_INVALID, "etas must be >= 0");
    t->box_eta = box_eta;
    t->vf_eta = vf;
    t->ee_eta = ee;
    t->flags = flags;
    return MCLCCD_OK;
}

int mclccd_get_options(const mclccd_tree *t, double *box_eta, double *vf, double *ee, unsigned *flags)
{
    if (!t) return MCLCCD_ERR_INVALID;
    if (box_eta) *box_eta = t->box_eta;
    if (vf) *vf = t->vf_eta;
    if (ee) *ee = t->ee_eta;
    if (flags) *flags = t->flags;
    return MCLCCD_OK;
}

int mclccd_set_stream(mclccd_tree *t, void *stream)
{
    if (!t) return MCLCCD_ERR_INVALID;
    t->stream = stream ? static_cast<cudaStream_t>(stream) : t->own_stream;
    return MCLCCD_OK;
}

int mclccd_set_precision(mclccd_tree *t, int precision)
{
    if (!t) return MCLCCD_ERR_INVALID;
    if (precision != MCLCCD_PREC_FP64 && precision != MCLCCD_PREC_FP32_CERTIFIED)
        return fail(t, MCLCCD_ERR_INVALID, "unknown precision");
    t->precision = precision;
    return MCLCCD_OK;
}

int mclccd_update(mclccd_tree *t, const double *V0, const double *V1, int nv, const int *P, int np, int pdim,
                  const int *active, int mem_kind)
{
    if (!t) return MCLCCD_ERR_INVALID;
    t->err.clear();
    if (mem_kind != MCLCCD_MEM_HOST && mem_kind != MCLCCD_MEM_DEVICE) return fail(t, MCLCCD_ERR_INVALID, "bad mem_kind");
    if (np < 0 || nv < 0) return fail(t, MCLCCD_ERR_INVALID, "negative size");
    if (!(t->box_eta >= 0) || !(t->vf_eta >= 0) || !(t->ee_eta >= 0)) return fail(t, MCLCCD_ERR_INVALID, "etas must be >= 0");
    // BVHTree.cpp:39-40: the narrow-phase gaps never exceed the box padding.
    t->vf_eta = std::min(t->vf_eta, t->box_eta);
    t->ee_eta = std::min(t->ee_eta, t->box_eta);
    t->traversed = false;
    if (np == 0) {   // BVHTree.cpp:29-34: clear
        t->built = true;
        t->np = 0;
        t->pdim = pdim;
        t->nv = nv;
        t->flags_np = 0;
        return MCLCCD_OK;
    }
    if (!V0 || !V1 || !P || nv < 0) return fail(t, MCLCCD_ERR_INVALID, "null array or nv < 0");
    if (pdim < 1 || pdim > 4) return fail(t, MCLCCD_ERR_INVALID, "pdim must be in [1, 4]");
    DeviceGuard g(t->device);
    cudaStream_t st = t->stream;
    const int dim = t->dim;
    const bool prof = (t->flags & MCLCCD_OPT_PROFILE) != 0;
    if (prof) cudaEventRecord(t->ev[0], st);
    const long long pcount = (long long)np * pdim;
    const size_t pbytes = sizeof(int) * (size_t)pcount;
    // The incoming P as the device reads it: the caller's device array as it
    // is, or one copy of host P.  The handle's own copy (Pd) is rewritten
    // only when the topology changed.
    const bool dev_p = mem_kind == MCLCCD_MEM_DEVICE;
    if (!dev_p) {
        MC_CUDA(t, ensure(t->Pstage, pbytes));
        MC_CUDA(t, cudaMemcpyAsync(t->Pstage.p, P, pbytes, cudaMemcpyHostToDevice, st));
    }
    const int *inP = dev_p ? P : as<int>(t->Pstage);
    // Pd := the incoming P
    auto adopt_p = [&]() -> cudaError_t {
        if (!dev_p) {
            std::swap(t->Pstage, t->Pd);
            return cudaSuccess;
        }
        cudaError_t e = ensure(t->Pd, pbytes);
        if (e == cudaSuccess) e = cudaMemcpyAsync(t->Pd.p, P, pbytes, cudaMemcpyDeviceToDevice, st);
        return e;
    };
    // Refit-only when the topology is byte-identical to the previous update.
    const bool may_refit = t->built && t->np > 1 && !(t->flags & MCLCCD_OPT_ALWAYS_REBUILD) && np == t->np &&
                           pdim == t->pdim && !t->force_rebuild;
    int p_known = -1;   // -1: P not compared yet; 0 / 1: P differs / equals the stored P
    const bool derive_nv = nv == 0;
    if (derive_nv) {
        // The reference's update carries no vertex count: it is 1 + the
        // largest index in P, found on the device (with the refit check's
        // compare, one small read-back).
        MC_CUDA(t, cudaMemsetAsync(t->diff.p, 0, 2 * sizeof(int), st));
        launch_max_index(inP, pcount, as<int>(t->diff) + 1, st);
        ++t->launches;
        if (may_refit) {
            launch_compare(inP, as<int>(t->Pd), pcount, as<int>(t->diff), st);
            ++t->launches;
        }
        MC_CUDA(t, cudaMemcpyAsync(t->h_diff, t->diff.p, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
        MC_CUDA(t, cudaStreamSynchronize(st));
        nv = t->h_diff[1];
        if (nv <= 0) return fail(t, MCLCCD_ERR_INVALID, "nv == 0 and P holds no vertex index >= 0");
        if (may_refit) p_known = t->h_diff[0] == 0 ? 1 : 0;
    }

    const double *dV0 = V0, *dV1 = V1;
    const int *dact = active;
    const size_t vbytes = sizeof(double) * (size_t)nv * dim;
    if (mem_kind == MCLCCD_MEM_HOST) {
        MC_CUDA(t, ensure(t->V0d, vbytes));
        MC_CUDA(t, ensure(t->V1d, vbytes));
        MC_CUDA(t, cudaMemcpyAsync(t->V0d.p, V0, vbytes, cudaMemcpyHostToDevice, st));
        MC_CUDA(t, cudaMemcpyAsync(t->V1d.p, V1, vbytes, cudaMemcpyHostToDevice, st));
        dV0 = as<double>(t->V0d);
        dV1 = as<double>(t->V1d);
        if (active) {
            MC_CUDA(t, ensure(t->actd, sizeof(int) * (size_t)nv));
            MC_CUDA(t, cudaMemcpyAsync(t->actd.p, active, sizeof(int) * (size_t)nv, cudaMemcpyHostToDevice, st));
            dact = as<int>(t->actd);
        }
    }
    MC_CUDA(t, cudaMemsetAsync(t->counters.p, 0, sizeof(Counters), st));

    bool same = may_refit && nv == t->nv;
    // P still to be compared: the refit is launched before the answer is
    // known (it runs while the host waits for the comparison alone), and a
    // differing P adds the full build after it.
    bool speculate = false;
    if (same && p_known >= 0) {
        same = p_known == 1;
    } else if (same) {
        MC_CUDA(t, cudaMemsetAsync(t->diff.p, 0, sizeof(int), st));
        launch_compare(inP, as<int>(t->Pd), pcount, as<int>(t->diff), st);
        ++t->launches;
        MC_CUDA(t, cudaMemcpyAsync(t->h_diff, t->diff.p, sizeof(int), cudaMemcpyDeviceToHost, st));
        MC_CUDA(t, cudaEventRecord(t->ev[7], st));
        speculate = true;
    }
    if (!speculate && !same) MC_CUDA(t, adopt_p());
    const int *dP = as<int>(t->Pd);   // (reassigned when the comparison after a speculative refit fails)
    Counters *cnt = as<Counters>(t->counters);

    // Representative flags: recomputed only when the primitive count changes
    // (BVHTree.cpp:44-48); new leaves default to "all represented" and old
    // leaves keep their flags when reptri is off (BVHLeaf.hpp:45-49).
    if (np != t->flags_np) {
        MC_CUDA(t, ensure(t->pflags_tmp, (size_t)np));
        MC_CUDA(t, cudaMemsetAsync(t->pflags_tmp.p, (int)kFlagAllRep, (size_t)np, st));
        if (t->flags_np > 0 && t->pflags.p)
            MC_CUDA(t, cudaMemcpyAsync(t->pflags_tmp.p, t->pflags.p, (size_t)std::min(np, t->flags_np),
                                       cudaMemcpyDeviceToDevice, st));
        std::swap(t->pflags, t->pflags_tmp);
        if ((t->flags & MCLCCD_OPT_REPTRI) && (pdim == 2 || pdim == 3)) {
            unsigned long long ecap = 1024;
            while (ecap < (unsigned long long)pcount * 2) ecap <<= 1;
            MC_CUDA(t, ensure(t->vowner, sizeof(int) * (size_t)nv));
            if (pdim == 3) {
                MC_CUDA(t, ensure(t->ekeys, sizeof(unsigned long long) * ecap));
                MC_CUDA(t, ensure(t->eowner, sizeof(int) * ecap));
            }
            launch_owner_flags(dP, np, pdim, nv, as<int>(t->vowner), as<unsigned long long>(t->ekeys),
                               as<int>(t->eowner), ecap, as<unsigned char>(t->pflags), cnt, st);
            t->launches += 2;
        }
        t->flags_np = np;
    }

    MC_CUDA(t, ensure(t->leaf_box, sizeof(double) * 4 * dim * (size_t)np));
    MC_CUDA(t, ensure(t->leaf_active, (size_t)np));
    MC_CUDA(t, ensure(t->visits, sizeof(int) * (size_t)std::max(1, np - 1)));
    // the refit, with the tree-quality sum after every build and every
    // kQualityEvery-th refit (box areas of the internal nodes and of the
    // leaves)
    bool track = false;
    auto refit = [&](bool built) -> int {
        track = np > 1 && t->tune[MCLCCD_TUNE_REBUILD_RATIO] > 0 &&
                (built || ++t->refits_since_check % kQualityEvery == 0);
        launch_refit(dim, dV0, dV1, dP, np, pdim, nv, t->box_eta, dact, as<int>(t->vals), as<int>(t->leaf_parent),
                     as<Node>(t->nodes), as<int>(t->visits), t->leaf_box.p, as<unsigned char>(t->leaf_active), cnt, st);
        ++t->launches;
        if (track) {
            MC_CUDA(t, ensure(t->quality, 2 * sizeof(double)));
            launch_tree_quality(dim, as<Node>(t->nodes), np, as<double>(t->quality), st);
            ++t->launches;
        }
        return check_launch(t, "refit kernel");
    };
    if (speculate) {
        if (prof) cudaEventRecord(t->ev[1], st);
        if (int rc = refit(false)) return rc;
        MC_CUDA(t, cudaEventSynchronize(t->ev[7]));
        same = *t->h_diff == 0;
        if (!same) {
            MC_CUDA(t, adopt_p());
            dP = as<int>(t->Pd);
        }
    }
    if (!same) {
        MC_CUDA(t, ensure(t->cent, sizeof(float) * (size_t)np * dim));
        MC_CUDA(t, ensure(t->bounds, sizeof(unsigned) * 8));
        MC_CUDA(t, ensure(t->keys, sizeof(unsigned) * (size_t)np));
        MC_CUDA(t, ensure(t->vals, sizeof(int) * (size_t)np));
        MC_CUDA(t, ensure(t->keys_alt, sizeof(unsigned) * (size_t)np));
        MC_CUDA(t, ensure(t->vals_alt, sizeof(int) * (size_t)np));
        MC_CUDA(t, ensure(t->sort_scratch, sort_scratch_bytes(np, sort_num_passes(30))));
        MC_CUDA(t, ensure(t->nodes, sizeof(Node) * (size_t)std::max(1, np - 1)));
        MC_CUDA(t, ensure(t->leaf_parent, sizeof(int) * (size_t)np));
        launch_centroids(dim, dV0, dV1, dP, np, pdim, nv, as<float>(t->cent), as<unsigned>(t->bounds), cnt, st);
        launch_morton(dim, as<float>(t->cent), np, as<unsigned>(t->bounds), as<unsigned>(t->keys), as<int>(t->vals), st);
        launch_sort_pairs(as<unsigned>(t->keys), as<int>(t->vals), as<unsigned>(t->keys_alt), as<int>(t->vals_alt), np,
                          30, t->sort_scratch.p, cnt, st);
        launch_karras(as<unsigned>(t->keys), np, as<Node>(t->nodes), as<int>(t->leaf_parent), st);
        t->launches += 4 + 1 + sort_num_passes(30) + (np > 1 ? 1 : 0);
        if (int rc = check_launch(t, "build kernels")) return rc;
    }
    if (!speculate || !same) {
        if (prof && !speculate) cudaEventRecord(t->ev[1], st);
        if (int rc = refit(!same)) return rc;
    }
    if (prof) cudaEventRecord(t->ev[2], st);
    MC_CUDA(t, cudaMemcpyAsync(t->h_cnt, cnt, sizeof(Counters), cudaMemcpyDeviceToHost, st));
    if (track)
        MC_CUDA(t, cudaMemcpyAsync(t->h_quality, t->quality.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
    MC_CUDA(t, cudaStreamSynchronize(st));
    if (!same) ++t->n_builds;
    if (t->force_rebuild && !same) ++t->n_quality_rebuilds;
    t->force_rebuild = false;
    if (track) {
        // quality = internal-node box areas / leaf box areas (the surface-area
        // cost of the hierarchy, normalised by the geometry's own).  A
        // refit-only tree whose quality grew past the ratio of the last
        // build's is rebuilt at the next update: the Morton order of the
        // positions it was built from no longer fits the motion.
        const double inner = t->h_quality[0], leaves = t->h_quality[1];
        const double q = leaves > 0.0 ? inner / leaves : 0.0;
        if (!same) t->q_build = q;
        else if (t->q_build > 0.0 && q > t->q_build * (t->tune[MCLCCD_TUNE_REBUILD_RATIO] / 100.0))
            t->force_rebuild = true;
    }
    if (prof) {
        cudaEventElapsedTime(&t->stage[0], t->ev[0], t->ev[2]);
        cudaEventElapsedTime(&t->stage[1], t->ev[0], t->ev[1]);
        cudaEventElapsedTime(&t->stage[2], t->ev[1], t->ev[2]);
    }
    t->np = np;
    t->pdim = pdim;
    t->nv = nv;
    t->upd_V0 = dV0;
    t->upd_V1 = dV1;
    const unsigned derr = t->h_cnt->err;
    t->built = derr == 0;
    if (derr) return device_errors(t, derr);
    return MCLCCD_OK;
}

int mclccd_update_ex(mclccd_tree *t, const void *V0, const void *V1, int nv, const int *P, int np, int pdim,
                     const int *active, int mem_kind, unsigned in_flags)
{
    if (!t) return MCLCCD_ERR_INVALID;
    if (in_flags & ~(MCLCCD_IN_F32 | MCLCCD_IN_V_COLMAJOR | MCLCCD_IN_P_COLMAJOR))
        return fail(t, MCLCCD_ERR_INVALID, "unknown input flags");
    if (in_flags == 0)
        return mclccd_update(t, (const double *)V0, (const double *)V1, nv, P, np, pdim, active, mem_kind);
    t->err.clear();
    if (mem_kind != MCLCCD_MEM_HOST && mem_kind != MCLCCD_MEM_DEVICE) return fail(t, MCLCCD_ERR_INVALID, "bad mem_kind");
    if (np < 0 || nv < 0) return fail(t, MCLCCD_ERR_INVALID, "negative size");
    if (np == 0) return mclccd_update(t, nullptr, nullptr, nv, nullptr, 0, pdim, nullptr, MCLCCD_MEM_DEVICE);
    if (!V0 || !V1 || !P || nv <= 0) return fail(t, MCLCCD_ERR_INVALID, "null array or nv == 0");
    if (pdim < 1 || pdim > 4) return fail(t, MCLCCD_ERR_INVALID, "pdim must be in [1, 4]");
    DeviceGuard g(t->device);
    const int *dP = nullptr, *dact = nullptr;
    const bool pcol = (in_flags & MCLCCD_IN_P_COLMAJOR) != 0;
    if (in_flags & (MCLCCD_IN_F32 | MCLCCD_IN_V_COLMAJOR)) {
        if (int rc = stage_positions(t, V0, V1, nv, mem_kind, in_flags)) return rc;
    } else if (mem_kind == MCLCCD_MEM_HOST) {   // row-major double on the host: plain copies
        const size_t vb = sizeof(double) * (size_t)nv * t->dim;
        MC_CUDA(t, ensure(t->V0d, vb));
        MC_CUDA(t, ensure(t->V1d, vb));
        MC_CUDA(t, cudaMemcpyAsync(t->V0d.p, V0, vb, cudaMemcpyHostToDevice, t->stream));
        MC_CUDA(t, cudaMemcpyAsync(t->V1d.p, V1, vb, cudaMemcpyHostToDevice, t->stream));
    }
    const bool vdev = !(in_flags & (MCLCCD_IN_F32 | MCLCCD_IN_V_COLMAJOR)) && mem_kind == MCLCCD_MEM_DEVICE;
    if (int rc = stage_ints(t, t->in_P, t->in_tmp, P, np, pdim, pcol, mem_kind, dP)) return rc;
    if (int rc = stage_ints(t, t->in_act, t->in_tmp, active, nv, 1, false, mem_kind, dact)) return rc;
    const double *a = vdev ? (const double *)V0 : as<double>(t->V0d), *b = vdev ? (const double *)V1 : as<double>(t->V1d);
    return mclccd_update(t, a, b, nv, dP, np, pdim, dact, MCLCCD_MEM_DEVICE);
}

int mclccd_traverse_ex(mclccd_tree *t, const void *V0, const void *V1, int nv, const int *P, int mem_kind,
                       unsigned in_flags)
{
    if (!t) return MCLCCD_ERR_INVALID;
    if (in_flags & ~(MCLCCD_IN_F32 | MCLCCD_IN_V_COLMAJOR | MCLCCD_IN_P_COLMAJOR))
        return fail(t, MCLCCD_ERR_INVALID, "unknown input flags");
    if (in_flags == 0 || (!V0 && !V1 && !P))
        return mclccd_traverse(t, (const double *)V0, (const double *)V1, nv, P, mem_kind);
    t->err.clear();
    if (!V0 || !V1 || !P) return fail(t, MCLCCD_ERR_INVALID, "V0, V1, P must all be given (or all NULL)");
    if (mem_kind != MCLCCD_MEM_HOST && mem_kind != MCLCCD_MEM_DEVICE) return fail(t, MCLCCD_ERR_INVALID, "bad mem_kind");
    if (!t->built) return fail(t, MCLCCD_ERR_STATE, "traverse before a successful update");
    if (nv <= 0) nv = t->nv;
    DeviceGuard g(t->device);
    const int *dP = nullptr;
    const bool vconv = (in_flags & (MCLCCD_IN_F32 | MCLCCD_IN_V_COLMAJOR)) != 0;
    if (vconv) {
        if (int rc = stage_positions(t, V0, V1, nv, mem_kind, in_flags)) return rc;
    } else if (mem_kind == MCLCCD_MEM_HOST) {
        const size_t vb = sizeof(double) * (size_t)nv * t->dim;
        MC_CUDA(t, ensure(t->V0d, vb));
        MC_CUDA(t, ensure(t->V1d, vb));
        MC_CUDA(t, cudaMemcpyAsync(t->V0d.p, V0, vb, cudaMemcpyHostToDevice, t->stream));
        MC_CUDA(t, cudaMemcpyAsync(t->V1d.p, V1, vb, cudaMemcpyHostToDevice, t->stream));
    }
    if (int rc = stage_ints(t, t->in_P, t->in_tmp, P, t->np, t->dim, (in_flags & MCLCCD_IN_P_COLMAJOR) != 0,
                            mem_kind, dP))
        return rc;
    const bool vdev = !vconv && mem_kind == MCLCCD_MEM_DEVICE;
    const double *a = vdev ? (const double *)V0 : as<double>(t->V0d), *b = vdev ? (const double *)V1 : as<double>(t->V1d);
    if (!vdev) {   // the update's arrays were overwritten
        t->upd_V0 = a;
        t->upd_V1 = b;
    }
    return mclccd_traverse(t, a, b, nv, dP, MCLCCD_MEM_DEVICE);
}

int mclccd_update_f32(mclccd_tree *t, const float *V0, const float *V1, int nv, const int *P, int np, int pdim,
                      const int *active, int mem_kind)
{
    return mclccd_update_ex(t, V0, V1, nv, P, np, pdim, active, mem_kind, MCLCCD_IN_F32);
}

int mclccd_traverse_f32(mclccd_tree *t, const float *V0, const float *V1, int nv, const int *P, int mem_kind)
{
    return mclccd_traverse_ex(t, V0, V1, nv, P, mem_kind, MCLCCD_IN_F32);
}

static int traverse_impl(mclccd_tree *t, const double *V0, const double *V1, int nv, const int *P, int mem_kind,
                         const HostOut *out);

int mclccd_traverse(mclccd_tree *t, const double *V0, const double *V1, int nv, const int *P, int mem_kind)
{
    if (!t) return MCLCCD_ERR_INVALID;
    return traverse_impl(t, V0, V1, nv, P, mem_kind, nullptr);
}

static int traverse_impl(mclccd_tree *t, const double *V0, const double *V1, int nv, const int *P, int mem_kind,
                         const HostOut *out)
{
    t->err.clear();
    if (!t->built) return fail(t, MCLCCD_ERR_STATE, "traverse before a successful update");
    if (mem_kind != MCLCCD_MEM_HOST && mem_kind != MCLCCD_MEM_DEVICE) return fail(t, MCLCCD_ERR_INVALID, "bad mem_kind");
    t->n_pairs = t->n_vf = t->n_ee = t->n_hits = t->n_disc = 0;
    t->traversed = true;
    if (t->np <= 1) return MCLCCD_OK;   // BVHTree.cpp:131-132
    const int dim = t->dim;
    if (t->pdim != dim)
        return fail(t, MCLCCD_ERR_INVALID, "traverse needs P as triangles (3D) or edges (2D): pdim must equal dim");
    DeviceGuard g(t->device);
    cudaStream_t st = t->stream;
    const bool prof = (t->flags & MCLCCD_OPT_PROFILE) != 0;
    if (prof) cudaEventRecord(t->ev[3], st);

    const double *dV0, *dV1;
    const int *dP;
    if (!V0 && !V1 && !P) {
        dV0 = t->upd_V0;
        dV1 = t->upd_V1;
        dP = as<int>(t->Pd);
        nv = t->nv;
    } else {
        if (!V0 || !V1 || !P) return fail(t, MCLCCD_ERR_INVALID, "V0, V1, P must all be given (or all NULL)");
        if (nv <= 0) nv = t->nv;
        dV0 = V0;
        dV1 = V1;
        dP = P;
        if (mem_kind == MCLCCD_MEM_HOST) {
            const size_t vbytes = sizeof(double) * (size_t)nv * dim;
            const size_t pbytes = sizeof(int) * (size_t)t->np * dim;
            MC_CUDA(t, ensure(t->V0d, vbytes));
            MC_CUDA(t, ensure(t->V1d, vbytes));
            MC_CUDA(t, ensure(t->Pstage, pbytes));
            MC_CUDA(t, cudaMemcpyAsync(t->V0d.p, V0, vbytes, cudaMemcpyHostToDevice, st));
            MC_CUDA(t, cudaMemcpyAsync(t->V1d.p, V1, vbytes, cudaMemcpyHostToDevice, st));
            MC_CUDA(t, cudaMemcpyAsync(t->Pstage.p, P, pbytes, cudaMemcpyHostToDevice, st));
            dV0 = as<double>(t->V0d);
            dV1 = as<double>(t->V1d);
            dP = as<int>(t->Pstage);
            t->upd_V0 = dV0;   // the update's copies were overwritten
            t->upd_V1 = dV1;
        }
    }
    const int np = t->np;
    t->tr_V0 = dV0;
    t->tr_V1 = dV1;
    t->tr_nv = nv;
    const bool cont = (t->flags & MCLCCD_OPT_CONTINUOUS) != 0;
    const bool discr = (t->flags & MCLCCD_OPT_DISCRETE) != 0;
    if (t->cap_pairs == 0) {
        t->cap_pairs = std::max<unsigned long long>(4096, 8ull * np);
        t->cap_vf = std::max<unsigned long long>(4096, 8ull * np);
        t->cap_ee = std::max<unsigned long long>(4096, dim == 3 ? 16ull * np : 16);
        t->cap_hits = t->cap_vf + t->cap_ee;
        t->cap_disc = std::max<unsigned long long>(1024, np / 4);
    }
    Counters *cnt = as<Counters>(t->counters);
    const bool one_sided = (t->flags & MCLCCD_OPT_VF_ONE_SIDED) != 0;
    const bool certified = t->precision == MCLCCD_PREC_FP32_CERTIFIED;
    // FP64 ACCD on both kinds: the fused kernel unless the list form is asked for
    const bool fused = cont && !one_sided && !certified && !t->tune[MCLCCD_TUNE_ACCD_REBIN] &&
                       t->tune[MCLCCD_TUNE_NARROW_FUSED] != 0;
    t->cand_lazy = fused;
    t->cand_ready = false;
    t->tr_P = dP;
    for (int attempt = 0;; ++attempt) {
        MC_CUDA(t, ensure(t->pairs, sizeof(int2) * t->cap_pairs));
        if (!fused) {
            MC_CUDA(t, ensure(t->vf, sizeof(int4) * t->cap_vf));
            MC_CUDA(t, ensure(t->ee, sizeof(int4) * t->cap_ee));
        }
        MC_CUDA(t, ensure(t->hit_sten, sizeof(int4) * t->cap_hits));
        MC_CUDA(t, ensure(t->hit_toi, sizeof(double) * t->cap_hits));
        MC_CUDA(t, ensure(t->hit_isvf, t->cap_hits));
        MC_CUDA(t, ensure(t->disc, sizeof(int2) * t->cap_disc));
        if (cont && !fused && !certified && t->tune[MCLCCD_TUNE_ACCD_REBIN] == 2) {
            const size_t qn = std::max(t->cap_vf, t->cap_ee);
            MC_CUDA(t, ensure(t->tq_idx, sizeof(unsigned) * qn));
            MC_CUDA(t, ensure(t->tq_state, sizeof(double2) * qn));
            MC_CUDA(t, ensure(t->tq_count, sizeof(unsigned long long)));
        }
        if (certified && cont) MC_CUDA(t, ensure(t->fp64_queue, sizeof(unsigned) * std::max(t->cap_vf, t->cap_ee)));
        MC_CUDA(t, cudaMemsetAsync(cnt, 0, sizeof(Counters), st));
        // narrow phase of one list, stencils [*lo, *n) (lo == nullptr: from 0)
        auto accd = [&](bool vf, DevBuf &list, const unsigned long long *n_ptr, unsigned long long cap, double eta,
                        const unsigned long long *lo, cudaStream_t s) {
            if (vf && one_sided) {   // BVHTree.cpp:445-447: CTCD with the wrong-side test
                launch_ctcd_pipeline(dim, as<int4>(list), n_ptr, cap, dV0, dV1, nv, eta, as<int4>(t->hit_sten),
                                     as<double>(t->hit_toi), as<unsigned char>(t->hit_isvf), t->cap_hits, cnt,
                                     t->tune[MCLCCD_TUNE_ACCD_GRID], s, lo);
                ++t->launches;
            } else if (certified) {   // an FP32 pass and an FP64 pass over its queue
                launch_accd_certified(dim, vf, as<int4>(list), n_ptr, cap, dV0, dV1, nv, eta, as<int4>(t->hit_sten),
                                      as<double>(t->hit_toi), as<unsigned char>(t->hit_isvf), t->cap_hits,
                                      as<unsigned>(t->fp64_queue), cnt, t->tune[MCLCCD_TUNE_ACCD_GRID], s);
                t->launches += 2;
            } else if (t->tune[MCLCCD_TUNE_ACCD_REBIN] == 2) {   // head and tail kernels over a queue
                launch_accd_split(dim, vf, as<int4>(list), n_ptr, cap, dV0, dV1, nv, eta, as<int4>(t->hit_sten),
                                  as<double>(t->hit_toi), as<unsigned char>(t->hit_isvf), t->cap_hits, cnt,
                                  t->tune[MCLCCD_TUNE_ACCD_GRID], as<unsigned>(t->tq_idx), as<double2>(t->tq_state),
                                  as<unsigned long long>(t->tq_count), s, lo);
                t->launches += 2;
            } else {
                launch_accd_pipeline(dim, vf, as<int4>(list), n_ptr, cap, dV0, dV1, nv, eta, as<int4>(t->hit_sten),
                                     as<double>(t->hit_toi), as<unsigned char>(t->hit_isvf), t->cap_hits, cnt,
                                     t->tune[MCLCCD_TUNE_ACCD_GRID], t->tune[MCLCCD_TUNE_ACCD_REBIN] == 1, s, lo);
                ++t->launches;
            }
        };
        const int chunks = t->tune[MCLCCD_TUNE_OVERLAP];
        // host results stream out chunk by chunk while later chunks compute
        const bool stream_out = out && out->mem_kind == MCLCCD_MEM_HOST && cont && !certified &&
                                !t->tune[MCLCCD_TUNE_WALK_PACKET] && np > 2 * kOutChunks * 128;
        if (stream_out) {
            if (int rc = enqueue_streamed(t, dim, np, nv, dP, dV0, dV1, discr, fused, cnt, accd, *out)) return rc;
        } else if (chunks >= 2 && cont && !certified && !t->tune[MCLCCD_TUNE_WALK_PACKET] && np > 2 * chunks * 128) {
            if (int rc = enqueue_overlapped(t, chunks, dim, np, nv, dP, dV0, dV1, discr, fused, cnt, accd)) return rc;
        } else {
            if (int rc = launch_walk(t, dim, t->tune[MCLCCD_TUNE_WALK_PACKET], np, cnt, st)) return rc;
            if (prof) cudaEventRecord(t->ev[4], st);
            if (fused) {   // expansion, discrete test and ACCD in one kernel: "expand" reads 0
                if (prof) cudaEventRecord(t->ev[5], st);
                launch_narrow_fused(dim, as<int2>(t->pairs), t->cap_pairs, dP, as<unsigned char>(t->pflags), dV0, dV1,
                                    nv, t->vf_eta, t->ee_eta, 1, discr, as<int2>(t->disc), t->cap_disc,
                                    as<int4>(t->hit_sten), as<double>(t->hit_toi), as<unsigned char>(t->hit_isvf),
                                    t->cap_hits, cnt, t->tune[MCLCCD_TUNE_FUSED_GRID], st);
                t->launches += 2;
            } else {
                t->launches += launch_expand(t, dim, dP, dV1, nv, cont, discr, cnt, st) - 1;
                if (prof) cudaEventRecord(t->ev[5], st);
                t->launches += 2;
                if (cont) {
                    accd(true, t->vf, &cnt->n_vf, t->cap_vf, t->vf_eta, nullptr, st);
                    if (dim == 3) accd(false, t->ee, &cnt->n_ee, t->cap_ee, t->ee_eta, nullptr, st);
                }
            }
        }
        if (prof) cudaEventRecord(t->ev[6], st);
        if (int rc = check_launch(t, "traverse kernels")) return rc;
        MC_CUDA(t, cudaMemcpyAsync(t->h_cnt, cnt, sizeof(Counters), cudaMemcpyDeviceToHost, st));
        MC_CUDA(t, cudaStreamSynchronize(st));
        const Counters &c = *t->h_cnt;
        bool grow = false;
        auto need = [&](double count, unsigned long long &cap) {
            if (count > (double)cap) { cap = (unsigned long long)(count * 1.25) + 1024; grow = true; }
        };
        // Stencil and discrete counts only cover the leaf pairs that fit; scale
        // them by the leaf-pair shortfall so one regrow usually suffices.
        const double r = c.n_pairs > t->cap_pairs ? (double)c.n_pairs / (double)t->cap_pairs : 1.0;
        need((double)c.n_pairs, t->cap_pairs);
        need(r * (double)c.n_discrete, t->cap_disc);
        if (fused) {   // no candidate lists: only the hits need room
            need(r * (double)c.n_hits, t->cap_hits);
        } else {
            // hits were counted over the stencils that fit their lists: scale
            // by that shortfall too (the hit list is sized by its own count,
            // not by the candidates, which can be many more)
            const double done = (double)(std::min(c.n_vf, t->cap_vf) + std::min(c.n_ee, t->cap_ee));
            const double rh = r * (done > 0 ? (double)(c.n_vf + c.n_ee) / done : 1.0);
            need(r * (double)c.n_vf, t->cap_vf);
            need(r * (double)c.n_ee, t->cap_ee);
            need(rh * (double)c.n_hits, t->cap_hits);
        }
        if (!grow) break;
        // a retry regrows and rewrites the device lists: let copies of this
        // attempt's hits (streamed results) finish first
        if (t->s_copy) MC_CUDA(t, cudaStreamSynchronize(t->s_copy));
        t->out_done = 0;
        if (attempt + 1 >= kMaxAttempts) return fail(t, MCLCCD_ERR_DEVICE, "result buffers kept overflowing");
    }
    const Counters &c = *t->h_cnt;
    if (prof) {
        cudaEventElapsedTime(&t->stage[3], t->ev[3], t->ev[6]);
        cudaEventElapsedTime(&t->stage[4], t->ev[3], t->ev[4]);
        cudaEventElapsedTime(&t->stage[5], t->ev[4], t->ev[5]);
        cudaEventElapsedTime(&t->stage[6], t->ev[5], t->ev[6]);
    }
    t->n_pairs = c.n_pairs;
    t->n_vf = c.n_vf;
    t->n_ee = c.n_ee;
    t->n_hits = c.n_hits;
    t->n_disc = c.n_discrete;
    t->n_fp64 = c.n_fp64[0] + c.n_fp64[1];
    t->n_bound_toi = c.n_bound_toi;
    // kErrAccdIters only notes that some stencil ran ACCD's full 1000
    // iterations (the reference then reports a hit too); it is not a failure.
    const unsigned fatal = c.err & ~kErrAccdIters;
    if (fatal) {
        if (t->s_copy) cudaStreamSynchronize(t->s_copy);
        t->traversed = false;
        return device_errors(t, fatal);
    }
    if (out) {
        if (int rc = deliver_out(t, *out)) return rc;
    }
    return MCLCCD_OK;
}

int mclccd_traverse_out(mclccd_tree *t, const double *V0, const double *V1, int nv, const int *P, int mem_kind,
                        int *out_sten, unsigned char *out_is_vf, double *out_toi, long long hit_capacity,
                        long long *n_hits, int *out_discrete, long long disc_capacity, long long *n_discrete,
                        int out_mem_kind)
{
    if (!t) return MCLCCD_ERR_INVALID;
    if (out_mem_kind != MCLCCD_MEM_HOST && out_mem_kind != MCLCCD_MEM_DEVICE)
        return fail(t, MCLCCD_ERR_INVALID, "bad output mem_kind");
    if (hit_capacity < 0 || disc_capacity < 0) return fail(t, MCLCCD_ERR_INVALID, "negative capacity");
    HostOut out{out_sten, out_is_vf, out_toi, hit_capacity, out_discrete, disc_capacity, out_mem_kind};
    t->out_done = 0;
    const int rc = traverse_impl(t, V0, V1, nv, P, mem_kind, &out);
    if (n_hits) *n_hits = rc == MCLCCD_OK ? (long long)t->n_hits : 0;
    if (n_discrete) *n_discrete = rc == MCLCCD_OK ? (long long)t->n_disc : 0;
    return rc;
}

int mclccd_counts(const mclccd_tree *t, long long *n_hits, long long *n_discrete, long long *n_vf, long long *n_ee,
                  long long *n_leaf_pairs)
{
    if (!t) return MCLCCD_ERR_INVALID;
    if (!t->traversed) return MCLCCD_ERR_STATE;
    if (n_hits) *n_hits = (long long)t->n_hits;
    if (n_discrete) *n_discrete = (long long)t->n_disc;
    if (n_vf) *n_vf = (long long)t->n_vf;
    if (n_ee) *n_ee = (long long)t->n_ee;
    if (n_leaf_pairs) *n_leaf_pairs = (long long)t->n_pairs;
    return MCLCCD_OK;
}

static int copy_out(mclccd_tree *t, void *dst, const void *src, size_t bytes, int mem_kind)
{
    if (!dst || bytes == 0) return MCLCCD_OK;
    cudaMemcpyKind k = mem_kind == MCLCCD_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    MC_CUDA(t, cudaMemcpyAsync(dst, src, bytes, k, t->stream));
    return MCLCCD_OK;
}

int mclccd_get_hits(mclccd_tree *t, int mem_kind, long long capacity, int *sten, unsigned char *is_vf, double *toi)
{
    if (!t) return MCLCCD_ERR_INVALID;
    if (!t->traversed) return fail(t, MCLCCD_ERR_STATE, "no traverse results");
    if (capacity < 0 || (mem_kind != MCLCCD_MEM_HOST && mem_kind != MCLCCD_MEM_DEVICE)) return MCLCCD_ERR_INVALID;
    DeviceGuard g(t->device);
    const size_t n = (size_t)std::min<unsigned long long>(t->n_hits, (unsigned long long)capacity);
    if (int rc = copy_out(t, sten, t->hit_sten.p, sizeof(int4) * n, mem_kind)) return rc;
    if (int rc = copy_out(t, is_vf, t->hit_isvf.p, n, mem_kind)) return rc;
    if (int rc = copy_out(t, toi, t->hit_toi.p, sizeof(double) * n, mem_kind)) return rc;
    MC_CUDA(t, cudaStreamSynchronize(t->stream));
    return n < t->n_hits ? MCLCCD_ERR_OVERFLOW : MCLCCD_OK;
}

int mclccd_get_discrete(mclccd_tree *t, int mem_kind, long long capacity, int *pairs)
{
    if (!t) return MCLCCD_ERR_INVALID;
    if (!t->traversed) return fail(t, MCLCCD_ERR_STATE, "no traverse results");
    if (capacity < 0 || (mem_kind != MCLCCD_MEM_HOST && mem_kind != MCLCCD_MEM_DEVICE)) return MCLCCD_ERR_INVALID;
    DeviceGuard g(t->device);
    const size_t n = (size_t)std::min<unsigned long long>(t->n_disc, (unsigned long long)capacity);
    if (int rc = copy_out(t, pairs, t->disc.p, sizeof(int2) * n, mem_kind)) return rc;
    MC_CUDA(t, cudaStreamSynchronize(t->stream));
    return n < t->n_disc ? MCLCCD_ERR_OVERFLOW : MCLCCD_OK;
}

int mclccd_get_candidates(mclccd_tree *t, int mem_kind, long long capacity, int *sten, unsigned char *is_vf)
{
    if (!t) return MCLCCD_ERR_INVALID;
    if (!t->traversed) return fail(t, MCLCCD_ERR_STATE, "no traverse results");
    if (capacity < 0 || (mem_kind != MCLCCD_MEM_HOST && mem_kind != MCLCCD_MEM_DEVICE)) return MCLCCD_ERR_INVALID;
    DeviceGuard g(t->device);
    if (t->cand_lazy && !t->cand_ready && sten) {
        // The fused narrow phase only counted the candidates: expand the leaf
        // pairs of the last traverse again (same kernel, same P and flags),
        // into lists sized by those counts.
        t->cap_vf = std::max<unsigned long long>(t->cap_vf, t->n_vf);
        t->cap_ee = std::max<unsigned long long>(t->cap_ee, t->n_ee);
        MC_CUDA(t, ensure(t->vf, sizeof(int4) * t->cap_vf));
        MC_CUDA(t, ensure(t->ee, sizeof(int4) * t->cap_ee));
        MC_CUDA(t, ensure(t->cand_cnt, sizeof(Counters)));
        Counters *cc = as<Counters>(t->cand_cnt);
        MC_CUDA(t, cudaMemsetAsync(cc, 0, sizeof(Counters), t->stream));
        launch_expand_pairs(t->dim, as<int2>(t->pairs), t->cap_pairs, t->tr_P, as<unsigned char>(t->pflags), t->tr_V1,
                            t->tr_nv, as<int4>(t->vf), t->cap_vf, as<int4>(t->ee), t->cap_ee, nullptr, 0, 1, 0, cc,
                            t->tune[MCLCCD_TUNE_EXPAND_GRID], t->stream, nullptr,
                            &as<Counters>(t->counters)->n_pairs);
        ++t->launches;
        if (int rc = check_launch(t, "candidate expansion")) return rc;
        t->cand_ready = true;
    }
    const unsigned long long total = t->n_vf + t->n_ee;
    const size_t nvf = (size_t)std::min<unsigned long long>(t->n_vf, (unsigned long long)capacity);
    const size_t nee = (size_t)std::min<unsigned long long>(t->n_ee, (unsigned long long)capacity - nvf);
    if (int rc = copy_out(t, sten, t->vf.p, sizeof(int4) * nvf, mem_kind)) return rc;
    if (sten) if (int rc = copy_out(t, sten + 4 * nvf, t->ee.p, sizeof(int4) * nee, mem_kind)) return rc;
    if (is_vf) {
        if (mem_kind == MCLCCD_MEM_HOST) {
            std::memset(is_vf, 1, nvf);
            std::memset(is_vf + nvf, 0, nee);
        } else {
            MC_CUDA(t, cudaMemsetAsync(is_vf, 1, nvf, t->stream));
            MC_CUDA(t, cudaMemsetAsync(is_vf + nvf, 0, nee, t->stream));
        }
    }
    MC_CUDA(t, cudaStreamSynchronize(t->stream));
    return nvf + nee < total ? MCLCCD_ERR_OVERFLOW : MCLCCD_OK;
}

int mclccd_get_leaves(mclccd_tree *t, double *boxes, unsigned char *flags)
{
    if (!t) return MCLCCD_ERR_INVALID;
    if (!t->built) return fail(t, MCLCCD_ERR_STATE, "no update");
    DeviceGuard g(t->device);
    const int np = t->np, dim = t->dim;
    if (np == 0) return MCLCCD_OK;
    std::vector<double> lb((size_t)np * 4 * dim);
    std::vector<int> sorted(np);
    std::vector<unsigned char> act(np), fl(np);
    MC_CUDA(t, cudaMemcpyAsync(lb.data(), t->leaf_box.p, lb.size() * sizeof(double), cudaMemcpyDeviceToHost, t->stream));
    MC_CUDA(t, cudaMemcpyAsync(sorted.data(), t->vals.p, sizeof(int) * np, cudaMemcpyDeviceToHost, t->stream));
    MC_CUDA(t, cudaMemcpyAsync(act.data(), t->leaf_active.p, np, cudaMemcpyDeviceToHost, t->stream));
    MC_CUDA(t, cudaMemcpyAsync(fl.data(), t->pflags.p, np, cudaMemcpyDeviceToHost, t->stream));
    MC_CUDA(t, cudaStreamSynchronize(t->stream));
    for (int k = 0; k < np; ++k) {
        const int prim = sorted[k];
        const double *s = &lb[(size_t)k * 4 * dim];   // lo0, hi0, lo1, hi1
        if (boxes) {
            double *b = boxes + (size_t)prim * 6 * dim;
            for (int c = 0; c < dim; ++c) {
                const double lo0 = s[c], hi0 = s[dim + c], lo1 = s[2 * dim + c], hi1 = s[3 * dim + c];
                b[c] = lo0 < lo1 ? lo0 : lo1;
                b[dim + c] = hi0 < hi1 ? hi1 : hi0;
                b[2 * dim + c] = lo0;
                b[3 * dim + c] = hi0;
                b[4 * dim + c] = lo1;
                b[5 * dim + c] = hi1;
            }
        }
        if (flags) flags[prim] = (unsigned char)((fl[prim] & kFlagAllRep) | (act[k] ? kFlagActive : 0));
    }
    return MCLCCD_OK;
}

int mclccd_narrow_phase_bulk(int dim, const double *V0, const double *V1, int nv, const int *sten,
                             const unsigned char *is_vf, long long n, double vf_eta, double ee_eta, double *out_toi,
                             int *out_hit, int mem_kind, void *stream)
{
    return mclccd_narrow_phase_bulk_ex(dim, V0, V1, nv, sten, is_vf, n, vf_eta, ee_eta, out_toi, out_hit, mem_kind,
                                       stream, MCLCCD_PREC_FP64, nullptr);
}

int mclccd_narrow_phase_bulk_ex(int dim, const double *V0, const double *V1, int nv, const int *sten,
                                const unsigned char *is_vf, long long n, double vf_eta, double ee_eta, double *out_toi,
                                int *out_hit, int mem_kind, void *stream, int precision, long long *n_fp64)
{
    if (n_fp64) *n_fp64 = 0;
    const bool one_sided = (precision & MCLCCD_BULK_VF_ONE_SIDED) != 0;
    precision &= ~MCLCCD_BULK_VF_ONE_SIDED;
    if (precision != MCLCCD_PREC_FP64 && precision != MCLCCD_PREC_FP32_CERTIFIED) return MCLCCD_ERR_INVALID;
    if (one_sided && precision != MCLCCD_PREC_FP64) return MCLCCD_ERR_UNSUPPORTED;
    if ((dim != 2 && dim != 3) || n < 0 || nv < 0) return MCLCCD_ERR_INVALID;
    if (mem_kind != MCLCCD_MEM_HOST && mem_kind != MCLCCD_MEM_DEVICE) return MCLCCD_ERR_INVALID;
    if (!(vf_eta >= 0) || !(ee_eta >= 0)) return MCLCCD_ERR_INVALID;
    if (n == 0) return MCLCCD_OK;
    if (!V0 || !V1 || !sten || !is_vf || !out_toi || !out_hit || nv == 0) return MCLCCD_ERR_INVALID;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t vbytes = sizeof(double) * (size_t)nv * dim;
    // Scratch: the device error word, plus device copies of host arrays.
    char *scratch = nullptr;
    // FP32-certified: plus the queue of stencils for the FP64 pass.
    size_t off_cnt = 0, off_q = 256, off_v0 = 256, off_v1 = 0, off_s = 0, off_f = 0, off_t = 0, off_h = 0, total = 256;
    auto align = [](size_t x) { return (x + 255) & ~(size_t)255; };
    if (precision == MCLCCD_PREC_FP32_CERTIFIED) total = off_v0 = off_q + align(sizeof(long long) * (size_t)n);
    if (mem_kind == MCLCCD_MEM_HOST) {
        off_v1 = off_v0 + align(vbytes);
        off_s = off_v1 + align(vbytes);
        off_f = off_s + align(sizeof(int) * 4 * (size_t)n);
        off_t = off_f + align((size_t)n);
        off_h = off_t + align(sizeof(double) * (size_t)n);
        total = off_h + align(sizeof(int) * (size_t)n);
    }
    cudaError_t e = cudaMallocAsync(reinterpret_cast<void **>(&scratch), total, st);
    if (e != cudaSuccess) { cudaGetLastError(); return e == cudaErrorMemoryAllocation ? MCLCCD_ERR_NOMEM : MCLCCD_ERR_CUDA; }
    Counters *cnt = reinterpret_cast<Counters *>(scratch + off_cnt);
    const double *dV0 = V0, *dV1 = V1;
    const int *ds = sten;
    const unsigned char *df = is_vf;
    double *dt = out_toi;
    int *dh = out_hit;
    int rc = MCLCCD_OK;
    e = cudaMemsetAsync(cnt, 0, sizeof(Counters), st);
    if (e == cudaSuccess && mem_kind == MCLCCD_MEM_HOST) {
        dV0 = reinterpret_cast<const double *>(scratch + off_v0);
        dV1 = reinterpret_cast<const double *>(scratch + off_v1);
        ds = reinterpret_cast<const int *>(scratch + off_s);
        df = reinterpret_cast<const unsigned char *>(scratch + off_f);
        dt = reinterpret_cast<double *>(scratch + off_t);
        dh = reinterpret_cast<int *>(scratch + off_h);
        e = cudaMemcpyAsync((void *)dV0, V0, vbytes, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync((void *)dV1, V1, vbytes, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync((void *)ds, sten, sizeof(int) * 4 * (size_t)n, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync((void *)df, is_vf, (size_t)n, cudaMemcpyHostToDevice, st);
    }
    if (e == cudaSuccess) {
        if (precision == MCLCCD_PREC_FP32_CERTIFIED)
            launch_accd_certified_bulk(dim, ds, df, n, dV0, dV1, nv, vf_eta, ee_eta, dt, dh,
                                       reinterpret_cast<long long *>(scratch + off_q), cnt, st);
        else
            launch_accd_bulk(dim, ds, df, n, dV0, dV1, nv, vf_eta, ee_eta, dt, dh, cnt, st, one_sided);
        e = cudaGetLastError();
    }
    Counters h{};
    if (e == cudaSuccess && mem_kind == MCLCCD_MEM_HOST) {
        e = cudaMemcpyAsync(out_toi, dt, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(out_hit, dh, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, st);
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, cnt, sizeof(Counters), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFreeAsync(scratch, st);
    if (e != cudaSuccess) rc = MCLCCD_ERR_CUDA;
    else if (h.err & kErrBadIndex) rc = MCLCCD_ERR_INVALID;
    if (n_fp64) *n_fp64 = (long long)(h.n_fp64[0] + h.n_fp64[1]);
    return rc;
}

int mclccd_vjp_toi(int dim, const double *V0, const double *V1, int nv, const int *sten, const unsigned char *is_vf,
                   const double *toi, const double *g_toi, long long n, double vf_eta, double ee_eta, double *dV0,
                   double *dV1, double *t_star, int *status, double *jac_rows, long long *n_ok, int mem_kind,
                   void *stream)
{
    if (n_ok) *n_ok = 0;
    if ((dim != 2 && dim != 3) || n < 0 || nv < 0) return MCLCCD_ERR_INVALID;
    if (mem_kind != MCLCCD_MEM_HOST && mem_kind != MCLCCD_MEM_DEVICE) return MCLCCD_ERR_INVALID;
    if (!(vf_eta >= 0) || !(ee_eta >= 0)) return MCLCCD_ERR_INVALID;
    if ((dV0 != nullptr) != (dV1 != nullptr)) return MCLCCD_ERR_INVALID;
    if (dV0 && !g_toi) return MCLCCD_ERR_INVALID;
    if (n > 0 && (!V0 || !V1 || !sten || !is_vf || !toi || nv == 0)) return MCLCCD_ERR_INVALID;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t vbytes = sizeof(double) * (size_t)nv * dim, un = (size_t)n;
    const size_t rbytes = sizeof(double) * un * 2 * (dim + 1) * dim;
    auto align = [](size_t x) { return (x + 255) & ~(size_t)255; };
    // Scratch: the counter, plus device copies of host arrays.
    size_t off[11] = {0};
    const size_t sizes[11] = {sizeof(unsigned long long), vbytes, vbytes, sizeof(int) * 4 * un, un,
                              sizeof(double) * un, g_toi ? sizeof(double) * un : 0, dV0 ? vbytes : 0,
                              dV0 ? vbytes : 0, t_star ? sizeof(double) * un : 0, status ? sizeof(int) * un : 0};
    const bool host = mem_kind == MCLCCD_MEM_HOST;
    size_t total = 0;
    for (int i = 0; i < 11; ++i) {
        off[i] = total;
        if (i == 0 || host) total += align(sizes[i]);
    }
    size_t off_rows = total;
    if (host && jac_rows) total += align(rbytes);
    char *scratch = nullptr;
    cudaError_t e = cudaMallocAsync(reinterpret_cast<void **>(&scratch), total, st);
    if (e != cudaSuccess) { cudaGetLastError(); return e == cudaErrorMemoryAllocation ? MCLCCD_ERR_NOMEM : MCLCCD_ERR_CUDA; }
    auto dev = [&](int i, const void *p) -> void * { return host ? (p ? scratch + off[i] : nullptr) : const_cast<void *>(p); };
    unsigned long long *cnt = reinterpret_cast<unsigned long long *>(scratch);
    const double *dv0 = (const double *)dev(1, V0), *dv1 = (const double *)dev(2, V1);
    const int *ds = (const int *)dev(3, sten);
    const unsigned char *df = (const unsigned char *)dev(4, is_vf);
    const double *dt = (const double *)dev(5, toi), *dg = (const double *)dev(6, g_toi);
    double *gV0 = (double *)dev(7, dV0), *gV1 = (double *)dev(8, dV1), *dts = (double *)dev(9, t_star);
    int *dst = (int *)dev(10, status);
    double *drows = host ? (jac_rows ? reinterpret_cast<double *>(scratch + off_rows) : nullptr) : jac_rows;
    e = cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), st);
    if (host) {
        const void *src[7] = {nullptr, V0, V1, sten, is_vf, toi, g_toi};
        for (int i = 1; i < 7 && e == cudaSuccess; ++i)
            if (src[i] && sizes[i]) e = cudaMemcpyAsync(scratch + off[i], src[i], sizes[i], cudaMemcpyHostToDevice, st);
    }
    if (e == cudaSuccess && gV0) e = cudaMemsetAsync(gV0, 0, vbytes, st);
    if (e == cudaSuccess && gV1) e = cudaMemsetAsync(gV1, 0, vbytes, st);
    if (e == cudaSuccess) {
        launch_vjp_toi(dim, ds, df, dt, dg, n, dv0, dv1, nv, vf_eta, ee_eta, gV0, gV1, dts, dst, drows, cnt, st);
        e = cudaGetLastError();
    }
    unsigned long long h_ok = 0;
    if (host && e == cudaSuccess) {
        if (dV0) e = cudaMemcpyAsync(dV0, gV0, vbytes, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess && dV1) e = cudaMemcpyAsync(dV1, gV1, vbytes, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess && t_star && n) e = cudaMemcpyAsync(t_star, dts, sizeof(double) * un, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess && status && n) e = cudaMemcpyAsync(status, dst, sizeof(int) * un, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess && jac_rows && n) e = cudaMemcpyAsync(jac_rows, drows, rbytes, cudaMemcpyDeviceToHost, st);
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h_ok, cnt, sizeof(h_ok), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFreeAsync(scratch, st);
    if (e != cudaSuccess) return MCLCCD_ERR_CUDA;
    if (n_ok) *n_ok = (long long)h_ok;
    return MCLCCD_OK;
}

int mclccd_tree_vjp_toi(mclccd_tree *t, const double *g_toi, double *dV0, double *dV1, long long *n_ok, int mem_kind)
{
    if (!t) return MCLCCD_ERR_INVALID;
    if (!t->traversed) return fail(t, MCLCCD_ERR_STATE, "no traverse results");
    if (t->n_hits > t->cap_hits) return fail(t, MCLCCD_ERR_STATE, "hit buffer overflowed");
    if (t->n_hits > 0 && !t->tr_V0) return fail(t, MCLCCD_ERR_STATE, "no traverse geometry");
    DeviceGuard g(t->device);
    const int dim = t->dim;
    const long long n = (long long)t->n_hits;
    // Device-side stencils of the hits; V0/V1 are the traverse's device arrays.
    const int *sten = as<int>(t->hit_sten);
    const unsigned char *is_vf = as<unsigned char>(t->hit_isvf);
    const double *toi = as<double>(t->hit_toi);
    if (mem_kind == MCLCCD_MEM_DEVICE)
        return mclccd_vjp_toi(dim, t->tr_V0, t->tr_V1, t->tr_nv, sten, is_vf, toi, g_toi, n, t->vf_eta, t->ee_eta, dV0,
                              dV1, nullptr, nullptr, nullptr, n_ok, MCLCCD_MEM_DEVICE, t->stream);
    if (mem_kind != MCLCCD_MEM_HOST) return MCLCCD_ERR_INVALID;
    // Host g / dV: stage through device scratch.
    const size_t vbytes = sizeof(double) * (size_t)t->tr_nv * dim;
    double *dg = nullptr, *d0 = nullptr, *d1 = nullptr;
    cudaStream_t st = t->stream;
    cudaError_t e = cudaMallocAsync(reinterpret_cast<void **>(&dg), sizeof(double) * (size_t)std::max<long long>(n, 1), st);
    if (e == cudaSuccess) e = cudaMallocAsync(reinterpret_cast<void **>(&d0), std::max<size_t>(vbytes, 8), st);
    if (e == cudaSuccess) e = cudaMallocAsync(reinterpret_cast<void **>(&d1), std::max<size_t>(vbytes, 8), st);
    if (e == cudaSuccess && g_toi && n) e = cudaMemcpyAsync(dg, g_toi, sizeof(double) * (size_t)n, cudaMemcpyHostToDevice, st);
    int rc = e == cudaSuccess ? MCLCCD_OK : MCLCCD_ERR_CUDA;
    if (rc == MCLCCD_OK)
        rc = mclccd_vjp_toi(dim, t->tr_V0, t->tr_V1, t->tr_nv, sten, is_vf, toi, g_toi ? dg : nullptr, n, t->vf_eta,
                            t->ee_eta, dV0 ? d0 : nullptr, dV1 ? d1 : nullptr, nullptr, nullptr, nullptr, n_ok,
                            MCLCCD_MEM_DEVICE, st);
    if (rc == MCLCCD_OK && dV0) rc = cudaMemcpyAsync(dV0, d0, vbytes, cudaMemcpyDeviceToHost, st) ? MCLCCD_ERR_CUDA : rc;
    if (rc == MCLCCD_OK && dV1) rc = cudaMemcpyAsync(dV1, d1, vbytes, cudaMemcpyDeviceToHost, st) ? MCLCCD_ERR_CUDA : rc;
    if (rc == MCLCCD_OK) rc = cudaStreamSynchronize(st) ? MCLCCD_ERR_CUDA : rc;
    if (dg) cudaFreeAsync(dg, st);
    if (d0) cudaFreeAsync(d0, st);
    if (d1) cudaFreeAsync(d1, st);
    if (rc != MCLCCD_OK) fail(t, rc, "vjp_toi failed");
    return rc;
}

int mclccd_precision_stats(const mclccd_tree *t, long long *n_fp64, long long *n_bound_toi)
{
    if (!t) return MCLCCD_ERR_INVALID;
    if (n_fp64) *n_fp64 = (long long)t->n_fp64;
    if (n_bound_toi) *n_bound_toi = (long long)t->n_bound_toi;
    return MCLCCD_OK;
}

int mclccd_get_tree_view(const mclccd_tree *t, mclccd_tree_view *view)
{
    if (!t || !view) return MCLCCD_ERR_INVALID;
    if (!t->built || t->np < 1) return MCLCCD_ERR_STATE;
    view->dim = t->dim;
    view->n_leaves = t->np;
    view->nodes = t->np > 1 ? t->nodes.p : nullptr;
    view->leaf_box = static_cast<const double *>(t->leaf_box.p);
    view->leaf_prim = static_cast<const int *>(t->vals.p);
    return MCLCCD_OK;
}

int mclccd_get_tree_host(mclccd_tree *t, void *nodes, double *leaf_box, int *leaf_prim, unsigned char *leaf_flags)
{
    if (!t) return MCLCCD_ERR_INVALID;
    if (!t->built || t->np < 1) return fail(t, MCLCCD_ERR_STATE, "no tree: update first");
    DeviceGuard g(t->device);
    const int np = t->np, dim = t->dim;
    cudaStream_t st = t->stream;
    if (nodes && np > 1)
        MC_CUDA(t, cudaMemcpyAsync(nodes, t->nodes.p, sizeof(Node) * (size_t)(np - 1), cudaMemcpyDeviceToHost, st));
    if (leaf_box)
        MC_CUDA(t, cudaMemcpyAsync(leaf_box, t->leaf_box.p, sizeof(double) * 4 * dim * (size_t)np,
                                   cudaMemcpyDeviceToHost, st));
    std::vector<int> sorted;
    int *prim = leaf_prim;
    if (!prim && leaf_flags) {
        sorted.resize(np);
        prim = sorted.data();
    }
    if (prim) MC_CUDA(t, cudaMemcpyAsync(prim, t->vals.p, sizeof(int) * (size_t)np, cudaMemcpyDeviceToHost, st));
    std::vector<unsigned char> act, fl;
    if (leaf_flags) {
        act.resize(np);
        fl.resize(np);
        MC_CUDA(t, cudaMemcpyAsync(act.data(), t->leaf_active.p, np, cudaMemcpyDeviceToHost, st));
        MC_CUDA(t, cudaMemcpyAsync(fl.data(), t->pflags.p, np, cudaMemcpyDeviceToHost, st));
    }
    MC_CUDA(t, cudaStreamSynchronize(st));
    if (leaf_flags)
        for (int k = 0; k < np; ++k)
            leaf_flags[k] = (unsigned char)((fl[prim[k]] & kFlagAllRep) | (act[k] ? kFlagActive : 0));
    return MCLCCD_OK;
}

int mclccd_build_stats(const mclccd_tree *t, long long *builds, long long *quality_rebuilds)
{
    if (!t) return MCLCCD_ERR_INVALID;
    if (builds) *builds = t->n_builds;
    if (quality_rebuilds) *quality_rebuilds = t->n_quality_rebuilds;
    return MCLCCD_OK;
}

int mclccd_tree_size(const mclccd_tree *t, int *nv, int *np, int *pdim)
{
    if (!t) return MCLCCD_ERR_INVALID;
    if (!t->built) return MCLCCD_ERR_STATE;
    if (nv) *nv = t->nv;
    if (np) *np = t->np;
    if (pdim) *pdim = t->pdim;
    return MCLCCD_OK;
}

int mclccd_host_alloc(size_t bytes, void **ptr)
{
    if (!ptr) return MCLCCD_ERR_INVALID;
    *ptr = nullptr;
    if (bytes == 0) return MCLCCD_OK;
    const cudaError_t e = cudaHostAlloc(ptr, bytes, cudaHostAllocPortable);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *ptr = nullptr;
        return e == cudaErrorMemoryAllocation ? MCLCCD_ERR_NOMEM : MCLCCD_ERR_CUDA;
    }
    return MCLCCD_OK;
}

int mclccd_host_free(void *ptr)
{
    if (ptr && cudaFreeHost(ptr) != cudaSuccess) {
        cudaGetLastError();
        return MCLCCD_ERR_CUDA;
    }
    return MCLCCD_OK;
}

int mclccd_stage_ms(const mclccd_tree *t, float *ms, int n)
{
    if (!t || !ms || n < 0) return -1;
    int k = std::min(n, 7);
    for (int i = 0; i < k; ++i) ms[i] = t->stage[i];
    return k;
}

int mclccd_set_tuning(mclccd_tree *t, int key, int value)
{
    if (!t || key < 0 || key >= MCLCCD_TUNE_COUNT) return MCLCCD_ERR_INVALID;
    const bool flag = key == MCLCCD_TUNE_WALK_PACKET || key == MCLCCD_TUNE_NARROW_FUSED ||
                      key == MCLCCD_TUNE_WALK_REFILL;
    if (key == MCLCCD_TUNE_WALK_BUFFER) {
        if (value < 0 || value > 2) return fail(t, MCLCCD_ERR_INVALID, "walk buffer must be 0, 1 or 2");
    } else if (key == MCLCCD_TUNE_EXPAND_SPLIT) {
        if (value < 0 || value > 2) return fail(t, MCLCCD_ERR_INVALID, "expansion split must be 0, 1 or 2");
    } else if (key == MCLCCD_TUNE_REBUILD_RATIO) {
        if (value != 0 && (value < 101 || value > 100000))
            return fail(t, MCLCCD_ERR_INVALID, "rebuild ratio is 0 (never) or a percentage above 100");
    } else if (key == MCLCCD_TUNE_ACCD_REBIN) {
        if (value < 0 || value > 2) return fail(t, MCLCCD_ERR_INVALID, "ACCD form must be 0, 1 or 2");
    } else if (key == MCLCCD_TUNE_OVERLAP) {
        if (value < 0 || value > 16) return fail(t, MCLCCD_ERR_INVALID, "overlap chunks must be in [0, 16]");
    } else if (key == MCLCCD_TUNE_WALK_WINDOW) {
        if (value != 0 && value != 8 && value != 16 && value != 32 && value != 64 && value != 128)
            return fail(t, MCLCCD_ERR_INVALID, "walk window must be 0, 8, 16, 32, 64 or 128");
        if (t->tune[MCLCCD_TUNE_WALK_REFILL] && (value == 0 || value > 32))
            return fail(t, MCLCCD_ERR_INVALID, "the refill walk takes a window of 8, 16 or 32");
    } else if (key == MCLCCD_TUNE_WALK_REFILL && value == 1 &&
               (t->tune[MCLCCD_TUNE_WALK_WINDOW] == 0 || t->tune[MCLCCD_TUNE_WALK_WINDOW] > 32)) {
        return fail(t, MCLCCD_ERR_INVALID, "the refill walk takes a window of 8, 16 or 32");
    } else if (flag ? (value != 0 && value != 1) : (value < 1 || value > (1 << 20)))
        return fail(t, MCLCCD_ERR_INVALID, "tuning value out of range");
    t->tune[key] = value;
    return MCLCCD_OK;
}

int mclccd_get_tuning(const mclccd_tree *t, int key, int *value)
{
    if (!t || !value || key < 0 || key >= MCLCCD_TUNE_COUNT) return MCLCCD_ERR_INVALID;
    *value = t->tune[key];
    return MCLCCD_OK;
}

int mclccd_kernel_launches(const mclccd_tree *t, long long *n)
{
    if (!t || !n) return MCLCCD_ERR_INVALID;
    *n = t->launches;
    return MCLCCD_OK;
}

} // extern "C"
