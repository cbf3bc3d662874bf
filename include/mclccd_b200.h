/*
 * mclccd_b200 -- C ABI of the B200 continuous-collision-detection path.
 *
 * Drop-in for the hot path of mattoverby/mclccd's mcl::BVHTree<double,DIM>
 * (include/MCL/BVHTree.hpp): update(V0,V1,P) builds the hierarchy over swept
 * primitive boxes, traverse(V0,V1,P) finds every candidate vertex-face /
 * edge-edge stencil, runs the ACCD narrow phase and the discrete test, and
 * leaves the results (what the reference hands to append_pair and
 * append_discrete) in device buffers that the get_* calls copy out.
 *
 * Conventions
 *   - Positions are float64, row-major nv x dim; primitives int32, row-major
 *     np x pdim (triangles in 3D, edges in 2D).
 *   - mem_kind says where the caller's arrays live (MCLCCD_MEM_HOST or
 *     MCLCCD_MEM_DEVICE, device = the current CUDA device's global memory).
 *   - Every call returns a status (MCLCCD_OK == 0).  The reference has no
 *     error codes (asserts and silent early returns); here bad input is an
 *     error instead of undefined behaviour.
 *   - A handle is not thread-safe; all its work is ordered on its stream.
 *   - Stencils are int32[4]: VF = [v, f0, f1, f2] (2D: [v, e0, e1, -1]),
 *     EE = [a, b, c, d] (edge a-b of the lower-indexed triangle first).
 *     Discrete pairs are (p0, p1) with p0 < p1.
 */
#ifndef MCLCCD_B200_H
#define MCLCCD_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mclccd_tree mclccd_tree;

/* Status codes. */
#define MCLCCD_OK 0
#define MCLCCD_ERR_INVALID 1     /* bad argument or primitive index out of [0, nv) */
#define MCLCCD_ERR_CUDA 2        /* a CUDA runtime call failed */
#define MCLCCD_ERR_NOMEM 3       /* device allocation failed */
#define MCLCCD_ERR_OVERFLOW 4    /* caller's output capacity too small (copied a prefix) */
#define MCLCCD_ERR_STATE 5       /* traverse before update, or results before traverse */
#define MCLCCD_ERR_DEVICE 6      /* a kernel gave up a bounded wait or overflowed its stack */
#define MCLCCD_ERR_UNSUPPORTED 7 /* option combination not provided (bulk: one-sided VF with the certified form) */
#define MCLCCD_ERR_SCRATCH_LIMIT 8 /* mclccd_narrow_phase_bulk_static: arrays exceed its fixed scratch */

/* Where caller arrays live. */
#define MCLCCD_MEM_HOST 0
#define MCLCCD_MEM_DEVICE 1

/* Option flags: the booleans of BVHTree::Options (BVHTree.hpp:42-64). */
#define MCLCCD_OPT_REPTRI (1u << 0)
#define MCLCCD_OPT_THREADED (1u << 1)     /* accepted; the device path is always parallel */
#define MCLCCD_OPT_DISCRETE (1u << 2)
#define MCLCCD_OPT_CONTINUOUS (1u << 3)
#define MCLCCD_OPT_VF_ONE_SIDED (1u << 4) /* VF narrow phase: CTCD with the wrong-side test (NarrowPhase.cpp:338-425) */
#define MCLCCD_OPT_EE_ROBUST (1u << 5)    /* accepted; unused by ACCD, as in the reference */
#define MCLCCD_OPT_DEFAULT (MCLCCD_OPT_REPTRI | MCLCCD_OPT_THREADED | MCLCCD_OPT_DISCRETE | \
                            MCLCCD_OPT_CONTINUOUS | MCLCCD_OPT_EE_ROBUST)
/* Extra behaviour flags (not in the reference). */
#define MCLCCD_OPT_ALWAYS_REBUILD (1u << 8) /* never take the refit-only path */
#define MCLCCD_OPT_PROFILE (1u << 9)        /* record per-stage CUDA-event times */

/* Narrow-phase precision. */
#define MCLCCD_PREC_FP64 0
#define MCLCCD_PREC_FP32_CERTIFIED 1

/* Replaces: BVHTree<double,DIM>::BVHTree() (BVHTree.cpp:20-24).  dim is 2 or
 * 3; the tree lives on the current CUDA device and gets its own stream.
 * Options start at the reference defaults (BVHTree.hpp:52-62). */
int mclccd_create(int dim, mclccd_tree **out);

/* Replaces: ~BVHTree().  Frees every device buffer the handle owns. */
int mclccd_destroy(mclccd_tree *tree);

/* Full hierarchy builds since creation, and how many of them the tree-
 * quality trigger (MCLCCD_TUNE_REBUILD_RATIO) caused. */
int mclccd_build_stats(const mclccd_tree *tree, long long *builds, long long *quality_rebuilds);

/* Sizes of the last update: vertex count (the derived one when the update
 * passed nv = 0), primitive count and primitive width (any may be NULL). */
int mclccd_tree_size(const mclccd_tree *tree, int *nv, int *np, int *pdim);

/* Replaces: writes to BVHTree::options (BVHTree.hpp:42-64). */
int mclccd_set_options(mclccd_tree *tree, double box_eta, double vf_ccd_eta, double ee_ccd_eta, unsigned flags);
/* Reads them back (update() clamps the two gaps to box_eta, BVHTree.cpp:39-40). */
int mclccd_get_options(const mclccd_tree *tree, double *box_eta, double *vf_ccd_eta, double *ee_ccd_eta,
                       unsigned *flags);

/* Orders all of the handle's work on a caller stream (cudaStream_t; NULL
 * restores the handle's own stream). */
int mclccd_set_stream(mclccd_tree *tree, void *stream);

/* MCLCCD_PREC_FP64 (default; bit-exact with the reference) or
 * MCLCCD_PREC_FP32_CERTIFIED (FP32 filter + FP64 certification). */
int mclccd_set_precision(mclccd_tree *tree, int precision);

/* Replaces: BVHTree::update(const T*V0, const T*V1, const int*P, int np,
 * int pdim, const int*active) (BVHTree.hpp:81-82, BVHTree.cpp:27-126).
 * nv is new: the device needs the vertex count to copy/validate V0, V1;
 * nv = 0 takes it as 1 + the largest index in P, as the reference's
 * signature implies (found on the device, no host pass over P).  active is
 * an optional per-vertex int mask (NULL = all active).  When np, pdim, nv
 * and the bytes of P equal the previous update, only the boxes are
 * refitted; otherwise the hierarchy is rebuilt.  np == 0 clears the tree. */
int mclccd_update(mclccd_tree *tree, const double *V0, const double *V1, int nv, const int *P, int np, int pdim,
                  const int *active, int mem_kind);

/* Replaces: BVHTree::traverse(const T*V0, const T*V1, const int*P) const
 * (BVHTree.hpp:86, BVHTree.cpp:129-159) with the default narrow phase and no
 * filter.  Passing V0 = V1 = P = NULL reuses the arrays of the last update.
 * Results stay on the device until read with mclccd_get_*. */
int mclccd_traverse(mclccd_tree *tree, const double *V0, const double *V1, int nv, const int *P, int mem_kind);

/* traverse and deliver the results into caller buffers in one call, as the
 * reference's traverse hands each hit to append_pair and each discrete pair
 * to append_discrete (BVHTree.cpp:262-281): hits (stencil int32 x 4, is_vf,
 * toi) and discrete pairs (int32 x 2) are written to the out_* arrays on the
 * out_mem_kind side, at most the given capacities (a prefix), in the order
 * of mclccd_get_hits / mclccd_get_discrete; n_hits / n_discrete receive the
 * full counts.  Host outputs are copied in chunks while later chunks of the
 * step compute (page-locked buffers let the copies overlap).  Any out_*
 * pointer may be NULL. */
int mclccd_traverse_out(mclccd_tree *tree, const double *V0, const double *V1, int nv, const int *P, int mem_kind,
                        int *out_sten, unsigned char *out_is_vf, double *out_toi, long long hit_capacity,
                        long long *n_hits, int *out_discrete, long long disc_capacity, long long *n_discrete,
                        int out_mem_kind);

/* Counts from the last traverse: CCD hits (append_pair calls), discrete
 * pairs (append_discrete calls), candidate VF / EE stencils (filter_pair
 * calls) and leaf pairs whose boxes intersect.  Any pointer may be NULL. */
int mclccd_counts(const mclccd_tree *tree, long long *n_hits, long long *n_discrete, long long *n_vf,
                  long long *n_ee, long long *n_leaf_pairs);

/* Copies up to capacity hits: sten int32[4*n], is_vf uint8[n], toi f64[n]
 * (any of them may be NULL).  The arguments of append_pair (BVHTree.hpp:102). */
int mclccd_get_hits(mclccd_tree *tree, int mem_kind, long long capacity, int *sten, unsigned char *is_vf,
                    double *toi);

/* Copies up to capacity discrete pairs int32[2*n], p0 < p1.  The arguments of
 * append_discrete (BVHTree.hpp:108). */
int mclccd_get_discrete(mclccd_tree *tree, int mem_kind, long long capacity, int *pairs);

/* Copies up to capacity candidate stencils (every stencil the reference
 * passes to filter_pair, BVHTree.cpp:345,368,393): VF first, then EE. */
int mclccd_get_candidates(mclccd_tree *tree, int mem_kind, long long capacity, int *sten, unsigned char *is_vf);

/* Leaf data of the last update in primitive order (BVHTree::leaves):
 * boxes f64[np * 6 * dim] as (box.min, box.max, t0.min, t0.max, t1.min,
 * t1.max) and flags uint8[np] (bit j: vertex slot j represented, bit 3+j:
 * edge slot j represented, bit 6: active). */
int mclccd_get_leaves(mclccd_tree *tree, double *boxes, unsigned char *flags);

/* Bulk narrow phase (added entry point): NarrowPhaseACCD::query_ccd_vf/ee
 * (NarrowPhase.cpp:609-631) over n caller stencils.  out_toi[i] = toi on a
 * hit, -1 otherwise; out_hit[i] = 1/0.  stream may be NULL (default stream).
 * All arrays are on the same side (mem_kind). */
int mclccd_narrow_phase_bulk(int dim, const double *V0, const double *V1, int nv, const int *sten,
                             const unsigned char *is_vf, long long n, double vf_ccd_eta, double ee_ccd_eta,
                             double *out_toi, int *out_hit, int mem_kind, void *stream);

/* The bulk narrow phase with a precision: MCLCCD_PREC_FP64 (same as above) or
 * MCLCCD_PREC_FP32_CERTIFIED (identical hit/miss; toi never later than the
 * FP64 value and within 1e-6 relative of it).  n_fp64 (may be NULL) receives
 * how many stencils the certified form had to evaluate in full FP64.
 * MCLCCD_PREC_FP64 | MCLCCD_BULK_VF_ONE_SIDED: VF stencils take the one-sided
 * CTCD narrow phase instead (NarrowPhaseCTCD::query_ccd_vf with the
 * wrong-side test, as BVHTree with vf_one_sided); a hit is a contact on the
 * right side, wrong-side-only contacts are misses.  With the certified form
 * it returns MCLCCD_ERR_UNSUPPORTED. */
#define MCLCCD_BULK_VF_ONE_SIDED 0x100
int mclccd_narrow_phase_bulk_ex(int dim, const double *V0, const double *V1, int nv, const int *sten,
                                const unsigned char *is_vf, long long n, double vf_ccd_eta, double ee_ccd_eta,
                                double *out_toi, int *out_hit, int mem_kind, void *stream, int precision,
                                long long *n_fp64);

/* Stencils of the last traverse that the FP32-certified form handed to its
 * FP64 pass (ACCD undecided by the FP32 brackets), and hits it reported with
 * the certified lower bound on toi (within 1e-6 relative) instead of the
 * bit-identical FP64 value (both 0 in MCLCCD_PREC_FP64 mode).  Either pointer
 * may be NULL. */
int mclccd_precision_stats(const mclccd_tree *tree, long long *n_fp64, long long *n_bound_toi);

/* No counterpart in the reference.  The bulk narrow phase above without any
 * device allocation, for callers that cannot call cudaMalloc: loops on a
 * fixed device-memory budget (cudaMalloc/cudaFree can stall the device and
 * fragment the budget), processes where another allocator already holds the
 * device memory, plugins whose host forbids device allocations.  Same
 * arguments and results as mclccd_narrow_phase_bulk (bit-identical).  Its
 * scratch -- the device status word and, for MCLCCD_MEM_HOST, the device
 * copies of V0, V1, sten, is_vf, out_toi and out_hit, each rounded up to 256
 * bytes -- lives in one fixed device array of MCLCCD_STATIC_SCRATCH_BYTES
 * that every GPU loading the library holds until exit; larger host-memory
 * calls return MCLCCD_ERR_SCRATCH_LIMIT (device-memory calls use only the
 * status word and have no size limit).  The first call on each device looks
 * up the array's device address (cudaGetSymbolAddress); make that first call
 * before any stream capture.  The address is kept for the life of the
 * process, so do not call this entry point after cudaDeviceReset (or any
 * reset of the device's primary context) in the same process.  All calls
 * share the array: calls that overlap on the GPU race on it. */
#define MCLCCD_STATIC_SCRATCH_BYTES (32u << 20)
int mclccd_narrow_phase_bulk_static(int dim, const double *V0, const double *V1, int nv, const int *sten,
                                    const unsigned char *is_vf, long long n, double vf_ccd_eta, double ee_ccd_eta,
                                    double *out_toi, int *out_hit, int mem_kind, void *stream);

/* No counterpart in the reference: the adjoint of the time of impact.
 * For each hit (stencil, is_vf, toi as ACCD reported it) the contact time t*
 * is the first root t >= toi of dist(x(t)) = eta with x(t) = V0 + t (V1 - V0)
 * (true closest points, FP64), refined from toi; its gradient follows from
 * implicit differentiation of that contact condition, recomputing the
 * closest-feature pair at t*.  Outputs (each may be NULL):
 *   dV0, dV1   nv x dim, overwritten with sum_h g_toi[h] d(t*_h)/dV0 (resp. V1)
 *              (the vector-Jacobian product a torch.autograd.Function
 *              backward computes; needs g_toi);
 *   t_star     n contact times;  status  n MCLCCD_VJP_* codes;
 *   jac_rows   n x 2 (dim+1) dim: d(t*)/dV0 of the stencil's dim+1 vertices,
 *              then d(t*)/dV1, slot-major;
 *   n_ok       how many hits had a gradient (status MCLCCD_VJP_OK).
 * A hit whose status is not OK contributes zero.  All arrays on the same side
 * (mem_kind). */
#define MCLCCD_VJP_OK 0
#define MCLCCD_VJP_TOI_ZERO 1   /* toi == 0 (within eta at t = 0): constant */
#define MCLCCD_VJP_NO_CONTACT 2 /* dist stays above eta on [toi, 1] */
#define MCLCCD_VJP_GRAZING 3    /* d/dt dist ~ 0 at t*: not differentiable */
#define MCLCCD_VJP_NO_CONVERGE 4
#define MCLCCD_VJP_BAD_TOI 5    /* toi outside [0, 1], or no root at all */
#define MCLCCD_VJP_BAD_INDEX 6  /* stencil vertex outside [0, nv) */
int mclccd_vjp_toi(int dim, const double *V0, const double *V1, int nv, const int *sten, const unsigned char *is_vf,
                   const double *toi, const double *g_toi, long long n, double vf_ccd_eta, double ee_ccd_eta,
                   double *dV0, double *dV1, double *t_star, int *status, double *jac_rows, long long *n_ok,
                   int mem_kind, void *stream);

/* The same for the hits of the handle's last traverse, in mclccd_get_hits
 * order, with the V0/V1 that traverse used (device copies or the caller's
 * device arrays, which must still be valid) and the handle's etas.  g_toi has
 * one entry per hit; dV0/dV1 are nv x dim; all on the mem_kind side. */
int mclccd_tree_vjp_toi(mclccd_tree *tree, const double *g_toi, double *dV0, double *dV1, long long *n_ok,
                        int mem_kind);

/* No counterpart in the reference: batched CCD of many independent scenes.
 * Each scene is what one BVHTree<double, dim> would process (dim 2: P is an
 * edge list, dim 3: triangles), with box_eta = vf_ccd_eta = ee_ccd_eta =
 * eta[s] and the default options.  One mclccd_batch_run builds a segmented
 * LBVH over all scenes, then traverses and scores them in one of two forms
 * (MCLCCD_BATCH_TUNE_FORM below), as a CUDA graph (captured on the first run
 * after the scenes, precision or tuning change, replayed afterwards).  In
 * the waves form a wave that overflows its buffers is redone smaller inside
 * the graph.  Results are
 * per-scene reductions rather than hit lists:
 *   n_hits, n_discrete, n_stencils  hits, discrete pairs and candidate
 *                                   stencils (VF + EE) of the scene;
 *   min_toi, min_sten, min_is_vf    earliest toi and its stencil (scene-local
 *                                   vertex ids; ties go to VF before EE, then
 *                                   the smallest ids), -1 when no hit;
 *   done_ms                         when the scene's last work finished,
 *                                   from the start of the run (device clock);
 *   batch_ms                        device time of the whole run.
 * V0/V1/P are the scenes' arrays concatenated in scene order (each scene's
 * own dim per row); P holds scene-local vertex ids. */
typedef struct mclccd_batch mclccd_batch;
#define MCLCCD_BATCH_TUNE_BLOCK 0   /* threads per block of the tree walk / persistent kernel: 128 or 256 */
#define MCLCCD_BATCH_TUNE_STACK 1   /* traversal stack entries per thread: 32 or 64 */
#define MCLCCD_BATCH_TUNE_CHUNK 2   /* persistent form: queries per lane a warp takes from the work queue: 1..64 */
#define MCLCCD_BATCH_TUNE_LEAF 3    /* subtrees of up to this many leaves are scanned, not descended: 1..16 */
#define MCLCCD_BATCH_TUNE_FORM 4    /* MCLCCD_BATCH_FORM_WAVES (default) or MCLCCD_BATCH_FORM_PERSISTENT */
#define MCLCCD_BATCH_TUNE_WAVE 5    /* waves form: wave buffer, in 2^16 leaf pairs (stencil buffers 2x VF, 4x EE): 1..4096 */
#define MCLCCD_BATCH_TUNE_COUNT 6
/* Forms of the batched step.  WAVES: per group, a device-driven loop of
 * waves (walk -> stencil expansion -> ACCD -> per-scene reductions) in a
 * conditional graph node.  PERSISTENT: per group, one persistent
 * traversal-plus-narrow-phase kernel whose warps take query chunks from a
 * global work queue.  Results are identical. */
#define MCLCCD_BATCH_FORM_WAVES 0
#define MCLCCD_BATCH_FORM_PERSISTENT 1
int mclccd_batch_create(mclccd_batch **out);
int mclccd_batch_destroy(mclccd_batch *batch);
int mclccd_batch_set_scenes(mclccd_batch *batch, int n_scenes, const int *scene_dim, const int *scene_nv,
                            const int *scene_np, const double *V0, const double *V1, const int *P, const double *eta,
                            int mem_kind);
int mclccd_batch_set_positions(mclccd_batch *batch, const double *V0, const double *V1, int mem_kind);
int mclccd_batch_set_precision(mclccd_batch *batch, int precision);
int mclccd_batch_set_tuning(mclccd_batch *batch, int key, int value);
int mclccd_batch_get_tuning(const mclccd_batch *batch, int key, int *value);
/* Waves form: waves completed and waves redone smaller (buffer overflow) in
 * the last run, summed over the 2D and 3D groups; 0, 0 in the persistent form. */
int mclccd_batch_wave_stats(mclccd_batch *batch, long long *waves, long long *redos);
int mclccd_batch_run(mclccd_batch *batch, void *stream);
int mclccd_batch_results(mclccd_batch *batch, long long *n_hits, double *min_toi, int *min_sten,
                         unsigned char *min_is_vf, long long *n_discrete, long long *n_stencils, double *done_ms,
                         double *batch_ms);
const char *mclccd_batch_last_error(const mclccd_batch *batch);

/* Replaces: BVHTree::traverse(BVHTraverse<T,DIM>*) (BVHTree.hpp:96,
 * BVHTree.cpp:162-166) through a device-side visitor (header-only
 * include/mclccd_b200/visit.cuh).  Read-only view of the tree of the last
 * update, valid until the next update or destroy (device memory):
 *   nodes      n_leaves - 1 nodes of 128 B, root = node 0: float4 l[3], r[3]
 *              = the left / right child's FP32 t0 and t1 boxes, outward
 *              rounded (3D: l[0] = t0lo.xyz, t0hi.x; l[1] = t0hi.yz, t1lo.xy;
 *              l[2] = t1lo.z, t1hi.xyz; 2D: l[0] = t0lo.xy, t0hi.xy;
 *              l[1] = t1lo.xy, t1hi.xy), then int4 d = {split, meta, last,
 *              parent}: the children are split and split + 1, each a leaf
 *              (sorted index) if meta bit 0 (left) / bit 1 (right) is set,
 *              else an internal node; last = the node's last leaf;
 *   leaf_box   per sorted leaf the exact FP64 boxes lo0[dim], hi0[dim],
 *              lo1[dim], hi1[dim] (t0 and t1, padded by box_eta);
 *   leaf_prim  sorted leaf -> primitive index. */
typedef struct {
    int dim, n_leaves;
    const void *nodes;
    const double *leaf_box;
    const int *leaf_prim;
} mclccd_tree_view;
int mclccd_get_tree_view(const mclccd_tree *tree, mclccd_tree_view *view);

/* Replaces: the host side of BVHTree::traverse(BVHTraverse<T,DIM>*)
 * (BVHTree.hpp:17-27, 96; BVHTree.cpp:162-166), which walks the tree on the
 * host calling a visitor's virtual intersectVolume / intersectObject: copies
 * the tree of the last update into caller host arrays (any may be NULL):
 * nodes (n_leaves - 1 records of 128 B, layout as in mclccd_tree_view),
 * leaf_box (n_leaves x 4 x dim doubles), leaf_prim (n_leaves ints) and
 * leaf_flags (n_leaves bytes: bits 0-2 vertex slots and 3-5 edge slots
 * represented, bit 6 active), all in sorted leaf order.  The C++ drop-in
 * (include/mclccd_b200/BVHTree.hpp) uses it for its visitor overload. */
int mclccd_get_tree_host(mclccd_tree *tree, void *nodes, double *leaf_box, int *leaf_prim, unsigned char *leaf_flags);

/* No counterpart in the reference: page-locked host memory from the CUDA
 * runtime, for callers that stage results without including CUDA headers
 * (device-to-host copies into it run asynchronously at full PCIe speed). */
int mclccd_host_alloc(size_t bytes, void **ptr);
int mclccd_host_free(void *ptr);

/* Input forms other than row-major double (no counterpart in the
 * reference; its Eigen overloads copy to RowMajor, BVHTree.hpp:151-186).
 * One device pass converts them into the arrays the path runs on, so the
 * caller's arrays are used as they are (host arrays are copied to the device
 * unchanged, with no host-side conversion):
 *   MCLCCD_IN_F32         V0/V1 are float (widened exactly to double);
 *   MCLCCD_IN_V_COLMAJOR  V0/V1 column-major: coordinate k of vertex i at
 *                         [k * nv + i] (Eigen's default MatrixXd layout);
 *   MCLCCD_IN_P_COLMAJOR  P column-major: slot j of primitive i at
 *                         [j * np + i] (Eigen's default MatrixXi layout).
 * in_flags = 0 is mclccd_update / mclccd_traverse. */
#define MCLCCD_IN_F32 1u
#define MCLCCD_IN_V_COLMAJOR 2u
#define MCLCCD_IN_P_COLMAJOR 4u
int mclccd_update_ex(mclccd_tree *tree, const void *V0, const void *V1, int nv, const int *P, int np, int pdim,
                     const int *active, int mem_kind, unsigned in_flags);
int mclccd_traverse_ex(mclccd_tree *tree, const void *V0, const void *V1, int nv, const int *P, int mem_kind,
                       unsigned in_flags);

/* float coordinates (the reference's BVHTree<float, DIM> instantiations,
 * BVHTree.cpp:506-507): V0/V1 are float (nv x dim, mem_kind side) and are
 * widened exactly to double on the device, then update / traverse run as
 * mclccd_update / mclccd_traverse on those doubles.  Results are therefore
 * the FP64 path's results for these coordinates (toi as double; the C++
 * BVHTree<float, DIM> rounds it down to float).  traverse_f32 with all
 * arrays NULL reuses the last update's. */
int mclccd_update_f32(mclccd_tree *tree, const float *V0, const float *V1, int nv, const int *P, int np, int pdim,
                      const int *active, int mem_kind);
int mclccd_traverse_f32(mclccd_tree *tree, const float *V0, const float *V1, int nv, const int *P, int mem_kind);

/* Per-stage device times (ms) of the last update + traverse when
 * MCLCCD_OPT_PROFILE is set: [update_total, build, refit, traverse_total,
 * tree_walk, expand, narrow]; returns how many were written. */
int mclccd_stage_ms(const mclccd_tree *tree, float *ms, int n);

/* No counterpart in the reference: launch-shape knobs of the device path
 * (chosen by the autotuner, mclccd_b200/autotune.py).  Keys: grid size (in
 * blocks) of the stencil-expansion kernel and of the ACCD kernels, the
 * tree-walk form (1: warp-cooperative packets, 0: one query per thread) and
 * the FP64 ACCD form (1: stencils that go on after the first distance are
 * re-binned in shared memory so warps run heads or tails, never both; 2: the
 * head in one kernel over the list, the tail in a second over a queue of the
 * stencils that go on; 0: one stencil per thread start to end), and the
 * walk's Morton window (W = 8, 16 (default), 32, 64 or 128: each query
 * first tests the W leaves after it in Morton order, staged by its block in
 * shared memory, then walks the tree only for leaves beyond them; 0: tree
 * walk only), and overlap (K = 2..16: the queries in K chunks, the walk of
 * chunk c + 1 running while chunk c is expanded and scored, on two internal
 * streams; 0: in sequence; FP64 and one-sided forms only), the FP64 narrow
 * phase form (0, the default: the expansion kernel writes the VF and EE
 * lists and one ACCD kernel runs over each; 1: one kernel takes the leaf
 * pairs to stencils, runs the discrete test and ACCD on them in per-warp
 * batches of one kind, and counts the candidate lists without writing them
 * (mclccd_get_candidates rebuilds them on request) -- measured slower), the grid size (in blocks) of
 * that fused kernel, and the refill walk (1: persistent warps take chunks of
 * 32 queries, run their window part, and refill lanes whose tree walk is
 * done from a per-warp pool of queries, so lanes do not idle behind the
 * longest walk of their warp; window 8, 16 or 32; 0: one query per thread
 * start to end), the expansion split (1: the stencil expansion and the
 * discrete test as two kernels; 2: the same with the discrete test's lanes
 * compacted, each warp queueing the pairs that share no vertex in shared
 * memory and testing them 32 at a time; 0: one kernel), and the rebuild ratio (in
 * percent; default 150): after each build and every fourth refit the box
 * areas of the internal nodes are summed relative to those of the leaves,
 * and when that grows past the ratio
 * of its value after the last full build, the next update rebuilds the
 * hierarchy (0: refit whenever P is unchanged), and the buffered walk (1:
 * the window walk collects each warp's leaf pairs in shared memory and
 * writes them in runs of 32 with one atomic, which also keeps neighbouring
 * queries' pairs together for the kernels that read them; 2, the default:
 * runs of 64; 0: one atomic per leaf test that hits; windows 0, 64 and 128
 * take the unbuffered walk).
 * The expansion split is on by default as well.  Results do not depend on
 * any of them. */
#define MCLCCD_TUNE_EXPAND_GRID 0
#define MCLCCD_TUNE_ACCD_GRID 1
#define MCLCCD_TUNE_WALK_PACKET 2
#define MCLCCD_TUNE_ACCD_REBIN 3
#define MCLCCD_TUNE_WALK_WINDOW 4
#define MCLCCD_TUNE_OVERLAP 5
#define MCLCCD_TUNE_NARROW_FUSED 6
#define MCLCCD_TUNE_FUSED_GRID 7
#define MCLCCD_TUNE_WALK_REFILL 8
#define MCLCCD_TUNE_EXPAND_SPLIT 9
#define MCLCCD_TUNE_REBUILD_RATIO 10
#define MCLCCD_TUNE_WALK_BUFFER 11
#define MCLCCD_TUNE_COUNT 12
int mclccd_set_tuning(mclccd_tree *tree, int key, int value);
int mclccd_get_tuning(const mclccd_tree *tree, int key, int *value);

/* Kernels launched by this handle since creation (for launch accounting). */
int mclccd_kernel_launches(const mclccd_tree *tree, long long *n);

/* Measured FP64 fused multiply-add throughput of a device, in TFLOP/s (one
 * FMA = 2 flops): eight independent FMA chains per thread over one wave of
 * 8 x 256-thread blocks per SM.  A diagnostic with no counterpart in the
 * reference: the measured denominator of the FP64 narrow phase's roofline. */
int mclccd_fp64_fma_rate(int device, double *tflops);

/* Human-readable message of the handle's last failure ("" if none). */
const char *mclccd_last_error(const mclccd_tree *tree);
const char *mclccd_status_string(int status);

#ifdef __cplusplus
}
#endif

#endif /* MCLCCD_B200_H */
