// Host-callable kernel launchers (internal to libmclccd_b200.so).
#pragma once

#include "common.cuh"
#include <cstddef>

namespace mclccd {

// build.cu
void launch_centroids(int dim, const double *V0, const double *V1, const int *P, int np, int pdim, int nv,
                      float *cent, unsigned *bounds, Counters *cnt, cudaStream_t st);
void launch_morton(int dim, const float *cent, int np, const unsigned *bounds, unsigned *keys, int *vals, cudaStream_t st);
void launch_karras(const unsigned *keys, int n, Node *nodes, int *leaf_parent, cudaStream_t st);
void launch_refit(int dim, const double *V0, const double *V1, const int *P, int np, int pdim, int nv, double eta,
                  const int *active, const int *sorted, const int *leaf_parent, Node *nodes, int *visits,
                  void *leaf_box, unsigned char *leaf_active, Counters *cnt, cudaStream_t st);
// out[0] = summed surface areas (perimeters in 2D) of the internal nodes'
// swept boxes, out[1] = of the leaves' boxes (2 device doubles)
void launch_tree_quality(int dim, const Node *nodes, int np, double *out, cudaStream_t st);
void launch_owner_flags(const int *P, int np, int pdim, int nv, int *vowner, unsigned long long *ekeys, int *eowner,
                        unsigned long long ecap, unsigned char *flags, Counters *cnt, cudaStream_t st);
void launch_compare(const int *a, const int *b, long long n, int *diff, cudaStream_t st);
void launch_max_index(const int *a, long long n, int *out, cudaStream_t st);

// sort.cu
int sort_num_passes(unsigned key_bits);
size_t sort_scratch_bytes(int n, int passes);
void launch_sort_pairs(unsigned *keys, int *vals, unsigned *keys_alt, int *vals_alt, int n, unsigned key_bits,
                       void *scratch, Counters *cnt, cudaStream_t st);

// traverse.cu
// queries [q_begin, q_end) (q_end < 0: to the end)
void launch_traverse(int dim, int packet, int window, const Node *nodes, const void *leaf_box, const unsigned char *leaf_active,
                     const int *sorted, int n, int2 *pairs, unsigned long long cap, Counters *cnt, cudaStream_t st,
                     int q_begin = 0, int q_end = -1);
// the window walk with idle lanes refilled from a per-warp pool of queries
// (persistent; cursor: one device unsigned, zeroed by the launcher)
void launch_traverse_refill(int dim, int window, const Node *nodes, const void *leaf_box,
                            const unsigned char *leaf_active, const int *sorted, int n, int2 *pairs,
                            unsigned long long cap, Counters *cnt, unsigned *cursor, cudaStream_t st,
                            int q_begin = 0, int q_end = -1);
void launch_expand_pairs(int dim, const int2 *pairs, unsigned long long pair_cap, const int *P,
                         const unsigned char *flags, const double *V1, int nv, int4 *vf, unsigned long long vf_cap,
                         int4 *ee, unsigned long long ee_cap, int2 *disc, unsigned long long disc_cap, int continuous,
                         int discrete, Counters *cnt, int grid, cudaStream_t st,
                         const unsigned long long *lo_ptr = nullptr, const unsigned long long *hi_ptr = nullptr);
// the discrete test of leaf pairs [*lo, *hi) alone (hi == nullptr: the pair count)
// the window walk with pairs collected per warp and written in runs of 32
// (run < 64) or 64
void launch_traverse_buffered(int dim, int window, int run, const Node *nodes, const void *leaf_box,
                              const unsigned char *leaf_active, const int *sorted, int n, int2 *pairs,
                              unsigned long long cap, Counters *cnt, cudaStream_t st, int q_begin = 0,
                              int q_end = -1);
void launch_discrete_pairs(int dim, const int2 *pairs, unsigned long long pair_cap, const int *P, const double *V1,
                           int nv, int2 *disc, unsigned long long disc_cap, Counters *cnt, int grid, cudaStream_t st,
                           const unsigned long long *lo_ptr = nullptr, const unsigned long long *hi_ptr = nullptr,
                           bool compact = false);
void launch_snapshot(const unsigned long long *a, unsigned long long *da, const unsigned long long *b,
                     unsigned long long *db, cudaStream_t st);

// narrow.cu
void launch_accd_pipeline(int dim, bool vf, const int4 *sten, const unsigned long long *n_ptr, unsigned long long cap,
                          const double *V0, const double *V1, int nv, double eta, int4 *hit_sten, double *hit_toi,
                          unsigned char *hit_isvf, unsigned long long hit_cap, Counters *cnt, int grid, bool rebin,
                          cudaStream_t st, const unsigned long long *lo_ptr = nullptr);
// narrow.cu: the head / tail split of the FP64 ACCD over one list (two
// launches; q_idx / q_state hold up to cap entries, q_count is zeroed here)
void launch_accd_split(int dim, bool vf, const int4 *sten, const unsigned long long *n_ptr, unsigned long long cap,
                       const double *V0, const double *V1, int nv, double eta, int4 *hit_sten, double *hit_toi,
                       unsigned char *hit_isvf, unsigned long long hit_cap, Counters *cnt, int grid, unsigned *q_idx,
                       double2 *q_state, unsigned long long *q_count, cudaStream_t st,
                       const unsigned long long *lo_ptr = nullptr);
// fused.cu: leaf pairs [*lo, *hi) -> stencils -> discrete test + FP64 ACCD in
// one kernel (candidate lists counted, not written)
void launch_narrow_fused(int dim, const int2 *pairs, unsigned long long pair_cap, const int *P,
                         const unsigned char *flags, const double *V0, const double *V1, int nv, double vf_eta,
                         double ee_eta, int continuous, int discrete, int2 *disc, unsigned long long disc_cap,
                         int4 *hit_sten, double *hit_toi, unsigned char *hit_isvf, unsigned long long hit_cap,
                         Counters *cnt, int grid, cudaStream_t st, const unsigned long long *lo_ptr = nullptr,
                         const unsigned long long *hi_ptr = nullptr);
// certified.cu
void launch_accd_certified(int dim, bool vf, const int4 *sten, const unsigned long long *n_ptr,
                           unsigned long long cap, const double *V0, const double *V1, int nv, double eta,
                           int4 *hit_sten, double *hit_toi, unsigned char *hit_isvf, unsigned long long hit_cap,
                           unsigned *queue, Counters *cnt, int grid, cudaStream_t st);
void launch_accd_certified_bulk(int dim, const int *sten, const unsigned char *is_vf, long long n, const double *V0,
                                const double *V1, int nv, double vf_eta, double ee_eta, double *out_toi, int *out_hit,
                                long long *queue, Counters *cnt, cudaStream_t st);
// adjoint.cu
void launch_vjp_toi(int dim, const int *sten, const unsigned char *is_vf, const double *toi, const double *g,
                    long long n, const double *V0, const double *V1, int nv, double vf_eta, double ee_eta,
                    double *dV0, double *dV1, double *t_star, int *status, double *rows, unsigned long long *n_ok,
                    cudaStream_t st);
void launch_accd_bulk(int dim, const int *sten, const unsigned char *is_vf, long long n, const double *V0,
                      const double *V1, int nv, double vf_eta, double ee_eta, double *out_toi, int *out_hit,
                      Counters *cnt, cudaStream_t st, bool vf_one_sided = false);
// narrow.cu: one-sided VF narrow phase (CTCD) over the VF list
void launch_ctcd_pipeline(int dim, const int4 *sten, const unsigned long long *n_ptr, unsigned long long cap,
                          const double *V0, const double *V1, int nv, double eta, int4 *hit_sten, double *hit_toi,
                          unsigned char *hit_isvf, unsigned long long hit_cap, Counters *cnt, int grid, cudaStream_t st,
                          const unsigned long long *lo_ptr = nullptr);

} // namespace mclccd
