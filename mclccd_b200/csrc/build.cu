// LBVH build over swept leaf boxes: centroids + scene bounds, Morton codes,
// Karras hierarchy, fused FP64 leaf boxes + bottom-up FP32 refit, and the
// representative vertex/edge owner flags.
//
// Replaces mclccd's BVHTree::update (BVHTree.cpp:27-126): the per-primitive
// boxes (83-121), the representative-triangle pass (50-80) and the serial
// median-split Kd-BVH (ccd_internal/KdBVH.hpp:103-222).  Any hierarchy gives
// the same candidate set (the leaf test is exact and every leaf pair is
// visited once), so the tree shape is free to be the GPU-friendly one.
#include "common.cuh"
#include "kernels.cuh"
#include "lbvh.cuh"

namespace mclccd {

// Scene bounds of box centres, as ordered uints: [min(DIM), max(DIM)].
__global__ void k_init_bounds(unsigned *bounds, int dim)
{
    int t = threadIdx.x;
    if (t < dim) bounds[t] = 0xff800000u;            // ordered(+inf)
    else if (t < 2 * dim) bounds[t] = 0x007fffffu;   // ordered(-inf)
}

template <int DIM>
__global__ void k_centroids(const double *__restrict__ V0, const double *__restrict__ V1, const int *__restrict__ P,
                            int np, int pdim, int nv, float *__restrict__ cent, unsigned *bounds, Counters *cnt)
{
    float lo[DIM], hi[DIM];
#pragma unroll
    for (int k = 0; k < DIM; ++k) { lo[k] = __int_as_float(0x7f800000); hi[k] = -lo[k]; }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += gridDim.x * blockDim.x) {
        LeafBox<DIM> b;
        bool act;
        if (!compute_leaf_box<DIM>(V0, V1, P, pdim, nv, i, 0.0, nullptr, b, act)) atomicOr(&cnt->err, kErrBadIndex);
#pragma unroll
        for (int k = 0; k < DIM; ++k) {
            double mn = b.lo0[k] < b.lo1[k] ? b.lo0[k] : b.lo1[k];
            double mx = b.hi0[k] < b.hi1[k] ? b.hi1[k] : b.hi0[k];
            float c = (float)(0.5 * (mn + mx));
            if (!(c == c) || fabsf(c) > 3.0e38f) c = 0.f;   // keep NaN/huge out of the bounds
            cent[(size_t)i * DIM + k] = c;
            lo[k] = fminf(lo[k], c);
            hi[k] = fmaxf(hi[k], c);
        }
    }
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
        for (int o = 16; o > 0; o >>= 1) {
            lo[k] = fminf(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], o));
            hi[k] = fmaxf(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], o));
        }
        if (lane_id() == 0) {
            atomicMin(bounds + k, float_to_ordered(lo[k]));
            atomicMax(bounds + DIM + k, float_to_ordered(hi[k]));
        }
    }
}

template <int DIM>
__global__ void k_morton(const float *__restrict__ cent, int np, const unsigned *__restrict__ bounds,
                         unsigned *__restrict__ keys, int *__restrict__ vals)
{
    constexpr float kCells = DIM == 3 ? 1024.f : 32768.f;
    float lo[DIM], inv[DIM];
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
        lo[k] = ordered_to_float(bounds[k]);
        float ext = ordered_to_float(bounds[DIM + k]) - lo[k];
        inv[k] = ext > 0.f ? kCells / ext : 0.f;
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += gridDim.x * blockDim.x) {
        unsigned code = 0;
#pragma unroll
        for (int k = 0; k < DIM; ++k) {
            float q = (cent[(size_t)i * DIM + k] - lo[k]) * inv[k];
            unsigned u = (unsigned)fminf(fmaxf(q, 0.f), kCells - 1.f);
            code |= (DIM == 3 ? expand_bits3(u) : expand_bits2(u)) << (DIM == 3 ? 2 - k : 1 - k);
        }
        keys[i] = code;
        vals[i] = i;
    }
}

// ---------------------------------------------------------------------------
// Karras hierarchy ("Maximizing Parallelism in the Construction of BVHs,
// Octrees, and k-d Trees", HPG 2012): internal node i covers a contiguous
// sorted range with i as one end; its split gamma gives children gamma and
// gamma+1.  Equal keys are disambiguated by index (32 + clz(i ^ j)).
// ---------------------------------------------------------------------------
__device__ __forceinline__ int kdelta(const unsigned *__restrict__ keys, int n, int i, int j)
{
    if (j < 0 || j >= n) return -1;
    unsigned a = keys[i], b = keys[j];
    return a == b ? 32 + __clz(i ^ j) : __clz(a ^ b);
}

__global__ void k_karras(const unsigned *__restrict__ keys, int n, Node *__restrict__ nodes, int *__restrict__ leaf_parent)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    const int d = (kdelta(keys, n, i, i + 1) - kdelta(keys, n, i, i - 1)) >= 0 ? 1 : -1;
    const int dmin = kdelta(keys, n, i, i - d);
    int lmax = 2;
    while (kdelta(keys, n, i, i + lmax * d) > dmin) lmax <<= 1;
    int l = 0;
    for (int t = lmax >> 1; t >= 1; t >>= 1)
        if (kdelta(keys, n, i, i + (l + t) * d) > dmin) l += t;
    const int j = i + l * d;
    const int dnode = kdelta(keys, n, i, j);
    int s = 0, t = l;
    for (;;) {
        t = (t + 1) >> 1;
        if (kdelta(keys, n, i, i + (s + t) * d) > dnode) s += t;
        if (t <= 1) break;
    }
    const int gamma = i + s * d + (d < 0 ? -1 : 0);
    const int first = min(i, j), last = max(i, j);
    if (gamma < first || gamma >= last) return;   // cannot happen for sorted keys
    const bool lleaf = first == gamma, rleaf = last == gamma + 1;
    Node &nd = nodes[i];
    nd.d.x = gamma;
    nd.d.y = (lleaf ? kMetaLeftLeaf : 0) | (rleaf ? kMetaRightLeaf : 0);
    nd.d.z = last;
    if (i == 0) nd.d.w = -1;
    if (lleaf) leaf_parent[gamma] = i; else nodes[gamma].d.w = i;
    if (rleaf) leaf_parent[gamma + 1] = i; else nodes[gamma + 1].d.w = i;
}

// ---------------------------------------------------------------------------
// Refit: one thread per sorted leaf computes the exact FP64 leaf box (stored
// in sorted order for the traversal's exact test) and its outward-rounded
// FP32 t0 and t1 boxes, writes them into the parent's child slot, then
// climbs: the second thread to reach an internal node merges both child slots
// and moves up (first arrival stops).  `visits` must be zero on entry.
// ---------------------------------------------------------------------------
// Surface area (3D; half of it) or perimeter (2D; half of it) of a swept box.
template <int DIM>
__device__ __forceinline__ float swept_area(const Box2T<DIM> &b)
{
    float e[DIM];
#pragma unroll
    for (int c = 0; c < DIM; ++c) e[c] = fmaxf(b.t0hi[c], b.t1hi[c]) - fminf(b.t0lo[c], b.t1lo[c]);
    if constexpr (DIM == 3) return e[0] * e[1] + e[1] * e[2] + e[2] * e[0];
    else return e[0] + e[1];
}

template <int DIM>
__global__ void k_refit(const double *__restrict__ V0, const double *__restrict__ V1, const int *__restrict__ P,
                        int np, int pdim, int nv, double eta, const int *__restrict__ active,
                        const int *__restrict__ sorted, const int *__restrict__ leaf_parent, Node *nodes,
                        int *__restrict__ visits, LeafBox<DIM> *__restrict__ leaf_box,
                        unsigned char *__restrict__ leaf_active, Counters *cnt)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= np) return;
    const int prim = sorted[k];
    LeafBox<DIM> b;
    bool act;
    if (!compute_leaf_box<DIM>(V0, V1, P, pdim, nv, prim, eta, active, b, act)) atomicOr(&cnt->err, kErrBadIndex);
    leaf_box[k] = b;
    leaf_active[k] = act ? 1 : 0;
    if (np < 2) return;
    Box2T<DIM> box = outward<DIM>(b);
    int parent = leaf_parent[k];
    bool right = __ldg(&nodes[parent].d.x) != k;
    write_child<DIM>(nodes, parent, right, box, act);
    for (int level = 0; level < 256; ++level) {   // depth of a Karras tree over 30-bit keys is < 64
        if (!refit_second_arrival(visits + parent)) return;   // sibling subtree not done yet
        const int node = parent;
        merge_sibling<DIM>(nodes + node, right, box, act);
        parent = __ldcg(&nodes[node].d.w);
        if (parent < 0) return;   // root: its own box is never needed
        const int psplit = __ldg(&nodes[parent].d.x);
        const int pmeta = __ldg(&nodes[parent].d.y) & 0xff;
        right = !(psplit == node && !(pmeta & kMetaLeftLeaf));
        write_child<DIM>(nodes, parent, right, box, act);
    }
    atomicOr(&cnt->err, kErrStack);
}

// ---------------------------------------------------------------------------
// Representative flags (BVHTree.cpp:50-80): a vertex slot (face i, slot j) is
// flagged iff i*pdim + j is the smallest such position holding that vertex;
// an edge slot iff it is the smallest position holding that unordered edge.
// Owners are reduced with atomicMin, so the result is order-independent.
// Edges are keyed (min << 32 | max) in an open-addressing table.
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long mix64(unsigned long long x)
{
    x ^= x >> 33; x *= 0xff51afd7ed558ccdULL; x ^= x >> 33; x *= 0xc4ceb9fe1a85ec53ULL; x ^= x >> 33;
    return x;
}

__device__ __forceinline__ long long edge_slot(unsigned long long *keys, unsigned long long key, unsigned long long mask,
                                               bool insert)
{
    unsigned long long h = mix64(key) & mask;
    for (unsigned long long probe = 0; probe <= mask; ++probe) {
        unsigned long long cur = insert ? atomicCAS(keys + h, ~0ull, key) : keys[h];
        if (cur == key || (insert && cur == ~0ull)) return (long long)h;
        if (!insert && cur == ~0ull) return -1;
        h = (h + 1) & mask;
    }
    return -1;
}

__global__ void k_owner_scatter(const int *__restrict__ P, int np, int pdim, int nv, int *__restrict__ vowner,
                                unsigned long long *ekeys, int *eowner, unsigned long long emask, Counters *cnt)
{
    long long total = (long long)np * pdim;
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < total; s += (long long)gridDim.x * blockDim.x) {
        int i = (int)(s / pdim), j = (int)(s - (long long)i * pdim);
        int v = P[s];
        if (v < 0 || v >= nv) { atomicOr(&cnt->err, kErrBadIndex); continue; }
        atomicMin(vowner + v, (int)s);
        if (pdim != 3) continue;
        unsigned a = (unsigned)v, b = (unsigned)P[(size_t)i * 3 + (j + 1) % 3];
        if (b < a) { unsigned t = a; a = b; b = t; }
        long long h = edge_slot(ekeys, ((unsigned long long)a << 32) | b, emask, true);
        if (h < 0) { atomicOr(&cnt->err, kErrHashFull); continue; }
        atomicMin(eowner + h, (int)s);
    }
}

__global__ void k_owner_flags(const int *__restrict__ P, int np, int pdim, int nv, const int *__restrict__ vowner,
                              unsigned long long *ekeys, const int *__restrict__ eowner, unsigned long long emask,
                              unsigned char *__restrict__ flags)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    unsigned f = 0;
    for (int j = 0; j < pdim && j < 3; ++j) {
        long long s = (long long)i * pdim + j;
        int v = P[s];
        if (v < 0 || v >= nv) continue;
        if (vowner[v] == (int)s) f |= kFlagV0 << j;
        if (pdim != 3) continue;
        unsigned a = (unsigned)v, b = (unsigned)P[(size_t)i * 3 + (j + 1) % 3];
        if (b < a) { unsigned t = a; a = b; b = t; }
        long long h = edge_slot(ekeys, ((unsigned long long)a << 32) | b, emask, false);
        if (h >= 0 && eowner[h] == (int)s) f |= kFlagE0 << j;
    }
    flags[i] = (unsigned char)f;
}

// Topology check for the refit-only path: any difference -> *diff = 1.
__global__ void k_compare_int(const int4 *__restrict__ a, const int4 *__restrict__ b, long long n4,
                              const int *__restrict__ a_tail, const int *__restrict__ b_tail, int tail, int *diff)
{
    bool d = false;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n4; i += (long long)gridDim.x * blockDim.x) {
        int4 x = __ldg(a + i), y = __ldg(b + i);
        d |= (x.x != y.x) | (x.y != y.y) | (x.z != y.z) | (x.w != y.w);
    }
    if (blockIdx.x == 0 && threadIdx.x < tail) d |= a_tail[threadIdx.x] != b_tail[threadIdx.x];
    if (__any_sync(0xffffffffu, d) && lane_id() == 0) atomicOr(diff, 1);
}

// ---------------------------------------------------------------------------
// Host-side launchers.
// ---------------------------------------------------------------------------
static inline int grid_for(long long n, int block, int cap)
{
    long long g = (n + block - 1) / block;
    if (g < 1) g = 1;
    return (int)(g < cap ? g : cap);
}

void launch_centroids(int dim, const double *V0, const double *V1, const int *P, int np, int pdim, int nv,
                      float *cent, unsigned *bounds, Counters *cnt, cudaStream_t st)
{
    k_init_bounds<<<1, 32, 0, st>>>(bounds, dim);
    int g = grid_for(np, 256, 148 * 16);
    if (dim == 3) k_centroids<3><<<g, 256, 0, st>>>(V0, V1, P, np, pdim, nv, cent, bounds, cnt);
    else k_centroids<2><<<g, 256, 0, st>>>(V0, V1, P, np, pdim, nv, cent, bounds, cnt);
}

void launch_morton(int dim, const float *cent, int np, const unsigned *bounds, unsigned *keys, int *vals, cudaStream_t st)
{
    int g = grid_for(np, 256, 148 * 16);
    if (dim == 3) k_morton<3><<<g, 256, 0, st>>>(cent, np, bounds, keys, vals);
    else k_morton<2><<<g, 256, 0, st>>>(cent, np, bounds, keys, vals);
}

void launch_karras(const unsigned *keys, int n, Node *nodes, int *leaf_parent, cudaStream_t st)
{
    if (n < 2) return;
    k_karras<<<(n - 1 + 255) / 256, 256, 0, st>>>(keys, n, nodes, leaf_parent);
}

void launch_refit(int dim, const double *V0, const double *V1, const int *P, int np, int pdim, int nv, double eta,
                  const int *active, const int *sorted, const int *leaf_parent, Node *nodes, int *visits,
                  void *leaf_box, unsigned char *leaf_active, Counters *cnt, cudaStream_t st)
{
    if (np < 1) return;
    if (np > 1) cudaMemsetAsync(visits, 0, sizeof(int) * (size_t)(np - 1), st);
    int g = (np + 255) / 256;
    if (dim == 3)
        k_refit<3><<<g, 256, 0, st>>>(V0, V1, P, np, pdim, nv, eta, active, sorted, leaf_parent, nodes, visits,
                                      reinterpret_cast<LeafBox<3> *>(leaf_box), leaf_active, cnt);
    else
        k_refit<2><<<g, 256, 0, st>>>(V0, V1, P, np, pdim, nv, eta, active, sorted, leaf_parent, nodes, visits,
                                      reinterpret_cast<LeafBox<2> *>(leaf_box), leaf_active, cnt);
}

// Tree quality after a refit: over every node record (both children's
// boxes), the summed areas of the internal children and of the leaf
// children; coalesced reads of the node array, one atomic per block.
template <int DIM>
__global__ void __launch_bounds__(256) k_tree_quality(const Node *__restrict__ nodes, int n_nodes, double *out)
{
    constexpr int S = DIM == 3 ? 3 : 2;
    double inner = 0.0, leaves = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_nodes; i += gridDim.x * blockDim.x) {
        float4 ls[S], rs[S];
#pragma unroll
        for (int j = 0; j < S; ++j) { ls[j] = __ldg(&nodes[i].l[j]); rs[j] = __ldg(&nodes[i].r[j]); }
        const int meta = __ldg(&nodes[i].d.y);
        Box2T<DIM> lb, rb;
        unpack_child<DIM>(ls, lb);
        unpack_child<DIM>(rs, rb);
        const double al = swept_area<DIM>(lb), ar = swept_area<DIM>(rb);
        if (meta & kMetaLeftLeaf) leaves += al; else inner += al;
        if (meta & kMetaRightLeaf) leaves += ar; else inner += ar;
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        inner += __shfl_xor_sync(0xffffffffu, inner, o);
        leaves += __shfl_xor_sync(0xffffffffu, leaves, o);
    }
    __shared__ double s[2][8];
    const int w = threadIdx.x >> 5;
    if (lane_id() == 0) { s[0][w] = inner; s[1][w] = leaves; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) { a += s[0][k]; b += s[1][k]; }
        atomicAdd(out, a);
        atomicAdd(out + 1, b);
    }
}

void launch_tree_quality(int dim, const Node *nodes, int np, double *out, cudaStream_t st)
{
    cudaMemsetAsync(out, 0, 2 * sizeof(double), st);
    if (np < 2) return;
    const int g = grid_for(np - 1, 256, 148 * 8);
    if (dim == 3) k_tree_quality<3><<<g, 256, 0, st>>>(nodes, np - 1, out);
    else k_tree_quality<2><<<g, 256, 0, st>>>(nodes, np - 1, out);
}

void launch_owner_flags(const int *P, int np, int pdim, int nv, int *vowner, unsigned long long *ekeys, int *eowner,
                        unsigned long long ecap, unsigned char *flags, Counters *cnt, cudaStream_t st)
{
    cudaMemsetAsync(vowner, 0x7f, sizeof(int) * (size_t)nv, st);
    if (pdim == 3) {
        cudaMemsetAsync(ekeys, 0xff, sizeof(unsigned long long) * ecap, st);
        cudaMemsetAsync(eowner, 0x7f, sizeof(int) * ecap, st);
    }
    long long total = (long long)np * pdim;
    k_owner_scatter<<<grid_for(total, 256, 148 * 16), 256, 0, st>>>(P, np, pdim, nv, vowner, ekeys, eowner, ecap - 1, cnt);
    k_owner_flags<<<(np + 255) / 256, 256, 0, st>>>(P, np, pdim, nv, vowner, ekeys, eowner, ecap - 1, flags);
}

// out = max(out, 1 + the largest entry of a[0..n)): the vertex count implied
// by a primitive array.
__global__ void k_max_index(const int *__restrict__ a, long long n, int *out)
{
    int m = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        m = max(m, __ldg(a + i) + 1);
#pragma unroll
    for (int o = 16; o; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane_id() == 0 && m > 0) atomicMax(out, m);
}

void launch_max_index(const int *a, long long n, int *out, cudaStream_t st)
{
    k_max_index<<<grid_for(n, 256, 148 * 8), 256, 0, st>>>(a, n, out);
}

void launch_compare(const int *a, const int *b, long long n, int *diff, cudaStream_t st)
{
    long long n4 = n / 4;
    int tail = (int)(n - n4 * 4);
    k_compare_int<<<grid_for(n4, 256, 148 * 8), 256, 0, st>>>(reinterpret_cast<const int4 *>(a),
                                                             reinterpret_cast<const int4 *>(b), n4, a + n4 * 4,
                                                             b + n4 * 4, tail, diff);
}

} // namespace mclccd
