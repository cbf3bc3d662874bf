// Device visitor traversal of the tree: the B200 form of the reference's
// BVHTree::traverse(BVHTraverse<T,DIM>*) (include/MCL/BVHTree.hpp:17-27, 96;
// BVHTree.cpp:162-166), used there for point-in-element queries
// (examples/traverser.cpp).  Header-only: include from a .cu file compiled by
// nvcc (for sm_100a) and link libmclccd_b200.so.
//
// The reference's visitor has intersectVolume(box) -> descend? and
// intersectObject(leaf) -> stop?.  Here many independent queries run at
// once, one thread each, and the visitor is a functor with the query index:
//
//   struct Visitor {
//       // node volume (swept box, FP32 bounds rounded outward, so never
//       // smaller than the reference's merged box): true = visit its children
//       __device__ bool volume(int q, const double *lo, const double *hi) const;
//       // a leaf whose parent volume passed: its primitive and exact FP64
//       // swept box; true = stop this query
//       __device__ bool object(int q, int prim, const double *lo, const double *hi) const;
//   };
//   mcl::b200::visit(tree, n_queries, Visitor{...});
//
// As in the reference, the root volume is tested first and a leaf reaches
// object() when its parent's volume test passed.  A visitor whose volume
// test is a conservative "may contain" test (box contains point, boxes
// overlap) reports the same objects as the reference's; it sees more
// volumes only when a test tells the outward FP32 bounds from the exact ones.
#pragma once

#include "BVHTree.hpp"

#include <cuda_runtime.h>

namespace mcl {
namespace b200 {

namespace detail_visit {

struct NodeView {
    float4 l[3], r[3];
    int4 d;
    int4 pad;
};

constexpr int kVisitStack = 64;

template <int DIM>
__device__ inline void child_box(const float4 *s, double *lo, double *hi)
{
    float t0lo[DIM], t0hi[DIM], t1lo[DIM], t1hi[DIM];
    if constexpr (DIM == 3) {
        t0lo[0] = s[0].x; t0lo[1] = s[0].y; t0lo[2] = s[0].z; t0hi[0] = s[0].w;
        t0hi[1] = s[1].x; t0hi[2] = s[1].y; t1lo[0] = s[1].z; t1lo[1] = s[1].w;
        t1lo[2] = s[2].x; t1hi[0] = s[2].y; t1hi[1] = s[2].z; t1hi[2] = s[2].w;
    } else {
        t0lo[0] = s[0].x; t0lo[1] = s[0].y; t0hi[0] = s[0].z; t0hi[1] = s[0].w;
        t1lo[0] = s[1].x; t1lo[1] = s[1].y; t1hi[0] = s[1].z; t1hi[1] = s[1].w;
    }
    for (int k = 0; k < DIM; ++k) {
        lo[k] = (double)fminf(t0lo[k], t1lo[k]);
        hi[k] = (double)fmaxf(t0hi[k], t1hi[k]);
    }
}

template <int DIM>
__device__ inline void leaf_swept(const double *lb, int k, double *lo, double *hi)
{
    const double *b = lb + (size_t)k * 4 * DIM;   // lo0, hi0, lo1, hi1
    for (int i = 0; i < DIM; ++i) {
        lo[i] = b[i] < b[2 * DIM + i] ? b[i] : b[2 * DIM + i];
        hi[i] = b[DIM + i] < b[3 * DIM + i] ? b[3 * DIM + i] : b[DIM + i];
    }
}

template <int DIM, class Visitor>
__global__ void k_visit(mclccd_tree_view view, int n_queries, Visitor vis, int *overflow)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n_queries) return;
    double lo[DIM], hi[DIM];
    if (view.n_leaves == 1) {
        leaf_swept<DIM>(view.leaf_box, 0, lo, hi);
        if (vis.volume(q, lo, hi)) vis.object(q, view.leaf_prim[0], lo, hi);
        return;
    }
    const NodeView *nodes = static_cast<const NodeView *>(view.nodes);
    constexpr int S = DIM == 3 ? 3 : 2;
    {   // root volume = hull of its children
        double l2[DIM], h2[DIM];
        child_box<DIM>(nodes[0].l, lo, hi);
        child_box<DIM>(nodes[0].r, l2, h2);
        for (int k = 0; k < DIM; ++k) { lo[k] = lo[k] < l2[k] ? lo[k] : l2[k]; hi[k] = hi[k] > h2[k] ? hi[k] : h2[k]; }
        if (!vis.volume(q, lo, hi)) return;
    }
    int stack[kVisitStack];
    int sp = 0, node = 0;
    for (int steps = 0; steps < view.n_leaves; ++steps) {
        const NodeView &nd = nodes[node];
        const int split = nd.d.x, meta = nd.d.y;
        int next[2], nn = 0;
        for (int c = 0; c < 2; ++c) {
            const int child = split + c;
            const bool leaf = (meta >> c) & 1;
            if (leaf) {
                leaf_swept<DIM>(view.leaf_box, child, lo, hi);
                if (vis.object(q, view.leaf_prim[child], lo, hi)) return;
            } else {
                child_box<DIM>(c ? nd.r : nd.l, lo, hi);
                if (vis.volume(q, lo, hi)) next[nn++] = child;
            }
        }
        (void)S;
        if (nn == 2) {
            if (sp < kVisitStack) stack[sp++] = next[1];
            else { atomicExch(overflow, 1); return; }
        }
        if (nn >= 1) node = next[0];
        else if (sp > 0) node = stack[--sp];
        else return;
    }
}

inline void check(cudaError_t e, const char *what)
{
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw CCDError(MCLCCD_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    }
}

} // namespace detail_visit

// Runs n_queries visitor queries over the tree of the last update.
template <int DIM, class Visitor>
void visit(const BVHTree<double, DIM> &tree, int n_queries, Visitor visitor, cudaStream_t stream = nullptr)
{
    mclccd_tree_view view;
    const int rc = mclccd_get_tree_view(tree.handle(), &view);
    if (rc != MCLCCD_OK) throw CCDError(rc, mclccd_status_string(rc));
    if (n_queries <= 0) return;
    int *overflow = nullptr;
    detail_visit::check(cudaMalloc(&overflow, sizeof(int)), "cudaMalloc");
    detail_visit::check(cudaMemsetAsync(overflow, 0, sizeof(int), stream), "cudaMemsetAsync");
    detail_visit::k_visit<DIM, Visitor><<<(n_queries + 127) / 128, 128, 0, stream>>>(view, n_queries, visitor,
                                                                                    overflow);
    int h = 0;
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, overflow, sizeof(int), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    cudaFree(overflow);
    detail_visit::check(e, "visit");
    if (h) throw CCDError(MCLCCD_ERR_DEVICE, "visit: traversal stack overflow");
}

} // namespace b200
} // namespace mcl
