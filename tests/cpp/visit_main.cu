// Driver for the device visitor (include/mclccd_b200/visit.cuh): the
// point-in-triangle query of the reference's examples/traverser.cpp on a 2D
// triangle mesh, many points at once.  Reads nv, nf, nq, V (nv x 2), F
// (nf x 3), Q (nq x 2); writes the number of (point, triangle) pairs found,
// then the pairs.
#include <cstdio>
#include <vector>

#include "mclccd_b200/visit.cuh"

struct PointInTriangle {
    const double *V;
    const int *F;
    const double *Q;
    int2 *out;
    unsigned long long *n_out;
    unsigned long long cap;

    __device__ bool volume(int q, const double *lo, const double *hi) const
    {
        const double x = Q[2 * q], y = Q[2 * q + 1];
        return lo[0] <= x && x <= hi[0] && lo[1] <= y && y <= hi[1];
    }
    __device__ bool object(int q, int prim, const double *, const double *) const
    {
        const double *a = V + 2 * F[3 * prim], *b = V + 2 * F[3 * prim + 1], *c = V + 2 * F[3 * prim + 2];
        const double px = Q[2 * q], py = Q[2 * q + 1];
        const double v0x = b[0] - a[0], v0y = b[1] - a[1], v1x = c[0] - a[0], v1y = c[1] - a[1];
        const double v2x = px - a[0], v2y = py - a[1];
        const double d00 = v0x * v0x + v0y * v0y, d01 = v0x * v1x + v0y * v1y, d11 = v1x * v1x + v1y * v1y;
        const double d20 = v2x * v0x + v2y * v0y, d21 = v2x * v1x + v2y * v1y;
        const double inv = 1.0 / (d00 * d11 - d01 * d01);
        const double r1 = (d11 * d20 - d01 * d21) * inv, r2 = (d00 * d21 - d01 * d20) * inv, r0 = 1.0 - r1 - r2;
        if (r0 >= 0 && r1 >= 0 && r2 >= 0) {
            const unsigned long long s = atomicAdd(n_out, 1ull);
            if (s < cap) out[s] = make_int2(q, prim);
        }
        return false;   // keep traversing
    }
};

int main(int argc, char **argv)
{
    if (argc != 3) return 2;
    FILE *f = std::fopen(argv[1], "rb");
    if (!f) return 2;
    int hdr[3];
    if (std::fread(hdr, sizeof(int), 3, f) != 3) return 2;
    const int nv = hdr[0], nf = hdr[1], nq = hdr[2];
    std::vector<double> V(2 * (size_t)nv), Q(2 * (size_t)nq);
    std::vector<int> F(3 * (size_t)nf);
    if (std::fread(V.data(), sizeof(double), V.size(), f) != V.size() ||
        std::fread(F.data(), sizeof(int), F.size(), f) != F.size() ||
        std::fread(Q.data(), sizeof(double), Q.size(), f) != Q.size())
        return 2;
    std::fclose(f);

    mcl::BVHTree<double, 2> tree;
    tree.update(V.data(), V.data(), F.data(), nf, 3);   // the reference's signature, host arrays

    PointInTriangle vis;
    double *dV, *dQ;
    int *dF;
    cudaMalloc(&dV, V.size() * sizeof(double));
    cudaMalloc(&dQ, Q.size() * sizeof(double));
    cudaMalloc(&dF, F.size() * sizeof(int));
    cudaMemcpy(dV, V.data(), V.size() * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(dQ, Q.data(), Q.size() * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(dF, F.data(), F.size() * sizeof(int), cudaMemcpyHostToDevice);
    vis.V = dV; vis.F = dF; vis.Q = dQ;
    vis.cap = 8ull * nq + 64;
    cudaMalloc(&vis.out, vis.cap * sizeof(int2));
    cudaMalloc(&vis.n_out, sizeof(unsigned long long));
    cudaMemset(vis.n_out, 0, sizeof(unsigned long long));
    mcl::b200::visit(tree, nq, vis);

    unsigned long long n = 0;
    cudaMemcpy(&n, vis.n_out, sizeof(n), cudaMemcpyDeviceToHost);
    if (n > vis.cap) return 3;
    std::vector<int2> pairs(n);
    cudaMemcpy(pairs.data(), vis.out, n * sizeof(int2), cudaMemcpyDeviceToHost);
    FILE *g = std::fopen(argv[2], "wb");
    if (!g) return 2;
    const long long nn = (long long)n;
    std::fwrite(&nn, sizeof(nn), 1, g);
    std::fwrite(pairs.data(), sizeof(int2), pairs.size(), g);
    std::fclose(g);
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 1;
}
