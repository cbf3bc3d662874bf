// The reference's visitor interface through the C++ drop-in: point-in-
// triangle queries on a 2D triangle mesh, written the way reference code
// writes them (examples/traverser.cpp: a BVHTraverse<double, 2> subclass
// whose intersectVolume tests box containment and whose intersectObject
// records the triangles whose barycentric coordinates are all >= 0), run by
// BVHTree<double, 2>::traverse(BVHTraverse *).
//
//   traverser_main scene.bin out.bin
// scene.bin: int32 nv, nf, nq; nv x 2 f64 V; nf x 3 int32 F; nq x 2 f64 points.
// out.bin:   per query: int32 count, then the triangle indices found.
#include "mclccd_b200/BVHTree.hpp"

#include <cstdio>
#include <vector>

namespace {

class PointInTriangle : public mcl::BVHTraverse<double, 2> {
public:
    std::array<double, 2> pt{};
    const double *V = nullptr;
    const int *F = nullptr;
    std::vector<int> in_tri;

    bool intersectVolume(const VolumeType &v) override { return v.contains(pt); }
    bool intersectObject(const ObjectType &o) override
    {
        const int *f = F + 3 * o.idx;
        const double *a = V + 2 * f[0], *b = V + 2 * f[1], *c = V + 2 * f[2];
        const double v0[2] = {b[0] - a[0], b[1] - a[1]}, v1[2] = {c[0] - a[0], c[1] - a[1]};
        const double v2[2] = {pt[0] - a[0], pt[1] - a[1]};
        const double d00 = v0[0] * v0[0] + v0[1] * v0[1], d01 = v0[0] * v1[0] + v0[1] * v1[1];
        const double d11 = v1[0] * v1[0] + v1[1] * v1[1], d20 = v2[0] * v0[0] + v2[1] * v0[1];
        const double d21 = v2[0] * v1[0] + v2[1] * v1[1];
        const double inv = 1.0 / (d00 * d11 - d01 * d01);
        const double s = (d11 * d20 - d01 * d21) * inv, t = (d00 * d21 - d01 * d20) * inv;
        if (s >= 0 && t >= 0 && 1.0 - s - t >= 0) in_tri.push_back(o.idx);
        return false;   // true would stop the traversal
    }
};

} // namespace

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
    if (std::fread(V.data(), sizeof(double), V.size(), f) != V.size()) return 2;
    if (std::fread(F.data(), sizeof(int), F.size(), f) != F.size()) return 2;
    if (std::fread(Q.data(), sizeof(double), Q.size(), f) != Q.size()) return 2;
    std::fclose(f);

    mcl::BVHTree<double, 2> tree;
    tree.update(V.data(), V.data(), F.data(), nf, 3);
    PointInTriangle vis;
    vis.V = V.data();
    vis.F = F.data();
    FILE *o = std::fopen(argv[2], "wb");
    if (!o) return 2;
    for (int q = 0; q < nq; ++q) {
        vis.pt = {Q[2 * q], Q[2 * q + 1]};
        vis.in_tri.clear();
        tree.traverse(&vis);
        const int n = (int)vis.in_tri.size();
        std::fwrite(&n, sizeof(int), 1, o);
        std::fwrite(vis.in_tri.data(), sizeof(int), vis.in_tri.size(), o);
    }
    std::fclose(o);
    return 0;
}
