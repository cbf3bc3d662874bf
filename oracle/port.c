/*
 * TEST INFRASTRUCTURE -- the oracle (CPU restatement).  Only tests/, the
 * smoke check and bench.py's CPU-baseline leg load it; the product library
 * never does.
 *
 * A plain-C restatement of mattoverby/mclccd's CCD hot path, written for this
 * project from the reference's semantics.  Parity of this restatement is
 * pinned against the reference's own sources (oracle/_ref, built from the
 * unmodified reference code) by tests/test_oracle.py.
 *
 * Conventions: FP64 throughout, every expression evaluated in the order the
 * reference writes it (compile with -ffp-contract=off: no FMA contraction);
 * reductions accumulate left to right ((x0*y0 + x1*y1) + x2*y2).
 *
 * Leaf boxes are stored per primitive as 6*dim doubles:
 *   [swept.min, swept.max, t0.min, t0.max, t1.min, t1.max].
 * Flags per primitive (uint8): bit j = vertex slot j represented, bit 3+j =
 * edge slot j represented, bit 6 = active.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define FLAG_V(j) (1u << (j))
#define FLAG_E(j) (1u << (3 + (j)))
#define FLAG_ACTIVE (1u << 6)

/* ---------------------------------------------------------------------- */
/* Leaf boxes: BVHTree.cpp:83-121 (AlignedBox extend over V0 and V1, then    */
/* min -= box_eta, max += box_eta; active if no mask or any vertex active).  */
/* ---------------------------------------------------------------------- */
void port_leaf_boxes(int dim, const double *V0, const double *V1, const int *P, int np, int pdim,
                     double eta, const int *active, double *boxes, unsigned char *flags)
{
    for (int i = 0; i < np; ++i) {
        double *b = boxes + (size_t)i * 6 * dim;
        for (int k = 0; k < dim; ++k) {
            b[0 * dim + k] = DBL_MAX; b[1 * dim + k] = -DBL_MAX;
            b[2 * dim + k] = DBL_MAX; b[3 * dim + k] = -DBL_MAX;
            b[4 * dim + k] = DBL_MAX; b[5 * dim + k] = -DBL_MAX;
        }
        int act = active == NULL;
        for (int j = 0; j < pdim; ++j) {
            int v = P[(size_t)i * pdim + j];
            for (int k = 0; k < dim; ++k) {
                double a = V0[(size_t)v * dim + k], c = V1[(size_t)v * dim + k];
                if (a < b[2 * dim + k]) b[2 * dim + k] = a;
                if (b[3 * dim + k] < a) b[3 * dim + k] = a;
                if (c < b[4 * dim + k]) b[4 * dim + k] = c;
                if (b[5 * dim + k] < c) b[5 * dim + k] = c;
                if (a < b[0 * dim + k]) b[0 * dim + k] = a;
                if (b[1 * dim + k] < a) b[1 * dim + k] = a;
                if (c < b[0 * dim + k]) b[0 * dim + k] = c;
                if (b[1 * dim + k] < c) b[1 * dim + k] = c;
            }
            if (active != NULL && active[v]) act = 1;
        }
        for (int k = 0; k < dim; ++k) {
            b[2 * dim + k] -= eta; b[4 * dim + k] -= eta; b[0 * dim + k] -= eta;
            b[3 * dim + k] += eta; b[5 * dim + k] += eta; b[1 * dim + k] += eta;
        }
        if (flags) flags[i] = (unsigned char)((flags[i] & ~FLAG_ACTIVE) | (act ? FLAG_ACTIVE : 0));
    }
}

/* ---------------------------------------------------------------------- */
/* Representative flags: BVHTree.cpp:50-80.  Vertex slot j of face i is      */
/* flagged iff it is the first occurrence of that vertex scanning P in row   */
/* order; edge slot j (vertices j,(j+1)%3, unordered) iff it is the first    */
/* occurrence of that edge.  Edges only for pdim == 3.                       */
/* ---------------------------------------------------------------------- */
static uint64_t mix64(uint64_t x)
{
    x ^= x >> 33; x *= 0xff51afd7ed558ccdULL; x ^= x >> 33; x *= 0xc4ceb9fe1a85ec53ULL; x ^= x >> 33;
    return x;
}

int port_reptri(const int *P, int np, int pdim, int nv, unsigned char *flags)
{
    unsigned char *seen = (unsigned char *)calloc((size_t)nv + 1, 1);
    size_t cap = 16;
    while (cap < (size_t)np * 3 * 2) cap <<= 1;
    uint64_t *tab = (uint64_t *)malloc(cap * sizeof(uint64_t));
    if (!seen || !tab) { free(seen); free(tab); return -1; }
    memset(tab, 0xff, cap * sizeof(uint64_t));
    for (int i = 0; i < np; ++i) {
        unsigned f = flags[i] & FLAG_ACTIVE;
        for (int j = 0; j < pdim; ++j) {
            int v = P[(size_t)i * pdim + j];
            if (v >= 0 && v < nv && !seen[v]) { seen[v] = 1; f |= FLAG_V(j); }
            if (pdim != 3) continue;
            uint32_t e0 = (uint32_t)v, e1 = (uint32_t)P[(size_t)i * pdim + (j + 1) % 3];
            if (e1 < e0) { uint32_t t = e0; e0 = e1; e1 = t; }
            uint64_t key = ((uint64_t)e0 << 32) | e1;
            size_t h = (size_t)(mix64(key) & (cap - 1));
            for (;;) {
                if (tab[h] == UINT64_MAX) { tab[h] = key; f |= FLAG_E(j); break; }
                if (tab[h] == key) break;
                h = (h + 1) & (cap - 1);
            }
        }
        flags[i] = (unsigned char)f;
    }
    free(seen); free(tab);
    return 0;
}

/* ---------------------------------------------------------------------- */
/* Box predicate: BVHTree.cpp:401-426.                                      */
/* ---------------------------------------------------------------------- */
static int box_empty(const double *lo, const double *hi, int dim)
{
    for (int k = 0; k < dim; ++k) if (!(lo[k] <= hi[k])) return 1;
    return 0;
}

int port_boxes_intersect(int dim, const double *l, const double *r, int l_active, int r_active)
{
    if (!l_active && !r_active) return 0;
    for (int k = 0; k < dim; ++k) {
        double lo = l[0 * dim + k] < r[0 * dim + k] ? r[0 * dim + k] : l[0 * dim + k];
        double hi = r[1 * dim + k] < l[1 * dim + k] ? r[1 * dim + k] : l[1 * dim + k];
        if (!(lo <= hi)) return 0;
    }
    if (box_empty(l + 2 * dim, l + 3 * dim, dim) || box_empty(r + 2 * dim, r + 3 * dim, dim)) return 1;
    if (box_empty(l + 4 * dim, l + 5 * dim, dim) || box_empty(r + 4 * dim, r + 5 * dim, dim)) return 1;
    for (int k = 0; k < dim; ++k) {
        if ((l[2 * dim + k] > r[3 * dim + k] && l[4 * dim + k] > r[5 * dim + k]) ||
            (l[3 * dim + k] < r[2 * dim + k] && l[5 * dim + k] < r[4 * dim + k]))
            return 0;
    }
    return 1;
}

/* ---------------------------------------------------------------------- */
/* Leaf pairs.  The reference enumerates, via its Kd-BVH self-traversal      */
/* (BVHTree.cpp:129-302), every unordered pair of distinct leaves whose      */
/* boxes pass boxes_intersect, each exactly once; the set does not depend    */
/* on the tree.  Here: sort by swept min-x and sweep.  Output pairs are       */
/* canonical (lower primitive index first).  Returns the pair count; writes   */
/* at most cap pairs.                                                         */
/* ---------------------------------------------------------------------- */
static const double *g_sort_boxes;
static int g_sort_dim, g_sort_axis;
static int cmp_minx(const void *a, const void *b)
{
    int i = *(const int *)a, j = *(const int *)b;
    double x = g_sort_boxes[(size_t)i * 6 * g_sort_dim + g_sort_axis];
    double y = g_sort_boxes[(size_t)j * 6 * g_sort_dim + g_sort_axis];
    if (x < y) return -1;
    if (y < x) return 1;
    return (i > j) - (i < j);
}

long long port_leaf_pairs(int dim, const double *boxes, const unsigned char *flags, int np,
                          int *pairs, long long cap)
{
    int *ord = (int *)malloc(sizeof(int) * (size_t)(np > 0 ? np : 1));
    if (!ord) return -1;
    for (int i = 0; i < np; ++i) ord[i] = i;
    /* Sweep along the axis where boxes are shortest relative to the scene. */
    const size_t st = (size_t)6 * dim;
    int axis = 0;
    double best = -1;
    for (int k = 0; k < dim; ++k) {
        double lo = DBL_MAX, hi = -DBL_MAX, w = 0;
        for (int i = 0; i < np; ++i) {
            const double *b = boxes + i * st;
            if (b[k] < lo) lo = b[k];
            if (b[dim + k] > hi) hi = b[dim + k];
            w += b[dim + k] - b[k];
        }
        double ratio = (hi > lo) ? w / (hi - lo) : 1e300;
        if (best < 0 || ratio < best) { best = ratio; axis = k; }
    }
    g_sort_boxes = boxes; g_sort_dim = dim; g_sort_axis = axis;
    qsort(ord, (size_t)np, sizeof(int), cmp_minx);
    long long n = 0;
    for (int a = 0; a < np; ++a) {
        int i = ord[a];
        const double *bi = boxes + i * st;
        for (int c = a + 1; c < np; ++c) {
            int j = ord[c];
            const double *bj = boxes + j * st;
            if (bj[axis] > bi[dim + axis]) break; /* later boxes start beyond this one's end */
            int ai = flags ? (flags[i] & FLAG_ACTIVE) != 0 : 1;
            int aj = flags ? (flags[j] & FLAG_ACTIVE) != 0 : 1;
            if (!port_boxes_intersect(dim, bi, bj, ai, aj)) continue;
            if (n < cap) {
                pairs[2 * n] = i < j ? i : j;
                pairs[2 * n + 1] = i < j ? j : i;
            }
            ++n;
        }
    }
    free(ord);
    return n;
}

/* ---------------------------------------------------------------------- */
/* Candidate stencils: BVHTree.cpp:305-398 with p0 = pairs[2k] as "left".    */
/* VF [v, f1[0..dim-1]] (-1 padded), both directions; 3D EE                   */
/* [f0[i], f0[i+1], f1[j], f1[j+1]].  Skips unrepresented slots and any       */
/* shared vertex.  Returns the stencil count; writes at most cap.             */
/* ---------------------------------------------------------------------- */
long long port_candidates(int dim, const int *P, const unsigned char *flags, const int *pairs,
                          long long npairs, int *sten, unsigned char *is_vf, long long cap)
{
    long long n = 0;
#define EMIT(a, b, c, d, vf)                                                          \
    do {                                                                              \
        if (n < cap) { sten[4 * n] = (a); sten[4 * n + 1] = (b); sten[4 * n + 2] = (c); \
                       sten[4 * n + 3] = (d); is_vf[n] = (unsigned char)(vf); }        \
        ++n;                                                                          \
    } while (0)
    for (long long k = 0; k < npairs; ++k) {
        int p0 = pairs[2 * k], p1 = pairs[2 * k + 1];
        const int *f0 = P + (size_t)p0 * dim, *f1 = P + (size_t)p1 * dim;
        unsigned g0 = flags[p0], g1 = flags[p1];
        for (int i = 0; i < dim; ++i) {
            if (!(g0 & FLAG_V(i))) continue;
            int v = f0[i], shared = 0;
            for (int j = 0; j < dim; ++j) shared |= v == f1[j];
            if (shared) continue;
            EMIT(v, f1[0], f1[1], dim == 3 ? f1[2] : -1, 1);
        }
        for (int i = 0; i < dim; ++i) {
            if (!(g1 & FLAG_V(i))) continue;
            int v = f1[i], shared = 0;
            for (int j = 0; j < dim; ++j) shared |= v == f0[j];
            if (shared) continue;
            EMIT(v, f0[0], f0[1], dim == 3 ? f0[2] : -1, 1);
        }
        if (dim != 3) continue;
        for (int i = 0; i < 3; ++i) {
            if (!(g0 & FLAG_E(i))) continue;
            for (int j = 0; j < 3; ++j) {
                if (!(g1 & FLAG_E(j))) continue;
                int a = f0[i], b = f0[(i + 1) % 3], c = f1[j], d = f1[(j + 1) % 3];
                if (a == c || a == d || b == c || b == d) continue;
                EMIT(a, b, c, d, 0);
            }
        }
    }
#undef EMIT
    return n;
}

#include "port_dist.h"

/* NarrowPhase.cpp:714-750 pair_distance. x is (dim+1) points of dim coords. */
static double pair_distance(int dim, const double *x, int is_vf)
{
    if (dim == 2) return port_vf_distance2(x, x + 2, x + 4);
    if (is_vf) return port_vf_distance3(x, x + 3, x + 6, x + 9);
    return port_ee_distance3(x, x + 3, x + 6, x + 9);
}

/* ---------------------------------------------------------------------- */
/* ACCD: NarrowPhase.cpp:634-711 additive_ccd (s = 1, t_c = 1), exactly as   */
/* the reference runs it (toi = sum of the accepted steps).  Returns hit;     */
/* *toi is 0 for an immediate hit (d <= eta) and untouched on l_p <= 0.       */
/* ---------------------------------------------------------------------- */
int port_additive_ccd(int dim, const double *v0, const double *v1, double eta, int is_vf, double *toi, int *iters)
{
    const int ns = dim + 1;
    const double s = 1, xsi = eta, t_c = 1;
    double p[4 * 3], x[4 * 3], pbar[3] = {0, 0, 0};
    for (int i = 0; i < ns; ++i)
        for (int k = 0; k < dim; ++k) {
            p[i * dim + k] = v1[i * dim + k] - v0[i * dim + k];
            x[i * dim + k] = v0[i * dim + k];
            pbar[k] += (1.0 / (double)ns) * p[i * dim + k];
        }
    for (int i = 0; i < ns; ++i)
        for (int k = 0; k < dim; ++k) p[i * dim + k] -= pbar[k];
    double lf = 0, ls = 0;
    for (int i = 0; i < ns; ++i) {
        double sq = 0;
        for (int k = 0; k < dim; ++k) sq = (k == 0) ? p[i * dim] * p[i * dim] : sq + p[i * dim + k] * p[i * dim + k];
        double nrm = sqrt(sq);
        int first = is_vf ? i == 0 : i <= 1;
        if (first) lf = lf < nrm ? nrm : lf;
        else ls = ls < nrm ? nrm : ls;
    }
    double l_p = lf + ls;
    if (iters) *iters = -1;
    if (l_p <= 0) return 0;
    double d = pair_distance(dim, x, is_vf);
    double g = s * (d * d - xsi * xsi) / (d - xsi);
    *toi = 0;
    double t_l = (1 - s) * (d * d - xsi * xsi) / ((d + xsi) * l_p);
    if (d <= xsi) { if (iters) *iters = 0; return 1; }
    int iter = 0;
    for (; iter < 1000; ++iter) {
        for (int i = 0; i < ns * dim; ++i) x[i] = x[i] + t_l * p[i];
        d = pair_distance(dim, x, is_vf);
        double eps = (d * d - xsi * xsi) / (d + xsi);
        if (*toi > 0 && iter > 0 && eps < g) break;
        *toi += t_l;
        if (*toi > t_c) { if (iters) *iters = iter; return 0; }
        t_l = 0.9 * (d * d - xsi * xsi) / ((d + xsi) * l_p);
    }
    if (iters) *iters = iter;
    return 1;
}

/* default_narrow_phase (BVHTree.cpp:429-461) over a stencil list: gather    */
/* 2 x (dim+1) vertices, run ACCD, toi if hit==1 else -1.                     */
void port_accd(int dim, const double *V0, const double *V1, const int *sten, const unsigned char *is_vf,
               long long n, double vf_eta, double ee_eta, int *hit, double *toi, int *iters)
{
    for (long long s = 0; s < n; ++s) {
        double a[4 * 3], b[4 * 3];
        for (int i = 0; i < dim + 1; ++i)
            for (int k = 0; k < dim; ++k) {
                a[i * dim + k] = V0[(size_t)sten[4 * s + i] * dim + k];
                b[i * dim + k] = V1[(size_t)sten[4 * s + i] * dim + k];
            }
        double t = -1;
        int h = port_additive_ccd(dim, a, b, is_vf[s] ? vf_eta : ee_eta, is_vf[s], &t, iters ? iters + s : NULL);
        hit[s] = h;
        toi[s] = h ? t : -1.0;
    }
}

/* ---------------------------------------------------------------------- */
/* Discrete triangle-triangle overlap (Guigue & Devillers, "Fast and Robust  */
/* Triangle-Triangle Overlap Test Using Orientation Predicates", JGT 2003),   */
/* as the reference evaluates it in tt_isect.hpp:141-284 and 553-589: same    */
/* predicates, same vertex permutations, exact zero tests.                    */
/* ---------------------------------------------------------------------- */
typedef const double *cpt;

static void sub3(double *o, cpt a, cpt b) { o[0] = a[0] - b[0]; o[1] = a[1] - b[1]; o[2] = a[2] - b[2]; }
static void cross3(double *o, const double *a, const double *b)
{
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}
static double orient2(cpt a, cpt b, cpt c) { return (a[0] - c[0]) * (b[1] - c[1]) - (a[1] - c[1]) * (b[0] - c[0]); }

/* Vertex of T1 in the region of a vertex of T2 (2D). */
static int tt2_vertex(cpt P1, cpt Q1, cpt R1, cpt P2, cpt Q2, cpt R2)
{
    if (orient2(R2, P2, Q1) >= 0) {
        if (orient2(R2, Q2, Q1) <= 0) {
            if (orient2(P1, P2, Q1) > 0) return orient2(P1, Q2, Q1) <= 0;
            if (orient2(P1, P2, R1) >= 0) return orient2(Q1, R1, P2) >= 0;
            return 0;
        }
        if (orient2(P1, Q2, Q1) <= 0) {
            if (orient2(R2, Q2, R1) <= 0) return orient2(Q1, R1, Q2) >= 0;
            return 0;
        }
        return 0;
    }
    if (orient2(R2, P2, R1) >= 0) {
        if (orient2(Q1, R1, R2) >= 0) return orient2(P1, P2, R1) >= 0;
        if (orient2(Q1, R1, Q2) >= 0) return orient2(R2, R1, Q2) >= 0;
        return 0;
    }
    return 0;
}

/* Vertex of T1 in the region of an edge of T2 (2D). */
static int tt2_edge(cpt P1, cpt Q1, cpt R1, cpt P2, cpt Q2, cpt R2)
{
    (void)Q2;
    if (orient2(R2, P2, Q1) >= 0) {
        if (orient2(P1, P2, Q1) >= 0) return orient2(P1, Q1, R2) >= 0;
        if (orient2(Q1, R1, P2) >= 0) return orient2(R1, P1, P2) >= 0;
        return 0;
    }
    if (orient2(R2, P2, R1) >= 0) {
        if (orient2(P1, P2, R1) >= 0) {
            if (orient2(P1, R1, R2) >= 0) return 1;
            return orient2(Q1, R1, R2) >= 0;
        }
        return 0;
    }
    return 0;
}

static int tt2_ccw(cpt p1, cpt q1, cpt r1, cpt p2, cpt q2, cpt r2)
{
    if (orient2(p2, q2, p1) >= 0) {
        if (orient2(q2, r2, p1) >= 0) {
            if (orient2(r2, p2, p1) >= 0) return 1;
            return tt2_edge(p1, q1, r1, p2, q2, r2);
        }
        if (orient2(r2, p2, p1) >= 0) return tt2_edge(p1, q1, r1, r2, p2, q2);
        return tt2_vertex(p1, q1, r1, p2, q2, r2);
    }
    if (orient2(q2, r2, p1) >= 0) {
        if (orient2(r2, p2, p1) >= 0) return tt2_edge(p1, q1, r1, q2, r2, p2);
        return tt2_vertex(p1, q1, r1, q2, r2, p2);
    }
    return tt2_vertex(p1, q1, r1, r2, p2, q2);
}

static int tt2_overlap(cpt p1, cpt q1, cpt r1, cpt p2, cpt q2, cpt r2)
{
    int a = orient2(p1, q1, r1) < 0, b = orient2(p2, q2, r2) < 0;
    cpt Q1 = a ? r1 : q1, R1 = a ? q1 : r1, Q2 = b ? r2 : q2, R2 = b ? q2 : r2;
    return tt2_ccw(p1, Q1, R1, p2, Q2, R2);
}

/* Coplanar case: project both triangles on the axis plane that maximises    */
/* the area of T1 (normal n1) and run the 2D test.                           */
static int tt3_coplanar(cpt p1, cpt q1, cpt r1, cpt p2, cpt q2, cpt r2, const double *n1)
{
    double nx = n1[0] < 0 ? -n1[0] : n1[0], ny = n1[1] < 0 ? -n1[1] : n1[1], nz = n1[2] < 0 ? -n1[2] : n1[2];
    double P1[2], Q1[2], R1[2], P2[2], Q2[2], R2[2];
    int u, v, swap;
    if (nx > nz && nx >= ny) { u = 2; v = 1; swap = 1; }
    else if (ny > nz && ny >= nx) { u = 0; v = 2; swap = 1; }
    else { u = 0; v = 1; swap = 0; }
    /* For the x- and y-dominant projections the reference also exchanges the
     * roles of p and q (keeps the projected orientation consistent). */
    cpt a1 = swap ? q1 : p1, b1 = swap ? p1 : q1, a2 = swap ? q2 : p2, b2 = swap ? p2 : q2;
    P1[0] = a1[u]; P1[1] = a1[v]; Q1[0] = b1[u]; Q1[1] = b1[v]; R1[0] = r1[u]; R1[1] = r1[v];
    P2[0] = a2[u]; P2[1] = a2[v]; Q2[0] = b2[u]; Q2[1] = b2[v]; R2[0] = r2[u]; R2[1] = r2[v];
    return tt2_overlap(P1, Q1, R1, P2, Q2, R2);
}

/* Final interval check once p1 (resp. p2) is alone on its side. */
static int tt3_minmax(cpt p1, cpt q1, cpt r1, cpt p2, cpt q2, cpt r2)
{
    double a[3], b[3], n[3];
    sub3(a, p2, q1); sub3(b, p1, q1); cross3(n, a, b);
    sub3(a, q2, q1);
    if (dot3(a, n) > 0) return 0;
    sub3(a, p2, p1); sub3(b, r1, p1); cross3(n, a, b);
    sub3(a, r2, p1);
    return dot3(a, n) > 0 ? 0 : 1;
}

/* Sign pattern -> (rotation of the first triangle, swap of the second).
 * rot 0: (p,q,r), 1: (q,r,p), 2: (r,p,q); swap: exchange q and r of the other
 * triangle (and its two distances).  Returns 0 when all three are zero.  */
static int tt3_canon(double dp, double dq, double dr, int *rot, int *swap)
{
    if (dp > 0) {
        if (dq > 0) { *rot = 2; *swap = 1; }
        else if (dr > 0) { *rot = 1; *swap = 1; }
        else { *rot = 0; *swap = 0; }
    } else if (dp < 0) {
        if (dq < 0) { *rot = 2; *swap = 0; }
        else if (dr < 0) { *rot = 1; *swap = 0; }
        else { *rot = 0; *swap = 1; }
    } else {
        if (dq < 0) {
            if (dr >= 0) { *rot = 1; *swap = 1; }
            else { *rot = 0; *swap = 0; }
        } else if (dq > 0) {
            if (dr > 0) { *rot = 0; *swap = 1; }
            else { *rot = 1; *swap = 0; }
        } else {
            if (dr > 0) { *rot = 2; *swap = 0; }
            else if (dr < 0) { *rot = 2; *swap = 1; }
            else return 0;
        }
    }
    return 1;
}

int port_tri_tri(cpt p1, cpt q1, cpt r1, cpt p2, cpt q2, cpt r2)
{
    double a[3], b[3], n1[3], n2[3];
    sub3(a, p2, r2); sub3(b, q2, r2); cross3(n2, a, b);
    sub3(a, p1, r2); double dp1 = dot3(a, n2);
    sub3(a, q1, r2); double dq1 = dot3(a, n2);
    sub3(a, r1, r2); double dr1 = dot3(a, n2);
    if (dp1 * dq1 > 0 && dp1 * dr1 > 0) return 0;
    sub3(a, q1, p1); sub3(b, r1, p1); cross3(n1, a, b);
    sub3(a, p2, r1); double dp2 = dot3(a, n1);
    sub3(a, q2, r1); double dq2 = dot3(a, n1);
    sub3(a, r2, r1); double dr2 = dot3(a, n1);
    if (dp2 * dq2 > 0 && dp2 * dr2 > 0) return 0;

    int rot1, sw2;
    if (!tt3_canon(dp1, dq1, dr1, &rot1, &sw2)) return tt3_coplanar(p1, q1, r1, p2, q2, r2, n1);
    cpt t1[3] = {p1, q1, r1};
    cpt A1 = t1[rot1 % 3], B1 = t1[(rot1 + 1) % 3], C1 = t1[(rot1 + 2) % 3];
    cpt A2 = p2, B2 = sw2 ? r2 : q2, C2 = sw2 ? q2 : r2;
    double da = dp2, db = sw2 ? dr2 : dq2, dc = sw2 ? dq2 : dr2;

    int rot2, sw1;
    if (!tt3_canon(da, db, dc, &rot2, &sw1)) return tt3_coplanar(A1, B1, C1, A2, B2, C2, n1);
    cpt t2[3] = {A2, B2, C2};
    cpt X2 = t2[rot2 % 3], Y2 = t2[(rot2 + 1) % 3], Z2 = t2[(rot2 + 2) % 3];
    cpt Y1 = sw1 ? C1 : B1, Z1 = sw1 ? B1 : C1;
    return tt3_minmax(A1, Y1, Z1, X2, Y2, Z2);
}

/* NarrowPhase.cpp:229-257 discrete_edge_edge (2D segments). */
int port_seg_seg(cpt p0, cpt p1, cpt q0, cpt q1)
{
    const double eps = DBL_EPSILON;
    double n[2] = {q0[0] - p0[0], q0[1] - p0[1]};
    double r[2] = {p1[0] - p0[0], p1[1] - p0[1]};
    double s[2] = {q1[0] - q0[0], q1[1] - q0[1]};
    double rxs = r[0] * s[1] - r[1] * s[0];
    if (fabs(rxs) < eps) return 0;
    double nxr = n[0] * r[1] - n[1] * r[0];
    if (fabs(nxr) < eps)
        return ((q0[0] - p0[0] < 0) != (q0[0] - p1[0] < 0)) || ((q0[1] - p0[1] < 0) != (q0[1] - p1[1] < 0));
    double nxs = n[0] * s[1] - n[1] * s[0];
    double inv = 1.0 / rxs;
    double t = nxs * inv, u = nxr * inv;
    return (t >= 0) && (t <= 1) && (u >= 0) && (u <= 1);
}

/* default_discrete_test (BVHTree.cpp:464-500) on V over leaf pairs: reject a */
/* shared vertex, then tri-tri (3D) or segment test (2D) with p0 first.       */
void port_discrete(int dim, const double *V, const int *P, const int *pairs, long long n, int *out)
{
    for (long long k = 0; k < n; ++k) {
        const int *f0 = P + (size_t)pairs[2 * k] * dim, *f1 = P + (size_t)pairs[2 * k + 1] * dim;
        int shared = 0;
        for (int i = 0; i < dim; ++i) for (int j = 0; j < dim; ++j) shared |= f0[i] == f1[j];
        if (shared) { out[k] = 0; continue; }
        if (dim == 3)
            out[k] = port_tri_tri(V + (size_t)f0[0] * 3, V + (size_t)f0[1] * 3, V + (size_t)f0[2] * 3,
                                  V + (size_t)f1[0] * 3, V + (size_t)f1[1] * 3, V + (size_t)f1[2] * 3);
        else
            out[k] = port_seg_seg(V + (size_t)f0[0] * 2, V + (size_t)f0[1] * 2, V + (size_t)f1[0] * 2, V + (size_t)f1[1] * 2);
    }
}
