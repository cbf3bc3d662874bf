// Exact FP64 geometry of the CCD path, as device functions.
//
// Every expression is evaluated in the order mclccd evaluates it, and every
// translation unit that includes this header is compiled with -fmad=false,
// so each result is bit-identical to the reference's x86-64 build (IEEE
// double add/mul/div/sqrt, no contraction, left-to-right reductions).
#pragma once

#include "common.cuh"

#include <cmath>

namespace mclccd {

// ---------------------------------------------------------------------------
// Leaf box predicate: BVHTree::boxes_intersect (BVHTree.cpp:401-426) on two
// leaves.  Closed-interval swept-box overlap, then per-axis rejection when the
// t0 boxes and the t1 boxes are separated on the same side.  The reference's
// "t0/t1 box empty" early-outs (BVHTree.cpp:415-416) never fire for leaves:
// a leaf box is the padded hull of >= 1 point.
// ---------------------------------------------------------------------------
template <int DIM>
__device__ __forceinline__ bool leaf_boxes_intersect(const LeafBox<DIM> &l, const LeafBox<DIM> &r)
{
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
        double lmin = l.lo0[k] < l.lo1[k] ? l.lo0[k] : l.lo1[k];
        double lmax = l.hi0[k] < l.hi1[k] ? l.hi1[k] : l.hi0[k];
        double rmin = r.lo0[k] < r.lo1[k] ? r.lo0[k] : r.lo1[k];
        double rmax = r.hi0[k] < r.hi1[k] ? r.hi1[k] : r.hi0[k];
        double lo = lmin < rmin ? rmin : lmin;
        double hi = rmax < lmax ? rmax : lmax;
        if (!(lo <= hi)) return false;
    }
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
        if ((l.lo0[k] > r.hi0[k] && l.lo1[k] > r.hi1[k]) || (l.hi0[k] < r.lo0[k] && l.hi1[k] < r.lo1[k]))
            return false;
    }
    return true;
}

// ---------------------------------------------------------------------------
// Distances (Projection.hpp).
//
// Each routine keeps the reference's case analysis and expressions, but the
// quotient a case needs is selected first and divided once: every case of
// point_on_triangle takes exactly one quotient (num / den), edge_to_edge at
// most two.  The same IEEE operations run on the same operands, so the
// results are the reference's bit for bit, while the lanes of a warp that
// fall into different cases share one division instead of taking each
// case's in turn.  Host-callable too, so the CPU tests can run this code.
// ---------------------------------------------------------------------------
MC_HD double dot3(const double *a, const double *b)
{
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}
MC_HD double clamp_zero_one(double v) { return v < 0 ? 0.0 : (v > 1 ? 1.0 : v); }
// std::min(T(1), std::max(x, T(0))) as the reference writes it.
MC_HD double clamp01(double x)
{
    double m = x < 0 ? 0.0 : x;
    return m < 1 ? m : 1.0;
}

// Distance from pt to triangle (p1,p2,p3): point_on_triangle
// (Projection.hpp:61-145) then (pt - closest).norm().  Cases, by the
// quotient q = num / den they take:
//   interior:               q = 1 / det,  s = s0 q, t = t0 q
//   s = clamp(q), t = 0:    q = -d / a  (Projection.hpp region 4 / 5), or
//                           q = -e / c  (the branch s >= 0, t < 0, s+t >= det,
//                                        a+d <= b+e, which the reference
//                                        writes as s = clamp(-e/c), t = 0)
//   s = 0, t = clamp(q):    q = -e / c
//   s = clamp(q), t = 1-s:  q = (c+e) - (b+d) over (a - 2b) + c  (region 2), or
//                           q = ((c+e) - b) - d over the same   (regions 6, 1)
MC_HD double vf_distance3(const double *pt, const double *p1, const double *p2, const double *p3)
{
    double e0[3], e1[3], v0[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) { e0[k] = p2[k] - p1[k]; e1[k] = p3[k] - p1[k]; v0[k] = p1[k] - pt[k]; }
    const double a = dot3(e0, e0), b = dot3(e0, e1), c = dot3(e1, e1), d = dot3(e0, v0), e = dot3(e1, v0);
    const double det = a * c - b * b;
    const double s0 = b * e - c * d, t0 = b * d - a * e;
    enum { kInterior, kSOnly, kTOnly, kEdge12 };
    double num, den;
    int kind;
    if (s0 + t0 < det) {
        if (s0 < 0) {
            if (t0 < 0 && d < 0) { num = -d; den = a; kind = kSOnly; }
            else { num = -e; den = c; kind = kTOnly; }
        } else if (t0 < 0) { num = -d; den = a; kind = kSOnly; }
        else { num = 1.0; den = det; kind = kInterior; }
    } else {
        const double den12 = a - 2.0 * b + c;
        if (s0 < 0) {
            const double tt0 = b + d, tt1 = c + e;
            if (tt1 > tt0) { num = tt1 - tt0; den = den12; kind = kEdge12; }
            else { num = -e; den = c; kind = kTOnly; }
        } else if (t0 < 0) {
            if (a + d > b + e) { num = c + e - b - d; den = den12; kind = kEdge12; }
            else { num = -e; den = c; kind = kSOnly; }
        } else { num = c + e - b - d; den = den12; kind = kEdge12; }
    }
    const double q = num / den;
    const double cq = clamp_zero_one(q);
    double s, t;
    if (kind == kInterior) { s = s0 * q; t = t0 * q; }
    else if (kind == kSOnly) { s = cq; t = 0.0; }
    else if (kind == kTOnly) { s = 0.0; t = cq; }
    else { s = cq; t = 1 - cq; }
    double r[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) r[k] = pt[k] - ((p1[k] + e0[k] * s) + e1[k] * t);
    return sqrt(dot3(r, r));
}

// Segment-segment distance: edge_to_edge (Projection.hpp:242-302), .norm().
// First quotient s = clamp((bf - ce) / denom) (unused when denom == 0), then
// one of -c / a, (b - c) / a (s re-clamped, t = 0 or 1) or t = tnom / e.
MC_HD double ee_distance3(const double *p0, const double *p1, const double *q0, const double *q1)
{
    double d1[3], d2[3], r[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) { d1[k] = p1[k] - p0[k]; d2[k] = q1[k] - q0[k]; r[k] = p0[k] - q0[k]; }
    const double a = dot3(d1, d1), e = dot3(d2, d2), f = dot3(d2, r);
    const double c = dot3(d1, r), b = dot3(d1, d2);
    const double denom = a * e - b * b;
    const double q1s = (b * f - c * e) / denom;
    double s = denom != 0 ? clamp01(q1s) : 0.0;
    const double tnom = b * s + f;
    double num, den, t;
    int kind;   // 0: t = 0, 1: t = 1 (s from q), 2: t = q
    if (tnom < 0 || e == 0) { num = -c; den = a; kind = 0; }
    else if (tnom > e) { num = b - c; den = a; kind = 1; }
    else { num = tnom; den = e; kind = 2; }
    const double q = num / den;
    if (kind == 2) t = q;
    else { t = kind == 0 ? 0.0 : 1.0; s = (a == 0) ? 0.0 : clamp01(q); }
    double w[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) w[k] = (q0[k] + t * d2[k]) - (p0[k] + s * d1[k]);
    return sqrt(dot3(w, w));
}

// Point-segment distance in 2D: point_on_edge (Projection.hpp:194-204).
MC_HD double vf_distance2(const double *p, const double *e0, const double *e1)
{
    const double e[2] = {e1[0] - e0[0], e1[1] - e0[1]};
    const double len2 = e[0] * e[0] + e[1] * e[1];
    const double t = ((p[0] - e0[0]) * e[0] + (p[1] - e0[1]) * e[1]) / len2;   // unused when len2 <= 0
    double q0, q1;
    if (len2 <= 0.0 || t < 0.0) { q0 = e0[0]; q1 = e0[1]; }
    else if (t > 1.0) { q0 = e1[0]; q1 = e1[1]; }
    else { q0 = e0[0] + t * e[0]; q1 = e0[1] + t * e[1]; }
    const double w0 = p[0] - q0, w1 = p[1] - q1;
    return sqrt(w0 * w0 + w1 * w1);
}

// NarrowPhaseACCD::pair_distance (NarrowPhase.cpp:714-750).
template <int DIM, bool VF>
MC_HD double pair_distance(const double (&x)[DIM + 1][DIM])
{
    if constexpr (DIM == 2) return vf_distance2(x[0], x[1], x[2]);
    else if constexpr (VF) return vf_distance3(x[0], x[1], x[2], x[3]);
    else return ee_distance3(x[0], x[1], x[2], x[3]);
}

// ---------------------------------------------------------------------------
// ACCD: NarrowPhaseACCD::additive_ccd (NarrowPhase.cpp:634-711) with s = 1 and
// t_c = 1, giving bit-identical (hit, toi).  Two evaluations whose results the
// reference never uses are skipped: the distance at loop iteration 0 (the
// step is 0, so x and d are unchanged when the motion is finite) and the
// distance at any iteration where no break is possible (toi == 0) and the
// accumulated toi already exceeds 1 (the reference returns "miss" right after
// computing it).  Returns 1 on hit; toi is the sum of accepted steps.
// (The iteration-0 skip is taken only when it cannot change a single bit.)
// iters receives the loop index at exit (0 for an immediate hit).
//
// The work is split into setup / head / tail so that other forms (the FP32
// certified pass) can share the exact FP64 pieces.
// ---------------------------------------------------------------------------

// Relative motion p_i = (v1_i - v0_i) - mean, start positions x = v0 and --
// when WANT_LP -- l_p = max first |p| + max second |p| (NarrowPhase.cpp:647-670).
// step0_noop: x + 0 * p == x bit for bit (every p finite, no x is -0.0, the
// only value whose bits change: -0.0 + 0.0 == +0.0).
// l_p is formed from the squared norms: sqrt is correctly rounded and
// monotone, so the larger of two square roots is the square root of the
// larger square (ties and NaN behave the same), which takes two square
// roots per stencil instead of DIM + 1.
template <int DIM, bool VF, bool WANT_LP>
MC_HD void accd_setup(const double (&v0)[DIM + 1][DIM], const double (&v1)[DIM + 1][DIM],
                      double (&p)[DIM + 1][DIM], double (&x)[DIM + 1][DIM], double &l_p, bool &step0_noop)
{
    constexpr int ns = DIM + 1;
    double pbar[DIM];
#pragma unroll
    for (int k = 0; k < DIM; ++k) pbar[k] = 0.0;
    const double w = 1.0 / (double)ns;
    step0_noop = true;
#pragma unroll
    for (int i = 0; i < ns; ++i)
#pragma unroll
        for (int k = 0; k < DIM; ++k) {
            p[i][k] = v1[i][k] - v0[i][k];
            x[i][k] = v0[i][k];
            pbar[k] = pbar[k] + w * p[i][k];
        }
    double lf2 = 0.0, ls2 = 0.0;
#pragma unroll
    for (int i = 0; i < ns; ++i) {
        double sq = 0.0;
#pragma unroll
        for (int k = 0; k < DIM; ++k) {
            p[i][k] = p[i][k] - pbar[k];
            sq = (k == 0) ? p[i][k] * p[i][k] : sq + p[i][k] * p[i][k];
            step0_noop = step0_noop && isfinite(p[i][k]) && !(x[i][k] == 0.0 && signbit(x[i][k]));
        }
        if constexpr (WANT_LP) {
            const bool first = VF ? (i == 0) : (i <= 1);
            if (first) lf2 = lf2 < sq ? sq : lf2;
            else ls2 = ls2 < sq ? sq : ls2;
        }
    }
    if constexpr (WANT_LP) l_p = sqrt(lf2) + sqrt(ls2);
}

// Iterations 1..999 of the reference loop, from the state after iteration 0
// (positions x, accumulated toi, next step t_l, threshold g).
template <int DIM, bool VF>
MC_HD int accd_tail(double (&x)[DIM + 1][DIM], const double (&p)[DIM + 1][DIM], double l_p, double xsi, double g,
                    double &toi, double t_l, int &iters)
{
    constexpr int ns = DIM + 1;
    const double xx = xsi * xsi;
    for (int iter = 1; iter < 1000; ++iter) {
        const bool can_break = toi > 0;
        if (!can_break && toi + t_l > 1.0) { toi = toi + t_l; iters = iter; return 0; }
#pragma unroll
        for (int i = 0; i < ns; ++i)
#pragma unroll
            for (int k = 0; k < DIM; ++k) x[i][k] = x[i][k] + t_l * p[i][k];
        const double d = pair_distance<DIM, VF>(x);
        const double A = d * d - xx;
        if (can_break && A / (d + xsi) < g) { iters = iter; return 1; }
        toi = toi + t_l;
        if (toi > 1.0) { iters = iter; return 0; }
        t_l = 0.9 * A / ((d + xsi) * l_p);
    }
    iters = 1000;
    return 1;
}

// Outcome of ACCD's head (everything before iteration 1).
enum AccdHead { kHeadMiss = 0, kHeadHit = 1, kHeadContinue = 2, kHeadLiteral = 3 };

// Head: l_p test, first distance, immediate hit, iteration 0, and the miss
// that iteration 1 would report before its distance is used.  On
// kHeadContinue, (x, toi, t_l, g) is the state entering iteration 1; d0 is
// the first distance.  exact_skip tells whether iteration 0 was skipped
// (then x == v0, toi == 0 and t_l is a function of d0 and l_p alone).
template <int DIM, bool VF>
MC_HD int accd_head(double (&x)[DIM + 1][DIM], const double (&p)[DIM + 1][DIM], double l_p, bool step0_noop,
                    double xsi, double &d0, double &g, double &toi, double &t_l, bool &exact_skip)
{
    constexpr int ns = DIM + 1;
    exact_skip = false;
    if (l_p <= 0) return kHeadMiss;
    double d = pair_distance<DIM, VF>(x);
    d0 = d;
    const double xx = xsi * xsi;
    double A = d * d - xx;
    g = (1.0 * A) / (d - xsi);
    toi = 0.0;
    t_l = ((1.0 - 1.0) * A) / ((d + xsi) * l_p);
    if (d <= xsi) return kHeadHit;
    exact_skip = t_l == 0.0 && step0_noop;
    if (!exact_skip) {   // iteration 0, literally
#pragma unroll
        for (int i = 0; i < ns; ++i)
#pragma unroll
            for (int k = 0; k < DIM; ++k) x[i][k] = x[i][k] + t_l * p[i][k];
        d = pair_distance<DIM, VF>(x);
        A = d * d - xx;
    }
    toi = toi + t_l;
    if (toi > 1.0) return kHeadMiss;
    t_l = 0.9 * A / ((d + xsi) * l_p);
    if (!(toi > 0) && toi + t_l > 1.0) return kHeadMiss;   // iteration 1 returns "miss"
    return kHeadContinue;
}

// The same head with the work the outcome does not need left out: the
// threshold g (used from iteration 2 on) is not formed, and iteration 0's
// step ((1 - 1) A) / X is not divided out when it is certainly zero (A
// finite, X neither zero nor NaN), which is exactly when the reference's
// step is +-0.  Outcomes: kHeadMiss, kHeadHit (toi = 0), kHeadContinue (the
// state entering iteration 1 is x = v0, toi = 0, t_l = t_l1, and g follows
// from d0: accd_resume) or kHeadLiteral (iteration 0 is not an exact no-op:
// run the literal accd).
template <int DIM, bool VF>
MC_HD int accd_head_fast(const double (&x)[DIM + 1][DIM], double l_p, bool step0_noop, double xsi, double &d0,
                         double &t_l1)
{
    if (l_p <= 0) return kHeadMiss;
    const double d = pair_distance<DIM, VF>(x);
    d0 = d;
    const double A = d * d - xsi * xsi;
    const double X = (d + xsi) * l_p;
    if (d <= xsi) return kHeadHit;
    const bool zero_step = isfinite(A) && X == X && X != 0.0;
    if (!(zero_step && step0_noop)) return kHeadLiteral;
    t_l1 = 0.9 * A / X;
    return t_l1 > 1.0 ? kHeadMiss : kHeadContinue;   // 0 + t_l1 > 1 at iteration 1
}

// Iterations 1.. for a stencil whose fast head said kHeadContinue: x holds
// v0 and p the relative motion (accd_setup), d0 the first distance.
template <int DIM, bool VF>
MC_HD int accd_resume(double (&x)[DIM + 1][DIM], const double (&p)[DIM + 1][DIM], double l_p, double xsi, double d0,
                      double &toi, int &iters)
{
    const double A = d0 * d0 - xsi * xsi;
    const double g = (1.0 * A) / (d0 - xsi);
    toi = 0.0;
    return accd_tail<DIM, VF>(x, p, l_p, xsi, g, toi, 0.9 * A / ((d0 + xsi) * l_p), iters);
}

template <int DIM, bool VF>
MC_HD int accd_literal(const double (&v0)[DIM + 1][DIM], const double (&v1)[DIM + 1][DIM], double xsi, double &toi,
                       int &iters)
{
    constexpr int ns = DIM + 1;
    double p[ns][DIM], x[ns][DIM], l_p, d0, g, t_l;
    bool noop, skip;
    accd_setup<DIM, VF, true>(v0, v1, p, x, l_p, noop);
    iters = -1;
    const int h = accd_head<DIM, VF>(x, p, l_p, noop, xsi, d0, g, toi, t_l, skip);
    if (h == kHeadHit) { iters = 0; return 1; }
    if (h == kHeadMiss) { iters = l_p <= 0 ? -1 : 0; return 0; }
    return accd_tail<DIM, VF>(x, p, l_p, xsi, g, toi, t_l, iters);
}

template <int DIM, bool VF>
MC_HD int accd(const double (&v0)[DIM + 1][DIM], const double (&v1)[DIM + 1][DIM], double xsi, double &toi,
               int &iters)
{
    constexpr int ns = DIM + 1;
    double p[ns][DIM], x[ns][DIM], l_p, d0, t_l1;
    bool noop;
    accd_setup<DIM, VF, true>(v0, v1, p, x, l_p, noop);
    const int h = accd_head_fast<DIM, VF>(x, l_p, noop, xsi, d0, t_l1);
    if (h == kHeadHit) { toi = 0.0; iters = 0; return 1; }
    if (h == kHeadMiss) { iters = l_p <= 0 ? -1 : 0; return 0; }
    if (h == kHeadLiteral) return accd_literal<DIM, VF>(v0, v1, xsi, toi, iters);
    return accd_resume<DIM, VF>(x, p, l_p, xsi, d0, toi, iters);
}

// ---------------------------------------------------------------------------
// Discrete triangle-triangle overlap at V1: the Guigue-Devillers orientation
// test ("Fast and Robust Triangle-Triangle Overlap Test Using Orientation
// Predicates", JGT 2003) evaluated as tt_isect.hpp:141-284,553-589 does
// (same predicates, same vertex permutations, exact zero tests).
// ---------------------------------------------------------------------------
typedef const double *cpt;

__device__ __forceinline__ void sub3(double *o, cpt a, cpt b) { o[0] = a[0] - b[0]; o[1] = a[1] - b[1]; o[2] = a[2] - b[2]; }
__device__ __forceinline__ void cross3(double *o, const double *a, const double *b)
{
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}
__device__ __forceinline__ double orient2(cpt a, cpt b, cpt c)
{
    return (a[0] - c[0]) * (b[1] - c[1]) - (a[1] - c[1]) * (b[0] - c[0]);
}

static __device__ __noinline__ int tt2_vertex(cpt P1, cpt Q1, cpt R1, cpt P2, cpt Q2, cpt R2)
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

static __device__ __noinline__ int tt2_edge(cpt P1, cpt Q1, cpt R1, cpt P2, cpt R2)
{
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

static __device__ __noinline__ int tt2_overlap(cpt p1, cpt q1_, cpt r1_, cpt p2, cpt q2_, cpt r2_)
{
    const bool a = orient2(p1, q1_, r1_) < 0, b = orient2(p2, q2_, r2_) < 0;
    cpt q1 = a ? r1_ : q1_, r1 = a ? q1_ : r1_, q2 = b ? r2_ : q2_, r2 = b ? q2_ : r2_;
    if (orient2(p2, q2, p1) >= 0) {
        if (orient2(q2, r2, p1) >= 0) {
            if (orient2(r2, p2, p1) >= 0) return 1;
            return tt2_edge(p1, q1, r1, p2, r2);
        }
        if (orient2(r2, p2, p1) >= 0) return tt2_edge(p1, q1, r1, r2, q2);
        return tt2_vertex(p1, q1, r1, p2, q2, r2);
    }
    if (orient2(q2, r2, p1) >= 0) {
        if (orient2(r2, p2, p1) >= 0) return tt2_edge(p1, q1, r1, q2, p2);
        return tt2_vertex(p1, q1, r1, q2, r2, p2);
    }
    return tt2_vertex(p1, q1, r1, r2, p2, q2);
}

// Coplanar case: project on the axis plane maximising T1's area (normal n1);
// for the x- and y-dominant planes the reference also exchanges p and q.
// The six vertices come by value (rows p1 q1 r1 p2 q2 r2), so the callers'
// copies can stay in registers on the common path.
struct TriPair {
    double v[6][3];
    double n[3];
};
static __device__ __noinline__ int tt3_coplanar(const TriPair t)
{
    const double *p1 = t.v[0], *q1 = t.v[1], *r1 = t.v[2], *p2 = t.v[3], *q2 = t.v[4], *r2 = t.v[5];
    const double *n1 = t.n;
    const double nx = n1[0] < 0 ? -n1[0] : n1[0], ny = n1[1] < 0 ? -n1[1] : n1[1], nz = n1[2] < 0 ? -n1[2] : n1[2];
    int u, v;
    bool sw;
    if (nx > nz && nx >= ny) { u = 2; v = 1; sw = true; }
    else if (ny > nz && ny >= nx) { u = 0; v = 2; sw = true; }
    else { u = 0; v = 1; sw = false; }
    cpt a1 = sw ? q1 : p1, b1 = sw ? p1 : q1, a2 = sw ? q2 : p2, b2 = sw ? p2 : q2;
    const double P1[2] = {a1[u], a1[v]}, Q1[2] = {b1[u], b1[v]}, R1[2] = {r1[u], r1[v]};
    const double P2[2] = {a2[u], a2[v]}, Q2[2] = {b2[u], b2[v]}, R2[2] = {r2[u], r2[v]};
    return tt2_overlap(P1, Q1, R1, P2, Q2, R2);
}

__device__ __forceinline__ int tt3_minmax(cpt p1, cpt q1, cpt r1, cpt p2, cpt q2, cpt r2)
{
    double a[3], b[3], n[3];
    sub3(a, p2, q1); sub3(b, p1, q1); cross3(n, a, b);
    sub3(a, q2, q1);
    if (dot3(a, n) > 0) return 0;
    sub3(a, p2, p1); sub3(b, r1, p1); cross3(n, a, b);
    sub3(a, r2, p1);
    return dot3(a, n) > 0 ? 0 : 1;
}

// Sign pattern of (dp,dq,dr) -> rotation of the first triangle (0:(p,q,r)
// 1:(q,r,p) 2:(r,p,q)) and whether the other triangle's q and r swap.
// False when all three distances are zero (coplanar).
__device__ __forceinline__ bool tt3_canon(double dp, double dq, double dr, int &rot, bool &swap)
{
    if (dp > 0) {
        if (dq > 0) { rot = 2; swap = true; }
        else if (dr > 0) { rot = 1; swap = true; }
        else { rot = 0; swap = false; }
    } else if (dp < 0) {
        if (dq < 0) { rot = 2; swap = false; }
        else if (dr < 0) { rot = 1; swap = false; }
        else { rot = 0; swap = true; }
    } else {
        if (dq < 0) {
            if (dr >= 0) { rot = 1; swap = true; }
            else { rot = 0; swap = false; }
        } else if (dq > 0) {
            if (dr > 0) { rot = 0; swap = true; }
            else { rot = 1; swap = false; }
        } else {
            if (dr > 0) { rot = 2; swap = false; }
            else if (dr < 0) { rot = 2; swap = true; }
            else return false;
        }
    }
    return true;
}

__device__ __forceinline__ TriPair tri_pair(cpt p1, cpt q1, cpt r1, cpt p2, cpt q2, cpt r2, cpt n)
{
    TriPair t;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        t.v[0][i] = p1[i]; t.v[1][i] = q1[i]; t.v[2][i] = r1[i];
        t.v[3][i] = p2[i]; t.v[4][i] = q2[i]; t.v[5][i] = r2[i];
        t.n[i] = n[i];
    }
    return t;
}

// o = (a, b, c)[k], by value, so the permuted vertices stay in registers.
__device__ __forceinline__ void pick3(double (&o)[3], int k, const double *a, const double *b, const double *c)
{
#pragma unroll
    for (int i = 0; i < 3; ++i) o[i] = k == 0 ? a[i] : (k == 1 ? b[i] : c[i]);
}

__device__ __forceinline__ int tri_tri(cpt p1, cpt q1, cpt r1, cpt p2, cpt q2, cpt r2)
{
    double a[3], b[3], n1[3], n2[3];
    sub3(a, p2, r2); sub3(b, q2, r2); cross3(n2, a, b);
    sub3(a, p1, r2); const double dp1 = dot3(a, n2);
    sub3(a, q1, r2); const double dq1 = dot3(a, n2);
    sub3(a, r1, r2); const double dr1 = dot3(a, n2);
    if (dp1 * dq1 > 0 && dp1 * dr1 > 0) return 0;
    sub3(a, q1, p1); sub3(b, r1, p1); cross3(n1, a, b);
    sub3(a, p2, r1); const double dp2 = dot3(a, n1);
    sub3(a, q2, r1); const double dq2 = dot3(a, n1);
    sub3(a, r2, r1); const double dr2 = dot3(a, n1);
    if (dp2 * dq2 > 0 && dp2 * dr2 > 0) return 0;

    int rot1;
    bool sw2;
    if (!tt3_canon(dp1, dq1, dr1, rot1, sw2)) return tt3_coplanar(tri_pair(p1, q1, r1, p2, q2, r2, n1));
    // the permuted vertices are selected by value, not by pointer, so that
    // they stay in registers (the same values reach the same operations)
    double A1[3], B1[3], C1[3], B2[3], C2[3];
    pick3(A1, rot1, p1, q1, r1);
    pick3(B1, rot1, q1, r1, p1);
    pick3(C1, rot1, r1, p1, q1);
    pick3(B2, sw2 ? 1 : 0, q2, r2, r2);
    pick3(C2, sw2 ? 1 : 0, r2, q2, q2);
    const double da = dp2, db = sw2 ? dr2 : dq2, dc = sw2 ? dq2 : dr2;

    int rot2;
    bool sw1;
    if (!tt3_canon(da, db, dc, rot2, sw1)) return tt3_coplanar(tri_pair(A1, B1, C1, p2, B2, C2, n1));
    double X2[3], Y2[3], Z2[3], M1[3], N1[3];
    pick3(X2, rot2, p2, B2, C2);
    pick3(Y2, rot2, B2, C2, p2);
    pick3(Z2, rot2, C2, p2, B2);
    pick3(M1, sw1 ? 1 : 0, B1, C1, C1);
    pick3(N1, sw1 ? 1 : 0, C1, B1, B1);
    return tt3_minmax(A1, M1, N1, X2, Y2, Z2);
}

// NarrowPhase<double,2>::discrete_edge_edge (NarrowPhase.cpp:229-257).
__device__ __forceinline__ int seg_seg(cpt p0, cpt p1, cpt q0, cpt q1)
{
    const double eps = 2.220446049250313080847e-16; // DBL_EPSILON
    const double n0 = q0[0] - p0[0], n1 = q0[1] - p0[1];
    const double r0 = p1[0] - p0[0], r1 = p1[1] - p0[1];
    const double s0 = q1[0] - q0[0], s1 = q1[1] - q0[1];
    const double rxs = r0 * s1 - r1 * s0;
    if (fabs(rxs) < eps) return 0;
    const double nxr = n0 * r1 - n1 * r0;
    if (fabs(nxr) < eps)
        return ((q0[0] - p0[0] < 0) != (q0[0] - p1[0] < 0)) || ((q0[1] - p0[1] < 0) != (q0[1] - p1[1] < 0));
    const double nxs = n0 * s1 - n1 * s0;
    const double inv = 1.0 / rxs;
    const double t = nxs * inv, u = nxr * inv;
    return (t >= 0) && (t <= 1) && (u >= 0) && (u <= 1);
}

} // namespace mclccd
