// CTCD one-sided vertex-face narrow phase, as device functions: the path
// BVHTree::default_narrow_phase takes for VF stencils when vf_one_sided is
// set (BVHTree.cpp:445-447) -> NarrowPhaseCTCD<double,DIM>::query_ccd_vf
// with test_wrong_side = true (NarrowPhase.cpp:282-333 in 2D, 338-425 in 3D).
//
// 3D: a ray-box reject of the moving vertex against the face's swept box
// (NarrowPhase.cpp:123-160); then the first of vertex-face
// (CTCD.cpp:435-534), vertex-edge x3 (CTCD.cpp:536-634) and vertex-vertex x3
// (CTCD.cpp:715-817) that finds a time; its candidate times are tried in
// ascending order and the first that is not a wrong-side contact
// (NarrowPhase.cpp:58-89) is the toi.  2D: vertex-edge
// (CTCD.cpp:636-713) and the 2D wrong-side test (NarrowPhase.cpp:22-55).
//
// Each test builds polynomials in t whose sign intervals on [0, 1] are
// intersected (findIntervals, CTCD.cpp:110-186).  Those steps follow the
// reference's expression order (compiled with -fmad=false).  The one piece
// that is not the reference's: roots of degree 3-6 polynomials come from this
// file's Aberth-Ehrlich iteration (all complex roots, their real parts split
// [0, 1], as the reference does with the real parts of its Jenkins-Traub
// roots, rpoly.h), not from Jenkins-Traub.  Root values can therefore differ
// in the last bits, and so can toi; hit/miss can differ only when a sign
// interval's end decides an overlap to within that difference.
#pragma once

#include <math.h>

namespace mclccd {
namespace ctcd {

constexpr int kMaxIv = 8;   // a degree-6 polynomial splits [0,1] into <= 7 pieces
constexpr int kAberthIters = 128;

struct Iv {
    double l, u;
};
struct IvList {
    Iv v[kMaxIv];
    int n;
};

__device__ __forceinline__ double smax(double a, double b) { return (a < b) ? b : a; }   // std::max
__device__ __forceinline__ double smin(double a, double b) { return (b < a) ? b : a; }   // std::min

// TimeInterval(l, u) (CTCD.hpp:14-19): ordered, clipped to [0, 1].
__device__ __forceinline__ Iv make_iv(double l, double u)
{
    if (l > u) { const double t = l; l = u; u = t; }
    return Iv{smax(l, 0.0), smin(u, 1.0)};
}

__device__ __forceinline__ void push(IvList &L, double l, double u)
{
    if (L.n < kMaxIv) L.v[L.n++] = make_iv(l, u);
}

// ---------------------------------------------------------------------------
// 3-vectors, evaluated left to right (Eigen's fixed-size reductions).
// ---------------------------------------------------------------------------
struct V3 {
    double x, y, z;
};
__device__ __forceinline__ V3 v3(const double *p) { return V3{p[0], p[1], p[2]}; }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3 operator*(V3 a, double s) { return V3{a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ V3 operator*(double s, V3 a) { return V3{s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ double dot(V3 a, V3 b)
{
    double s = a.x * b.x;
    s = s + a.y * b.y;
    return s + a.z * b.z;
}
__device__ __forceinline__ V3 cross(V3 a, V3 b)
{
    return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

struct V2 {
    double x, y;
};
__device__ __forceinline__ V2 v2(const double *p) { return V2{p[0], p[1]}; }
__device__ __forceinline__ V2 operator-(V2 a, V2 b) { return V2{a.x - b.x, a.y - b.y}; }
__device__ __forceinline__ V2 operator+(V2 a, V2 b) { return V2{a.x + b.x, a.y + b.y}; }
__device__ __forceinline__ V2 operator*(V2 a, double s) { return V2{a.x * s, a.y * s}; }
__device__ __forceinline__ V2 operator*(double s, V2 a) { return V2{s * a.x, s * a.y}; }
__device__ __forceinline__ double dot(V2 a, V2 b)
{
    double s = a.x * b.x;
    return s + a.y * b.y;
}
__device__ __forceinline__ double norm(V2 a) { return sqrt(dot(a, a)); }

// ---------------------------------------------------------------------------
// Polynomial roots.  All n complex roots of c[0] x^n + ... + c[n] (n <= 6,
// c[0] != 0) by the Aberth-Ehrlich simultaneous iteration (O. Aberth, Math.
// Comp. 27, 1973; L. W. Ehrlich, CACM 10, 1967), started on circles whose
// radii come from the Newton polygon of the coefficient moduli (D. A. Bini,
// Numer. Algorithms 13, 1996).  Exact zeros at the origin are deflated first
// and reported as exact 0.  A root stops moving once |p(z)| is within the
// rounding-error bound of Horner's rule; points outside the unit circle are
// evaluated through the reversed polynomial so nothing overflows.  The
// iteration count is capped (kAberthIters).
// ---------------------------------------------------------------------------
struct Cx {
    double r, i;
};
__device__ __forceinline__ Cx cadd(Cx a, Cx b) { return Cx{a.r + b.r, a.i + b.i}; }
__device__ __forceinline__ Cx csub(Cx a, Cx b) { return Cx{a.r - b.r, a.i - b.i}; }
__device__ __forceinline__ Cx cmul(Cx a, Cx b) { return Cx{a.r * b.r - a.i * b.i, a.r * b.i + a.i * b.r}; }
__device__ __forceinline__ double cabs2(Cx a) { return hypot(a.r, a.i); }
// Smith's division (R. L. Smith, CACM 5, 1962): no overflow for large parts.
__device__ __forceinline__ Cx cdiv(Cx a, Cx b)
{
    if (fabs(b.r) >= fabs(b.i)) {
        if (b.r == 0.0) return Cx{a.r / b.r, a.i / b.r};
        const double q = b.i / b.r, d = b.r + b.i * q;
        return Cx{(a.r + a.i * q) / d, (a.i - a.r * q) / d};
    }
    const double q = b.r / b.i, d = b.r * q + b.i;
    return Cx{(a.r * q + a.i) / d, (a.i * q - a.r) / d};
}

// Newton correction p(z)/p'(z) of the degree-n polynomial c (descending
// powers) and whether p(z) is already at rounding level.
__device__ __forceinline__ Cx newton_step(const double *c, int n, Cx z, bool &done)
{
    const double az = cabs2(z);
    if (az <= 1.0) {   // Horner in z
        Cx p{c[0], 0.0}, dp{0.0, 0.0};
        double bound = fabs(c[0]);
        for (int k = 1; k <= n; ++k) {
            dp = cadd(cmul(dp, z), p);
            p = cadd(cmul(p, z), Cx{c[k], 0.0});
            bound = bound * az + fabs(c[k]);
        }
        done = cabs2(p) <= 2.0 * 1.1102230246251565e-16 * (double)(n + 1) * bound;
        return cdiv(p, dp);
    }
    // reversed polynomial q(y) = sum c[k] y^k at y = 1/z: p(z) = z^n q(y) and
    // p'(z)/p(z) = y (n - y q'(y) / q(y))
    const Cx y = cdiv(Cx{1.0, 0.0}, z);
    const double ay = cabs2(y);
    Cx q{c[n], 0.0}, dq{0.0, 0.0};
    double bound = fabs(c[n]);
    for (int k = n - 1; k >= 0; --k) {
        dq = cadd(cmul(dq, y), q);
        q = cadd(cmul(q, y), Cx{c[k], 0.0});
        bound = bound * ay + fabs(c[k]);
    }
    done = cabs2(q) <= 2.0 * 1.1102230246251565e-16 * (double)(n + 1) * bound;
    const Cx r = cmul(y, csub(Cx{(double)n, 0.0}, cmul(y, cdiv(dq, q))));
    return cdiv(Cx{1.0, 0.0}, r);
}

// Real parts of all roots of op[0] x^n + ... + op[n] into re[0..n); returns n.
__device__ inline int poly_real_parts(const double *op, int n, double *re)
{
    int m = n, out = 0;
    while (m > 0 && op[m] == 0.0) { re[out++] = 0.0; --m; }   // exact zeros at the origin
    if (m == 0) return out;
    double c[7];
    for (int k = 0; k <= m; ++k) c[k] = op[k];
    // Newton polygon: upper convex hull of (j, log|coefficient of x^j|)
    double lg[7];
    int j_of[7], np = 0;
    for (int j = 0; j <= m; ++j) {
        const double a = fabs(c[m - j]);
        lg[j] = a > 0.0 ? log(a) : -INFINITY;
    }
    for (int j = 0; j <= m; ++j) {
        if (lg[j] == -INFINITY) continue;
        while (np >= 2) {   // drop the last hull point if it lies on or below the chord
            const int a = j_of[np - 2], b = j_of[np - 1];
            if ((lg[b] - lg[a]) * (double)(j - a) <= (lg[j] - lg[a]) * (double)(b - a)) --np;
            else break;
        }
        j_of[np++] = j;
    }
    Cx z[6] = {};   // every slot set below when the coefficients are finite
    int nz = 0;
    for (int e = 0; e + 1 < np; ++e) {
        const int a = j_of[e], b = j_of[e + 1], cnt = b - a;
        const double r = exp((lg[a] - lg[b]) / (double)cnt);
        for (int k = 0; k < cnt && nz < 6; ++k) {
            const double ang = 6.283185307179586 * (double)k / (double)cnt + 1.5707963267948966 / (double)m +
                               0.4 * (double)e;
            z[nz++] = Cx{r * cos(ang), r * sin(ang)};
        }
    }
    bool conv[6] = {false, false, false, false, false, false};
    for (int it = 0; it < kAberthIters; ++it) {
        bool moved = false;
        for (int k = 0; k < m; ++k) {
            if (conv[k]) continue;
            bool done;
            const Cx N = newton_step(c, m, z[k], done);
            Cx S{0.0, 0.0};
            for (int j = 0; j < m; ++j) {
                if (j == k) continue;
                const Cx d = csub(z[k], z[j]);
                if (d.r != 0.0 || d.i != 0.0) S = cadd(S, cdiv(Cx{1.0, 0.0}, d));
            }
            const Cx den = csub(Cx{1.0, 0.0}, cmul(N, S));
            const Cx w = (den.r == 0.0 && den.i == 0.0) ? N : cdiv(N, den);
            if (!(isfinite(w.r) && isfinite(w.i))) {   // p'(z) = 0 or overflow: step aside
                const double h = 1e-3 * (1.0 + cabs2(z[k]));
                z[k] = cadd(z[k], Cx{h, 0.5 * h});
                moved = true;
                continue;
            }
            z[k] = csub(z[k], w);   // a point at rounding level takes this last correction and stops
            if (done) conv[k] = true;
            moved = true;
        }
        if (!moved) break;
    }
    for (int k = 0; k < m; ++k) re[out++] = z[k].r;
    return out;
}

// ---------------------------------------------------------------------------
// Sign intervals (CTCD.cpp:47-186).
// ---------------------------------------------------------------------------
// getQuadRoots (CTCD.cpp:47-64).
__device__ __forceinline__ int quad_roots(double a, double b, double c, double &t0, double &t1)
{
    const double sign = b < 0 ? -1.0 : 1.0;
    const double D = b * b - 4.0 * a * c;
    if (D >= 0) {
        const double q = -0.5 * (b + sign * sqrt(D));
        t0 = q / a;
        t1 = c / q;
        if (t0 > t1) { const double t = t0; t0 = t1; t1 = t; }
        return 2;
    }
    return 0;
}

// checkInterval (CTCD.cpp:67-86).
__device__ __forceinline__ void check_interval(double t1, double t2, const double *op, int degree, IvList &L, bool pos)
{
    t1 = smax(0.0, t1);
    t2 = smax(0.0, t2);
    t1 = smin(1.0, t1);
    t2 = smin(1.0, t2);
    const double tmid = (t2 + t1) / 2;
    double f = op[0];
    for (int i = 1; i <= degree; ++i) {
        f *= tmid;
        f += op[i];
    }
    if ((pos && f >= 0) || (!pos && f <= 0)) push(L, t1, t2);
}

// couldHaveRoots (CTCD.cpp:88-101).
__device__ __forceinline__ bool could_have_roots(const double *op, int degree, bool pos)
{
    double result = 0;
    if ((pos && op[0] > 0) || (!pos && op[0] < 0)) result = op[0];
    for (int i = 1; i < degree; ++i) {
        result *= 1.0;
        if ((pos && op[i] > 0) || (!pos && op[i] < 0)) result += op[i];
    }
    result *= 1.0;
    result += op[degree];
    return !((pos && result < 0) || (!pos && result > 0));
}

// findIntervals (CTCD.cpp:105-186): where the polynomial is >= 0 (pos) or
// <= 0 on [0, 1], as pieces between its (real parts of) roots.  op is
// normalised in place, as the reference does.
__device__ inline void find_intervals(double *op, int n, IvList &L, bool pos)
{
    double time[6];
    double maxval = 0;
    for (int i = 0; i <= n; ++i) maxval = smax(maxval, fabs(op[i]));
    if (maxval != 0)
        for (int i = 0; i <= n; ++i) op[i] /= maxval;
    int rd = n;
    for (int i = 0; i < n; ++i) {
        if (op[i] == 0) --rd;
        else break;
    }
    if (rd < n)
        for (int i = 0; i <= rd; ++i) op[i] = op[i + n - rd];
    int roots = 0;
    if (rd > 2) {
        if (!could_have_roots(op, rd, pos)) return;
        roots = poly_real_parts(op, rd, time);
    } else if (rd == 2) {
        roots = quad_roots(op[0], op[1], op[2], time[0], time[1]);
    } else if (rd == 1) {
        time[0] = -op[1] / op[0];
        roots = 1;
    } else {
        if ((!pos && op[0] <= 0) || (pos && op[0] >= 0)) push(L, 0.0, 1.0);
        return;
    }
    if (roots > 0) {
        for (int i = 1; i < roots; ++i)   // ascending (insertion sort, <= 6)
            for (int j = i; j > 0 && time[j] < time[j - 1]; --j) { const double t = time[j]; time[j] = time[j - 1]; time[j - 1] = t; }
        if (time[0] >= 0) check_interval(0, time[0], op, rd, L, pos);
        for (int i = 0; i < roots - 1; ++i)
            if (!((time[i] < 0 && time[i + 1] < 0) || (time[i] > 1.0 && time[i + 1] > 1.0)))
                check_interval(time[i], time[i + 1], op, rd, L, pos);
        if (time[roots - 1] <= 1.0) check_interval(time[roots - 1], 1.0, op, rd, L, pos);
    } else {
        check_interval(0.0, 1.0, op, rd, L, pos);
    }
}

// TimeInterval::overlap of a list (every pair) and the lower end of
// TimeInterval::intersect (CTCD.cpp:17-43).
__device__ __forceinline__ bool ov(const Iv &a, const Iv &b) { return !(a.l > b.u || b.l > a.u); }
__device__ __forceinline__ double isect_lo(const Iv *const *v, int n)
{
    double l = 0.0;
    for (int i = 0; i < n; ++i) l = smax(v[i]->l, l);
    return l;
}

// ---------------------------------------------------------------------------
// 3D tests.
// ---------------------------------------------------------------------------
// planePoly3D (CTCD.cpp:221-235): sign of the triple product in time.
__device__ inline void plane_poly(V3 x10, V3 x20, V3 x30, V3 v10, V3 v20, V3 v30, IvList &L)
{
    double op[4];
    op[0] = dot(v10, cross(v20, v30));
    op[1] = dot(x10, cross(v20, v30)) + dot(v10, cross(x20, v30)) + dot(v10, cross(v20, x30));
    op[2] = dot(x10, cross(x20, v30)) + dot(x10, cross(v20, x30)) + dot(v10, cross(x20, x30));
    op[3] = dot(x10, cross(x20, x30));
    find_intervals(op, 3, L, true);
}

// distancePoly3D (CTCD.cpp:237-263): squared distance to the plane minus eta^2, times |n|^2.
__device__ inline void distance_poly(V3 x10, V3 x20, V3 x30, V3 v10, V3 v20, V3 v30, double minD, IvList &L)
{
    const double A = dot(v10, cross(v20, v30));
    const double B = dot(x10, cross(v20, v30)) + dot(v10, cross(x20, v30)) + dot(v10, cross(v20, x30));
    const double C = dot(x10, cross(x20, v30)) + dot(x10, cross(v20, x30)) + dot(v10, cross(x20, x30));
    const double D = dot(x10, cross(x20, x30));
    const V3 E = cross(x20, x30);
    const V3 F = cross(x20, v30) + cross(v20, x30);
    const V3 G = cross(v20, v30);
    double op[7];
    op[0] = A * A;
    op[1] = 2 * A * B;
    op[2] = B * B + 2 * A * C - dot(G, G) * minD;
    op[3] = 2 * A * D + 2 * B * C - 2 * dot(G, F) * minD;
    op[4] = 2 * B * D + C * C - (2 * dot(G, E) + dot(F, F)) * minD;
    op[5] = 2 * C * D - 2 * dot(F, E) * minD;
    op[6] = D * D - dot(E, E) * minD;
    find_intervals(op, 6, L, false);
}

// Interval lists of the vertex-face test (CTCD.cpp:435-501); false when one is empty.
__device__ inline bool vf_lists(const V3 (&s)[4], const V3 (&e)[4], double eta, IvList (&L)[4])
{
    const double minD = eta * eta;
    const V3 v0 = e[0] - s[0], v1 = e[1] - s[1], v2 = e[2] - s[2], v3 = e[3] - s[3];
    for (auto &l : L) l.n = 0;
    plane_poly(s[0] - s[1], cross(s[3] - s[1], s[2] - s[1]), s[3] - s[1], v0 - v1, cross(v3 - v1, v2 - v1), v3 - v1, L[1]);
    if (L[1].n == 0) return false;
    plane_poly(s[0] - s[2], cross(s[1] - s[2], s[3] - s[2]), s[1] - s[2], v0 - v2, cross(v1 - v2, v3 - v2), v1 - v2, L[2]);
    if (L[2].n == 0) return false;
    plane_poly(s[0] - s[3], cross(s[2] - s[3], s[1] - s[3]), s[2] - s[3], v0 - v3, cross(v2 - v3, v1 - v3), v2 - v3, L[3]);
    if (L[3].n == 0) return false;
    distance_poly(s[0] - s[1], s[2] - s[1], s[3] - s[1], v0 - v1, v2 - v1, v3 - v1, minD, L[0]);
    return L[0].n > 0;
}

// Interval lists of vertexEdgeCTCD (CTCD.cpp:536-603): L[0] colinear within
// eta, L[1], L[2] the vertex between the edge's end planes.
__device__ inline bool ve_lists(V3 q0s, V3 q1s, V3 q2s, V3 q0e, V3 q1e, V3 q2e, double eta, IvList (&L)[4])
{
    double op[5];
    const double minD = eta * eta;
    const V3 v0 = q0e - q0s, v1 = q1e - q1s, v2 = q2e - q2s;
    const V3 ab = q2s - q1s, ac = q0s - q1s, cb = q2s - q0s;
    const V3 vab = v2 - v1, vac = v0 - v1, vcb = v2 - v0;
    for (auto &l : L) l.n = 0;
    double c = dot(ab, ac), b = dot(ac, vab) + dot(ab, vac), a = dot(vab, vac);
    op[0] = a; op[1] = b; op[2] = c;
    find_intervals(op, 2, L[1], true);
    if (L[1].n == 0) return false;
    c = dot(ab, cb); b = dot(cb, vab) + dot(ab, vcb); a = dot(vab, vcb);
    op[0] = a; op[1] = b; op[2] = c;
    find_intervals(op, 2, L[2], true);
    if (L[2].n == 0) return false;
    const double A = dot(ab, ab), B = 2 * dot(ab, vab), C = dot(vab, vab);
    const double D = dot(ac, ac), E = 2 * dot(ac, vac), F = dot(vac, vac);
    const double G = dot(ac, ab), H = dot(vab, ac) + dot(vac, ab), I = dot(vab, vac);
    op[4] = A * D - G * G - minD * A;
    op[3] = B * D + A * E - 2 * G * H - minD * B;
    op[2] = B * E + A * F + C * D - H * H - 2 * G * I - minD * C;
    op[1] = B * F + C * E - 2 * H * I;
    op[0] = C * F - I * I;
    find_intervals(op, 4, L[0], false);
    return L[0].n > 0;
}

// Smallest time > cur among the lower ends of the overlapping combinations
// of the first `nl` lists (one interval from each); +inf if none.
__device__ inline double next_combo_time(const IvList (&L)[4], int nl, double cur)
{
    double best = INFINITY;
    const int n0 = L[0].n, n1 = L[1].n, n2 = L[2].n, n3 = nl > 3 ? L[3].n : 1;
    for (int i = 0; i < n0; ++i)
        for (int j = 0; j < n1; ++j)
            for (int k = 0; k < n2; ++k)
                for (int l = 0; l < n3; ++l) {
                    const Iv *v[4] = {&L[0].v[i], &L[1].v[j], &L[2].v[k], nl > 3 ? &L[3].v[l] : nullptr};
                    bool o = true;
                    for (int a = 0; a < nl && o; ++a)
                        for (int b = a + 1; b < nl && o; ++b) o = ov(*v[a], *v[b]);
                    if (!o) continue;
                    const double t = isect_lo(v, nl);
                    if (t > cur && t < best) best = t;
                }
    return best;
}

// vertexVertexCTCD in 3D (CTCD.cpp:715-817) with a time list: the times it
// records, in order; returns whether it records any.
__device__ inline bool vv_times(V3 q1s, V3 q2s, V3 q1e, V3 q2e, double eta, double (&out)[3], int &nout)
{
    nout = 0;
    const double min_d = eta * eta;
    double t1 = 0, t2 = 0;
    const V3 v1 = q1e - q1s, v2 = q2e - q2s;
    const double a = dot(v1, v1) + dot(v2, v2) - 2 * dot(v1, v2);
    const double b = 2 * (dot(v1, q1s) - dot(v2, q1s) - dot(v1, q2s) + dot(v2, q2s));
    const double c = dot(q1s, q1s) + dot(q2s, q2s) - 2 * dot(q1s, q2s) - min_d;
    int roots;
    if (a != 0) {
        roots = quad_roots(a, b, c, t1, t2);
    } else if (b != 0) {
        t1 = -c / b;
        roots = 1;
    } else {
        if (c <= 0) { out[nout++] = 0; return true; }
        return false;
    }
    const double op[3] = {a, b, c};
    IvList iv;
    iv.n = 0;   // accumulates across the checks, as the reference's vector does
    if (roots == 2) {
        double curr_t = 1.0;
        check_interval(0, t1, op, 2, iv, false);
        if (iv.n) { curr_t = 0; out[nout++] = 0; }
        check_interval(t1, t2, op, 2, iv, false);
        if (iv.n) { curr_t = smin(curr_t, t1); out[nout++] = curr_t; }
        check_interval(t2, 1.0, op, 2, iv, false);
        if (iv.n) { curr_t = smin(t2, curr_t); out[nout++] = curr_t; }
        return nout > 0;
    }
    if (roots == 1) {
        check_interval(0, t1, op, 2, iv, false);
        if (iv.n) { out[nout++] = 0; return true; }
        check_interval(t1, 1.0, op, 2, iv, false);
        if (iv.n) { out[nout++] = t1; return true; }
        return false;
    }
    check_interval(0, 1.0, op, 2, iv, false);
    if (iv.n) { out[nout++] = 0; return true; }
    return false;
}

// Barycentric weights of the closest point of triangle (q0, q1, q2) to p,
// clamped to [0, 1]: the Voronoi-region walk of C. Ericson, Real-Time
// Collision Detection (2005) sec. 5.1.5, as ctcd::vertexFaceDistance
// evaluates it (Distance.hpp:34-124).
__device__ inline void closest_barys(V3 p, V3 q0, V3 q1, V3 q2, double &b0, double &b1, double &b2)
{
    const V3 ab = q1 - q0, ac = q2 - q0, ap = p - q0;
    const double d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0 && d2 <= 0) { b0 = 1.0; b1 = 0.0; b2 = 0.0; return; }
    const V3 bp = p - q1;
    const double d3 = dot(ab, bp), d4 = dot(ac, bp);
    if (d3 >= 0 && d4 <= d3) { b0 = 0.0; b1 = 1.0; b2 = 0.0; return; }
    const double vc = d1 * d4 - d3 * d2;
    if ((vc <= 0) && (d1 >= 0) && (d3 <= 0)) {
        const double v = d1 / (d1 - d3);
        b0 = 1.0 - v; b1 = v; b2 = 0; return;
    }
    const V3 cp = p - q2;
    const double d5 = dot(ab, cp), d6 = dot(ac, cp);
    if (d6 >= 0 && d5 <= d6) { b0 = 0; b1 = 0; b2 = 1.0; return; }
    const double vb = d5 * d2 - d1 * d6;
    if ((vb <= 0) && (d2 >= 0) && (d6 <= 0)) {
        const double w = d2 / (d2 - d6);
        b0 = 1 - w; b1 = 0; b2 = w; return;
    }
    const double va = d3 * d6 - d5 * d4;
    if ((va <= 0) && (d4 - d3 >= 0) && (d5 - d6 >= 0)) {
        const double w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        b0 = 0; b1 = 1.0 - w; b2 = w; return;
    }
    const double denom = 1.0 / (va + vb + vc);
    const double v = vb * denom, w = vc * denom;
    const double u = 1.0 - v - w;
    b0 = smin(smax(u, 0.0), 1.0);
    b1 = smin(smax(v, 0.0), 1.0);
    b2 = smin(smax(w, 0.0), 1.0);
}

// Eigen's stableNormalize: scale by the largest magnitude, then normalise.
__device__ __forceinline__ V3 stable_normalized(V3 n)
{
    double m = fabs(n.x);
    m = (m < fabs(n.y)) ? fabs(n.y) : m;
    m = (m < fabs(n.z)) ? fabs(n.z) : m;
    if (m > 0) {
        const V3 s{n.x / m, n.y / m, n.z / m};
        const double z = dot(s, s);
        if (z > 0) { const double r = sqrt(z); return V3{s.x / r, s.y / r, s.z / r}; }
    }
    return n;
}
__device__ __forceinline__ V2 stable_normalized(V2 n)
{
    double m = fabs(n.x);
    m = (m < fabs(n.y)) ? fabs(n.y) : m;
    if (m > 0) {
        const V2 s{n.x / m, n.y / m};
        const double z = dot(s, s);
        if (z > 0) { const double r = sqrt(z); return V2{s.x / r, s.y / r}; }
    }
    return n;
}

// NarrowPhase<double,3>::hit_wrong_side_vf (NarrowPhase.cpp:58-89).
__device__ inline bool wrong_side3(const V3 (&s)[4], const V3 (&e)[4], double t)
{
    if (fabs(t) <= 0.0) return false;
    V3 xt[4];
    for (int i = 0; i < 4; ++i) xt[i] = s[i] * (1.0 - t) + e[i] * t;
    V3 n = cross(xt[2] - xt[1], xt[3] - xt[1]);
    if (dot(n, n) <= 0) return false;
    n = stable_normalized(n);
    double b0 = 0, b1 = 0, b2 = 0;
    closest_barys(xt[0], xt[1], xt[2], xt[3], b0, b1, b2);
    const V3 apex_vel = e[0] - s[0];
    const V3 face_pt0 = b0 * s[1] + b1 * s[2] + b2 * s[3];
    const V3 face_pt1 = b0 * e[1] + b1 * e[2] + b2 * e[3];
    const V3 v = apex_vel - (face_pt1 - face_pt0);
    return dot(n, v) > 0.0;
}

// NarrowPhase<double,3>::query_ray_box (NarrowPhase.cpp:123-160): the slab
// test of A. Williams et al., "An Efficient and Robust Ray-Box Intersection
// Algorithm", JGT 10(1), 2005, on the segment p0 -> p1.
__device__ inline bool ray_box(V3 p0, V3 p1, V3 bmin, V3 bmax)
{
    V3 dir = p1 - p0;
    const double t0 = 0;
    const double t1 = sqrt(dot(dir, dir));
    auto inside = [&](V3 p) {
        return bmin.x <= p.x && bmin.y <= p.y && bmin.z <= p.z && p.x <= bmax.x && p.y <= bmax.y && p.z <= bmax.z;
    };
    if (inside(p0) || inside(p1)) return true;
    const double z = dot(dir, dir);
    if (z > 0) { const double r = sqrt(z); dir = V3{dir.x / r, dir.y / r, dir.z / r}; }
    const V3 inv{1. / dir.x, 1. / dir.y, 1. / dir.z};
    const bool sx = inv.x < 0, sy = inv.y < 0, sz = inv.z < 0;
    double tmin = ((sx ? bmax.x : bmin.x) - p0.x) * inv.x;
    double tmax = ((sx ? bmin.x : bmax.x) - p0.x) * inv.x;
    const double tymin = ((sy ? bmax.y : bmin.y) - p0.y) * inv.y;
    const double tymax = ((sy ? bmin.y : bmax.y) - p0.y) * inv.y;
    if ((tmin > tymax) || (tymin > tmax)) return false;
    if (tymin > tmin) tmin = tymin;
    if (tymax < tmax) tmax = tymax;
    const double tzmin = ((sz ? bmax.z : bmin.z) - p0.z) * inv.z;
    const double tzmax = ((sz ? bmin.z : bmax.z) - p0.z) * inv.z;
    if ((tmin > tzmax) || (tzmin > tmax)) return false;
    if (tzmin > tmin) tmin = tzmin;
    if (tzmax < tmax) tmax = tzmax;
    return (tmin < t1) && (tmax > t0);
}

// NarrowPhaseCTCD<double,3>::query_ccd_vf with test_wrong_side (NarrowPhase.cpp:338-425):
// 1 hit (toi set), 0 no contact, -1 only wrong-side contacts.
__device__ inline int query_vf3(const double (&x0)[4][3], const double (&x1)[4][3], double eta, double &toi)
{
    V3 s[4], e[4];
    for (int i = 0; i < 4; ++i) { s[i] = v3(x0[i]); e[i] = v3(x1[i]); }
    {   // the face's swept box, padded by eta
        V3 lo = s[1], hi = s[1];
        const V3 pts[5] = {e[1], s[2], e[2], s[3], e[3]};
        for (const V3 &p : pts) {
            lo = V3{(p.x < lo.x) ? p.x : lo.x, (p.y < lo.y) ? p.y : lo.y, (p.z < lo.z) ? p.z : lo.z};
            hi = V3{(hi.x < p.x) ? p.x : hi.x, (hi.y < p.y) ? p.y : hi.y, (hi.z < p.z) ? p.z : hi.z};
        }
        lo = V3{lo.x - eta, lo.y - eta, lo.z - eta};
        hi = V3{hi.x + eta, hi.y + eta, hi.z + eta};
        if (!ray_box(s[0], e[0], lo, hi)) return 0;
    }
    IvList L[4];
    int src = 0, nl = 4;
    double vvt[3];
    int nvv = 0;
    if (vf_lists(s, e, eta, L) && next_combo_time(L, 4, -INFINITY) < INFINITY) src = 1;
    for (int edge = 0; edge < 3 && !src; ++edge) {
        const int a = 1 + edge % 3, b = 1 + (edge + 1) % 3;
        if (ve_lists(s[0], s[a], s[b], e[0], e[a], e[b], eta, L) && next_combo_time(L, 3, -INFINITY) < INFINITY) {
            src = 2;
            nl = 3;
        }
    }
    for (int vert = 0; vert < 3 && !src; ++vert)
        if (vv_times(s[0], s[1 + vert], e[0], e[1 + vert], eta, vvt, nvv)) src = 3;
    if (!src) return 0;
    // candidate times ascending, negatives skipped; the first that is not a
    // wrong-side contact is the toi
    double cur = -INFINITY;
    for (int guard = 0; guard < kMaxIv * kMaxIv * kMaxIv * kMaxIv + 3; ++guard) {
        double t = INFINITY;
        if (src == 3) {
            for (int i = 0; i < nvv; ++i)
                if (vvt[i] > cur && vvt[i] < t) t = vvt[i];
        } else {
            t = next_combo_time(L, nl, cur);
        }
        if (!(t < INFINITY)) return -1;
        cur = t;
        if (t < 0) continue;
        if (!wrong_side3(s, e, t)) { toi = t; return 1; }
    }
    return -1;
}

// ---------------------------------------------------------------------------
// 2D (NarrowPhase.cpp:282-333; the 2D ray-box test always passes, 164-171).
// ---------------------------------------------------------------------------
// NarrowPhase<double,2>::hit_wrong_side_vf (NarrowPhase.cpp:22-55).
__device__ inline bool wrong_side2(const V2 (&s)[3], const V2 (&e)[3], double t)
{
    if (fabs(t) <= 0.0) return false;
    const V2 p = s[0] * (1.0 - t) + e[0] * t;
    const V2 e0 = s[1] * (1.0 - t) + e[1] * t;
    const V2 e1 = s[2] * (1.0 - t) + e[2] * t;
    const V2 n = stable_normalized(V2{e1.y - e0.y, -(e1.x - e0.x)});
    const double denom = norm(e0 - e1);
    if (denom < 2.220446049250313e-16) return false;
    const double bary0 = norm(e1 - p) / denom, bary1 = norm(e0 - p) / denom;
    const V2 e0bary = bary0 * s[1] + bary1 * s[2];
    const V2 e1bary = bary0 * e[1] + bary1 * e[2];
    const V2 v = (e[0] - s[0]) - (e1bary - e0bary);
    return dot(n, v) > 0.0;
}

// vertexEdgeCTCD in 2D (CTCD.cpp:636-713) with its recorded times, then the
// wrong-side pass of query_ccd_vf.
__device__ inline int query_vf2(const double (&x0)[3][2], const double (&x1)[3][2], double &toi)
{
    V2 s[3], e[3];
    for (int i = 0; i < 3; ++i) { s[i] = v2(x0[i]); e[i] = v2(x1[i]); }
    auto on_line = [](V2 p, V2 a, V2 b) {
        const double len = norm(a - b);
        if (norm(p - a) > len) return false;
        if (norm(p - b) > len) return false;
        return true;
    };
    const V2 u0 = s[1] - s[0], w0 = s[2] - s[0], u1 = e[1] - e[0], w1 = e[2] - e[0];
    const V2 up = u1 - u0, wp = w1 - w0;
    const double c = u0.x * w0.y - u0.y * w0.x;
    const double b = (u0.x * wp.y - u0.y * wp.x) + (up.x * w0.y - up.y * w0.x);
    const double a = up.x * wp.y - up.y * wp.x;
    double t0 = 2, t1 = 2;
    if (quad_roots(a, b, c, t0, t1) == 0) return 0;
    const bool on0 = on_line(s[0] * (1.0 - t0) + e[0] * t0, s[1] * (1.0 - t0) + e[1] * t0, s[2] * (1.0 - t0) + e[2] * t0);
    const bool on1 = on_line(s[0] * (1.0 - t1) + e[0] * t1, s[1] * (1.0 - t1) + e[1] * t1, s[2] * (1.0 - t1) + e[2] * t1);
    double c2[2];
    int nc = 0;
    if (t0 >= 0 && t0 <= 1 && on0) c2[nc++] = t0;
    if (t1 >= 0 && t1 <= 1 && on1) c2[nc++] = t1;
    if (nc == 0) return 0;
    if (nc == 2 && c2[1] < c2[0]) { const double t = c2[0]; c2[0] = c2[1]; c2[1] = t; }
    for (int i = 0; i < nc; ++i)
        if (!wrong_side2(s, e, c2[i])) { toi = c2[i]; return 1; }
    return -1;
}

} // namespace ctcd
} // namespace mclccd
