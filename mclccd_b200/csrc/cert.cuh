// FP32-certified ACCD for one stencil (device functions), shared by the
// stencil-list kernels (certified.cu) and the batched path (batch.cu).  The
// method is described at the top of certified.cu.
#pragma once

#include "common.cuh"
#include "geom.cuh"

namespace mclccd {

namespace cert {

constexpr float kU = 0x1p-24f;        // FP32 unit roundoff
constexpr float kRel = 0x1p-20f;      // relative safety on every bracket (16 u)
constexpr float kRel64 = 0x1p-40f;    // relative slack for FP64 sums (per step)
constexpr float kDelta64 = 0x1p-36f;  // FP64 deviation allowance, relative to S
constexpr float kCond = 0x1p-10f;     // conditioning threshold (sin^2)
constexpr float kToiRel = 9.5e-7f;    // reported-toi bracket width allowed (inside 1e-6)
constexpr int kMaxIter = 8;           // FP32 iterations before handing over to FP64

struct Bracket {
    float lo, hi;
    bool ok;   // false: ill-conditioned, use FP64
};

__device__ __forceinline__ float dot3f(const float *a, const float *b)
{
    return __fmaf_rn(a[2], b[2], __fmaf_rn(a[1], b[1], a[0] * b[0]));
}
__device__ __forceinline__ float clampf01(float x) { return fminf(fmaxf(x, 0.f), 1.f); }

// Final bracket from an upper estimate hi_raw and a support-function lower
// estimate lo_raw, for points of magnitude <= M: both widened by 64 u M
// absolute plus kRel relative (covers every rounding of the evaluation).
__device__ __forceinline__ Bracket finish(float hi_raw, float lo_raw, float M)
{
    Bracket b;
    const float abs_err = __fmul_ru(64.f * kU, M) + 1e-36f;
    b.hi = __fmul_ru(__fadd_ru(hi_raw, abs_err), 1.f + kRel);
    b.lo = fmaxf(0.f, __fmul_rd(__fsub_rd(lo_raw, abs_err), 1.f - kRel));
    b.ok = true;
    return b;
}

// Bound on |Q32 - Q64| for a dot product Q of two difference vectors whose
// components are <= 2M and each off by <= eta_c from the vectors the FP64
// evaluation forms: 3 (4 M eta_c + eta_c^2) from the inputs plus the FP32
// rounding of the products and sums, doubled.
__device__ __forceinline__ float dot_err(float M, float eta_c)
{
    return __fmul_ru(2.f, __fadd_ru(__fmul_ru(__fmul_ru(12.f, M), eta_c),
                                    __fadd_ru(__fmul_ru(3.f * eta_c, eta_c), __fmul_ru(40.f * kU, __fmul_ru(M, M)))));
}

// Component error of the FP32 difference vectors against the FP64 ones: both
// endpoints off by perr, the FP32 and FP64 subtractions' rounding.
__device__ __forceinline__ float diff_err(float M, float S, float perr)
{
    return __fadd_ru(__fmul_ru(2.f, perr), __fadd_ru(__fmul_ru(4.f * kU, M), __fmul_ru(0x1p-50f, S)));
}

// Point pt to triangle (a, b, c), as Projection.hpp:61-145 point_on_triangle.
// M bounds the coordinates, S the FP64 coordinates, perr how far each FP32
// vertex coordinate sits from the one the FP64 evaluation uses.
__device__ __forceinline__ Bracket vf3(const float *pt, const float *a, const float *b, const float *c, float M,
                                       float S, float perr)
{
    float e0[3], e1[3], v[3];
    for (int k = 0; k < 3; ++k) { e0[k] = b[k] - a[k]; e1[k] = c[k] - a[k]; v[k] = a[k] - pt[k]; }
    const float A = dot3f(e0, e0), B = dot3f(e0, e1), C = dot3f(e1, e1), D = dot3f(e0, v), E = dot3f(e1, v);
    const float det = A * C - B * B;
    const Bracket bad{0.f, 0.f, false};
    if (!(A > 0.f) || !(C > 0.f) || !(det >= kCond * A * C)) return bad;
    float s = B * E - C * D, t = B * D - A * E;
    const float eta_c = diff_err(M, S, perr);
    const float Ed = dot_err(M, eta_c);
    // Which branch can the FP64 evaluation take?  The reference's only
    // off-closest branch is s + t >= det, s >= 0, t < 0, a + d <= b + e.
    bool may_bug, must_bug;
    {
        // With Sg = |A| + |B| + |C| + |D| + |E|, each of s, t, det and
        // s + t - det differs from its FP64 value by at most
        // E2 = 8 Sg Ed + 12 Ed^2 + 18 u Sg^2 (products of two perturbed dot
        // products, FP32 and FP64 rounding), and (a + d) - (b + e) by at most
        // E1 = 8 Ed + 4 u Sg.
        const float Sg = __fadd_ru(__fadd_ru(fabsf(A), fabsf(B)), __fadd_ru(__fadd_ru(fabsf(C), fabsf(D)), fabsf(E)));
        const float E2 = __fadd_ru(__fmul_ru(__fmul_ru(8.f, Sg), Ed),
                                   __fadd_ru(__fmul_ru(__fmul_ru(12.f, Ed), Ed), __fmul_ru(__fmul_ru(18.f * kU, Sg), Sg)));
        const float E1 = __fadd_ru(__fmul_ru(8.f, Ed), __fmul_ru(4.f * kU, Sg));
        const float st = s + t - det, ad = (A + D) - (B + E);
        may_bug = !(st < -E2 || s < -E2 || t > E2 || ad > E1);
        must_bug = st > E2 && s > E2 && t < -E2 && ad < -E1;
    }
    Bracket out{INFINITY, 0.f, true};
    if (!must_bug) {
        // Eberly's region logic: the closest point up to rounding (any point
        // of the triangle is a valid upper bound).
        if (s + t <= det) {
            if (s < 0.f) {
                if (t < 0.f) {
                    if (D < 0.f) { s = clampf01(-D / A); t = 0.f; }
                    else { s = 0.f; t = clampf01(-E / C); }
                } else { s = 0.f; t = clampf01(-E / C); }
            } else if (t < 0.f) { s = clampf01(-D / A); t = 0.f; }
            else { const float inv = 1.f / det; s *= inv; t *= inv; }
        } else {
            const float den = A - 2.f * B + C;
            if (s < 0.f) {
                const float t0 = B + D, t1 = C + E;
                if (t1 > t0) { s = clampf01((t1 - t0) / den); t = 1.f - s; }
                else { t = clampf01(-E / C); s = 0.f; }
            } else if (t < 0.f) {
                if (A + D > B + E) { s = clampf01((C + E - B - D) / den); t = 1.f - s; }
                else { s = clampf01(-D / A); t = 0.f; }
            } else { s = clampf01((C + E - B - D) / den); t = 1.f - s; }
        }
        s = clampf01(s);
        t = fminf(clampf01(t), __fsub_rd(1.f, s));   // s, t >= 0 and s + t <= 1 exactly
        float n[3];
        for (int k = 0; k < 3; ++k) n[k] = pt[k] - __fmaf_rn(t, e1[k], __fmaf_rn(s, e0[k], a[k]));
        const float nlen = sqrtf(dot3f(n, n));
        float lo_raw = 0.f;
        if (nlen > 1e-30f) {
            const float sp = dot3f(n, pt);
            const float sv = fmaxf(dot3f(n, a), fmaxf(dot3f(n, b), dot3f(n, c)));
            lo_raw = (sp - sv) / nlen;
        }
        out = finish(nlen, lo_raw, M);
    }
    if (may_bug) {
        // The branch's point a + clamp(-E/C) e0; the FP64 parameter differs
        // from the FP32 one by <= (Ed + |E/C| Ed) / (C - Ed) (clamp is
        // 1-Lipschitz), which moves the point by that times |e0|.
        if (!(C > 4.f * Ed)) return bad;
        const float sb = clampf01(-E / C);
        const float dsb = __fadd_ru(__fmul_ru(__fdiv_ru(__fadd_ru(Ed, __fmul_ru(__fdiv_ru(fabsf(E), C), Ed)),
                                                        __fsub_rd(C, Ed)), 1.f + kRel), 2.f * kU);
        const float len0 = __fadd_ru(__fmul_ru(sqrtf(A), 1.f + kRel), __fmul_ru(2.f, eta_c));   // >= |e0| in FP64
        float nb[3];
        for (int k = 0; k < 3; ++k) nb[k] = pt[k] - __fmaf_rn(sb, e0[k], a[k]);
        const float nl = sqrtf(dot3f(nb, nb));
        const float err = __fadd_ru(__fmul_ru(dsb, len0), __fmul_ru(64.f * kU, M) + 1e-36f);
        out.hi = fmaxf(out.hi, __fmul_ru(__fadd_ru(nl, err), 1.f + kRel));
        out.lo = fminf(out.lo, fmaxf(0.f, __fmul_rd(__fsub_rd(nl, err), 1.f - kRel)));
    }
    return out;
}

// Segment (p0,p1) to segment (q0,q1), as Projection.hpp:242-302 edge_to_edge.
__device__ __forceinline__ Bracket ee3(const float *p0, const float *p1, const float *q0, const float *q1, float M,
                                       float S, float perr)
{
    float d1[3], d2[3], r[3];
    for (int k = 0; k < 3; ++k) { d1[k] = p1[k] - p0[k]; d2[k] = q1[k] - q0[k]; r[k] = p0[k] - q0[k]; }
    const float a = dot3f(d1, d1), e = dot3f(d2, d2), f = dot3f(d2, r), c = dot3f(d1, r), b = dot3f(d1, d2);
    const float den = a * e - b * b;
    const Bracket bad{0.f, 0.f, false};
    const float Ed = dot_err(M, diff_err(M, S, perr));
    if (!(a > 4.f * Ed) || !(e > 4.f * Ed)) return bad;
    const float Ed2 = __fmul_ru(2.f, __fmul_ru(Ed, Ed));
    const float ED = __fmul_ru(2.f, __fadd_ru(__fadd_ru(__fmul_ru(a + e + 2.f * fabsf(b), Ed), Ed2),
                                               __fmul_ru(2.f * kU, __fadd_ru(a * e, b * b))));
    if (__fsub_rd(den, ED) >= kCond * a * e) {
        // Well-conditioned: the FP64 routine returns the closest pair.
        float s = clampf01((b * f - c * e) / den);
        float t;
        const float tnom = __fmaf_rn(b, s, f);
        if (tnom < 0.f) { t = 0.f; s = clampf01(-c / a); }
        else if (tnom > e) { t = 1.f; s = clampf01((b - c) / a); }
        else t = clampf01(tnom / e);
        float n[3];
        for (int k = 0; k < 3; ++k) n[k] = __fmaf_rn(s, d1[k], p0[k]) - __fmaf_rn(t, d2[k], q0[k]);
        const float nlen = sqrtf(dot3f(n, n));
        float lo_raw = 0.f;
        if (nlen > 1e-30f) {
            const float pa = fminf(dot3f(n, p0), dot3f(n, p1));
            const float qb = fmaxf(dot3f(n, q0), dot3f(n, q1));
            lo_raw = (pa - qb) / nlen;
        }
        return finish(nlen, lo_raw, M);
    }
    // Near-parallel: the FP64 s = clamp((b f - c e) / denom) can be anywhere in
    // [s_lo, s_hi] (all of [0, 1] when denom may be ~0).  Then t = (b s + f)/e
    // unclamped gives dist(P(s), segment q), convex in s, so at most its value
    // at s_lo or s_hi; t clamped to 0 or 1 gives the exact distance from q0 or
    // q1 to segment p.  Every value is a distance between points of the two
    // segments, so the exact distance bounds them all from below.
    float slo = 0.f, shi = 1.f;
    {
        const float EN = __fmul_ru(2.f, __fadd_ru(__fadd_ru(__fmul_ru(fabsf(b) + fabsf(f) + fabsf(c) + fabsf(e), Ed), Ed2),
                                                   __fmul_ru(2.f * kU, __fadd_ru(fabsf(b * f), fabsf(c * e)))));
        const float N = b * f - c * e;
        const float dlo = __fsub_rd(den, ED);
        if (dlo > 0.f) {
            const float dhi = __fadd_ru(den, ED);
            const float nlo = __fsub_rd(N, EN), nhi = __fadd_ru(N, EN);
            slo = clampf01(__fsub_rd(__fdiv_rd(nlo, nlo >= 0.f ? dhi : dlo), 0x1p-30f));
            shi = clampf01(__fadd_ru(__fdiv_ru(nhi, nhi >= 0.f ? dlo : dhi), 0x1p-30f));
        }
    }
    const float Et = __fmul_ru(2.f, __fadd_ru(__fmul_ru(2.f, Ed), __fmul_ru(2.f * kU, fabsf(b) + fabsf(f))));
    const float ta = __fmaf_rn(b, slo, f), tb = __fmaf_rn(b, shi, f);
    const float tnlo = __fsub_rd(fminf(ta, tb), Et), tnhi = __fadd_ru(fmaxf(ta, tb), Et);
    const bool reach0 = tnlo < 0.f;
    const bool reach1 = tnhi > __fsub_rd(e, Ed);
    const bool reachm = tnhi >= 0.f && tnlo <= __fadd_ru(e, Ed);
    float hi = 0.f, best = INFINITY, nb[3] = {0.f, 0.f, 0.f};
    auto take = [&](const float *P, const float *Qp) {
        float n[3];
        for (int k = 0; k < 3; ++k) n[k] = P[k] - Qp[k];
        const float L = sqrtf(dot3f(n, n));
        hi = fmaxf(hi, L);
        if (L < best) { best = L; nb[0] = n[0]; nb[1] = n[1]; nb[2] = n[2]; }
    };
    if (reachm) {
        for (int j = 0; j < 2; ++j) {
            const float s = j ? shi : slo;
            float P[3], w[3], Qp[3];
            for (int k = 0; k < 3; ++k) { P[k] = __fmaf_rn(s, d1[k], p0[k]); w[k] = P[k] - q0[k]; }
            const float t = clampf01(dot3f(w, d2) / e);
            for (int k = 0; k < 3; ++k) Qp[k] = __fmaf_rn(t, d2[k], q0[k]);
            take(P, Qp);
        }
    }
    if (reach0) {
        const float s = clampf01(-c / a);
        float P[3];
        for (int k = 0; k < 3; ++k) P[k] = __fmaf_rn(s, d1[k], p0[k]);
        take(P, q0);
    }
    if (reach1) {
        const float s = clampf01((b - c) / a);
        float P[3];
        for (int k = 0; k < 3; ++k) P[k] = __fmaf_rn(s, d1[k], p0[k]);
        take(P, q1);
    }
    if (!(best < INFINITY)) return bad;
    float lo_raw = 0.f;
    if (best > 1e-30f) {
        const float pa = fminf(dot3f(nb, p0), dot3f(nb, p1));
        const float qb = fmaxf(dot3f(nb, q0), dot3f(nb, q1));
        lo_raw = (pa - qb) / best;
    }
    return finish(hi, lo_raw, M);
}

// Point pt to segment (e0, e1) in 2D, as Projection.hpp:194-204 point_on_edge.
__device__ __forceinline__ Bracket vf2(const float *pt, const float *e0, const float *e1, float M)
{
    const float e[2] = {e1[0] - e0[0], e1[1] - e0[1]};
    const float len2 = __fmaf_rn(e[1], e[1], e[0] * e[0]);
    const Bracket bad{0.f, 0.f, false};
    if (!(len2 > 0.f)) return bad;
    const float t = clampf01(__fmaf_rn(pt[1] - e0[1], e[1], (pt[0] - e0[0]) * e[0]) / len2);
    const float n[2] = {pt[0] - __fmaf_rn(t, e[0], e0[0]), pt[1] - __fmaf_rn(t, e[1], e0[1])};
    const float nlen = sqrtf(__fmaf_rn(n[1], n[1], n[0] * n[0]));
    float lo_raw = 0.f;
    if (nlen > 1e-30f) {
        const float sp = __fmaf_rn(n[1], pt[1], n[0] * pt[0]);
        const float sv = fmaxf(__fmaf_rn(n[1], e0[1], n[0] * e0[0]), __fmaf_rn(n[1], e1[1], n[0] * e1[0]));
        lo_raw = (sp - sv) / nlen;
    }
    return finish(nlen, lo_raw, M);
}

template <int DIM, bool VF>
__device__ __forceinline__ Bracket dist_bracket(const float (&x)[DIM + 1][DIM], float M, float S, float perr)
{
    if constexpr (DIM == 2) return vf2(x[0], x[1], x[2], M);
    else if constexpr (VF) return vf3(x[0], x[1], x[2], x[3], M, S, perr);
    else return ee3(x[0], x[1], x[2], x[3], M, S, perr);
}

__device__ __forceinline__ float ru_d(double x) { return __double2float_ru(x); }
__device__ __forceinline__ float rd_d(double x) { return __double2float_rd(x); }

} // namespace cert

// Outcome codes of the certified evaluation.
enum { kCertMiss = 0, kCertHit = 1, kCertFallback = 2 };

// Certified ACCD for one stencil.  On kCertHit, toi is the reported toi and
// bound tells whether it is the certified lower bound (within 1e-6 relative)
// rather than the FP64 value itself.
template <int DIM, bool VF>
__device__ __forceinline__ int accd_certified(const double (&v0)[DIM + 1][DIM], const double (&v1)[DIM + 1][DIM],
                                              double eta, double &toi, bool &bound)
{
    using namespace cert;
    constexpr int ns = DIM + 1;
    bound = false;
    double p[ns][DIM], x[ns][DIM], l_p, d0, g, t_l;
    bool noop, skip;
    accd_setup<DIM, VF, true>(v0, v1, p, x, l_p, noop);
    const int h = accd_head<DIM, VF>(x, p, l_p, noop, eta, d0, g, toi, t_l, skip);
    if (h == kHeadHit) return kCertHit;           // toi == 0
    if (h == kHeadMiss) return kCertMiss;
    // Continue: x == v0, toi == 0 and t_l = L1 in (0, 1] when iteration 0 was
    // a no-op (it is unless an input is -0.0 or non-finite).
    if (!skip || !(t_l > 0.0)) return kCertFallback;
    const double L1 = t_l;

    double S = 0.0, Pmax = 0.0;
#pragma unroll
    for (int i = 0; i < ns; ++i)
#pragma unroll
        for (int k = 0; k < DIM; ++k) { S = fmax(S, fabs(v0[i][k])); Pmax = fmax(Pmax, fabs(p[i][k])); }
    if (!(S < 1e15) || !(Pmax < 1e15)) return kCertFallback;
    // Local frame at the first vertex (y) and motion relative to it (qf).
    float y[ns][DIM], qf[ns][DIM];
    float M0 = 0.f, Q = 0.f;
#pragma unroll
    for (int i = 0; i < ns; ++i)
#pragma unroll
        for (int k = 0; k < DIM; ++k) {
            y[i][k] = (float)(v0[i][k] - v0[0][k]);
            qf[i][k] = (float)(p[i][k] - p[0][k]);
            M0 = fmaxf(M0, fabsf(y[i][k]));
            Q = fmaxf(Q, fabsf(qf[i][k]));
        }
    if (!(M0 > 1e-12f)) return kCertFallback;
    const float Qb = __fadd_ru(__fmul_ru(Q, 1.f + kRel), 1e-36f);
    const float Sd = ru_d(S), Pd = ru_d(Pmax);
    const float eta_lo = rd_d(eta), eta_hi = ru_d(eta);
    const float lp_lo = rd_d(l_p), lp_hi = ru_d(l_p);
    const float g_lo = rd_d(g), g_hi = ru_d(g);
    if (!(lp_lo > 0.f) || !(lp_hi < INFINITY) || !(g_hi < INFINITY)) return kCertFallback;

    // [slo, shi] contains s_k = L1 + ... + Lk (the FP64 iterate is x0 + s_k p up
    // to its accumulated rounding); [plo, phi] holds s_{k-1}, the toi a break
    // at iteration k reports.
    float slo = rd_d(L1), shi = ru_d(L1), plo = 0.f, phi = 0.f;
#pragma unroll 1
    for (int it = 1; it <= kMaxIter; ++it) {
        const float sm = 0.5f * (slo + shi);
        const float hw = fmaxf(__fsub_ru(shi, sm), __fsub_ru(sm, slo));
        float z[ns][DIM];
        float Mk = 0.f;
#pragma unroll
        for (int i = 0; i < ns; ++i)
#pragma unroll
            for (int k = 0; k < DIM; ++k) { z[i][k] = __fmaf_rn(sm, qf[i][k], y[i][k]); Mk = fmaxf(Mk, fabsf(z[i][k])); }
        const float Sf = __fadd_ru(Sd, __fmul_ru(fabsf(shi), Pd));   // FP64 coordinate magnitude
        // Per-coordinate error of z against x0 + sm p (FP32 inputs and their
        // FP64 differences, FP32 evaluation) and of x0 + sm p against the
        // FP64 iterate (its accumulated rounding).
        const float comp = __fadd_ru(__fmul_ru(__fmul_ru(kU, __fadd_ru(__fadd_ru(M0, Mk), __fmul_ru(2.f * fabsf(sm), Q))), 1.f + kRel),
                                     __fmul_ru(0x1p-50f * (float)(it + 1), Sf));
        const float perr = __fadd_ru(comp, __fmul_ru(hw, Qb));
        const Bracket b = dist_bracket<DIM, VF>(z, Mk, Sf, perr);
        if (!b.ok) return kCertFallback;
        // FP64 distance within: the bracket, 2 sqrt(3) comp (each vertex off by
        // sqrt(3) comp moves the distance by at most twice that), l_p hw (the
        // spread of s) and DELTA64.
        const float wid = __fadd_ru(__fadd_ru(__fmul_ru(2.f * 1.7320509f, comp), __fmul_ru(lp_hi, hw)),
                                    __fadd_ru(__fmul_ru(kDelta64, Sf), 1e-36f));
        const float Dlo = fmaxf(0.f, __fsub_rd(b.lo, wid));
        const float Dhi = __fadd_ru(b.hi, wid);
        // FP64 (d^2 - eta^2) / (d + eta) = d - eta up to 4 u64 (d + eta).
        const float slack = __fmul_ru(kRel, __fadd_ru(Dhi, eta_hi));
        const float elo = __fsub_rd(__fsub_rd(Dlo, eta_hi), slack);
        const float ehi = __fadd_ru(__fsub_ru(Dhi, eta_lo), slack);
        if (it >= 2) {                                     // toi >= L1 > 0: the break test runs
            if (ehi < g_lo) {                              // eps < g: hit at toi s_{k-1}
                if (it == 2) { toi = L1; return kCertHit; }
                const float tl = __fmul_rd(plo, 1.f - kRel64 * (float)it);
                const float th = __fmul_ru(phi, 1.f + kRel64 * (float)it);
                if (!(__fsub_ru(th, tl) <= __fmul_rd(kToiRel, tl))) return kCertFallback;
                toi = (double)tl;
                bound = true;
                return kCertHit;
            }
            if (!(elo >= g_hi)) return kCertFallback;      // break undecided
            // No break: toi becomes s_k; miss once it exceeds 1.
            if (__fmul_rd(slo, 1.f - kRel64 * (float)it) > 1.f) return kCertMiss;
            if (!(__fmul_ru(shi, 1.f + kRel64 * (float)it) <= 1.f)) return kCertFallback;
        }
        // Next step L_{k+1} = 0.9 (d^2 - eta^2) / ((d + eta) l_p).
        const float nlo = __fmul_rd(0.9f * (1.f - kRel), elo);
        const float nhi = __fmul_ru(0.9f * (1.f + kRel), ehi);
        const float Llo = __fdiv_rd(nlo, nlo >= 0.f ? lp_hi : lp_lo);
        const float Lhi = __fdiv_ru(nhi, nhi >= 0.f ? lp_lo : lp_hi);
        plo = slo;
        phi = shi;
        slo = __fadd_rd(slo, Llo);
        shi = __fadd_ru(shi, Lhi);
        if (!(shi < 1e30f) || !(slo > -1e30f)) return kCertFallback;
    }
    return kCertFallback;
}

template <int DIM>
__device__ __forceinline__ bool gather_c(const int *s, const double *__restrict__ V0, const double *__restrict__ V1,
                                         int nv, double (&x0)[DIM + 1][DIM], double (&x1)[DIM + 1][DIM])
{
    bool ok = true;
#pragma unroll
    for (int i = 0; i < DIM + 1; ++i) {
        int v = s[i];
        if (v < 0 || v >= nv) { ok = false; v = 0; }
#pragma unroll
        for (int k = 0; k < DIM; ++k) {
            x0[i][k] = __ldg(V0 + (size_t)v * DIM + k);
            x1[i][k] = __ldg(V1 + (size_t)v * DIM + k);
        }
    }
    return ok;
}

} // namespace mclccd
