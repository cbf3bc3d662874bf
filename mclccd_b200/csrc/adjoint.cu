// Adjoint of the time of impact: dTOI/dV0 and dTOI/dV1 per hit, as a
// vector-Jacobian product.
//
// The reference's toi is a sum of conservative steps (NarrowPhase.cpp:
// 686-707), not a root of anything, so the quantity differentiated is the
// contact time it approximates: t* = the first root t >= toi of
//     f(t) = dist(x(t)) - eta,   x_i(t) = V0_i + t (V1_i - V0_i)
// (ACCD's toi never passes that root: the distance shrinks at most at l_p per
// unit time and ACCD steps at most 0.9 (d - eta) / l_p).  At a simple root the
// implicit function theorem gives
//     dt*/dV0_i = -(1 - t*) (df/dx_i) / f_t,   dt*/dV1_i = -t* (df/dx_i) / f_t,
// with df/dx_i = +w_i n for the vertices of the first primitive and -w_i n
// for the second (w = barycentric weights of the closest points, n the unit
// separation from the second primitive's closest point to the first's) and
// f_t = n . (sum_A w_i D_i - sum_B w_j D_j), D = V1 - V0.  The kernel recomputes
// the closest-feature pair at t* (nothing is stored from the forward pass).
//
// Closest points are the true ones (Ericson, Real-Time Collision Detection,
// 2005, 5.1.5 point-triangle and 5.1.9 segment-segment), evaluated in FP64.
// The root is found from toi by conservative advancement along the current
// separating direction (no root is ever passed; a step beyond t = 1 proves
// there is none), which converges to the first root quadratically.
#include "common.cuh"
#include "kernels.cuh"

namespace mclccd {

namespace adj {

// Status per hit (MCLCCD_VJP_* in the public header).
enum { kOk = 0, kToiZero = 1, kNoContact = 2, kGrazing = 3, kNoConverge = 4, kBadToi = 5, kBadIndex = 6 };

__device__ __forceinline__ double dot3(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
__device__ __forceinline__ double clamp01(double x) { return x < 0.0 ? 0.0 : (x > 1.0 ? 1.0 : x); }

// Closest point of triangle (a, b, c) to p as barycentric weights (u, v, w).
__device__ void closest_pt_tri(const double *p, const double *a, const double *b, const double *c, double *wt)
{
    double ab[3], ac[3], ap[3], bp[3], cp[3];
    for (int k = 0; k < 3; ++k) { ab[k] = b[k] - a[k]; ac[k] = c[k] - a[k]; ap[k] = p[k] - a[k]; }
    const double d1 = dot3(ab, ap), d2 = dot3(ac, ap);
    if (d1 <= 0.0 && d2 <= 0.0) { wt[0] = 1.0; wt[1] = 0.0; wt[2] = 0.0; return; }
    for (int k = 0; k < 3; ++k) bp[k] = p[k] - b[k];
    const double d3 = dot3(ab, bp), d4 = dot3(ac, bp);
    if (d3 >= 0.0 && d4 <= d3) { wt[0] = 0.0; wt[1] = 1.0; wt[2] = 0.0; return; }
    const double vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) {
        const double t = d1 / (d1 - d3);
        wt[0] = 1.0 - t; wt[1] = t; wt[2] = 0.0;
        return;
    }
    for (int k = 0; k < 3; ++k) cp[k] = p[k] - c[k];
    const double d5 = dot3(ab, cp), d6 = dot3(ac, cp);
    if (d6 >= 0.0 && d5 <= d6) { wt[0] = 0.0; wt[1] = 0.0; wt[2] = 1.0; return; }
    const double vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) {
        const double t = d2 / (d2 - d6);
        wt[0] = 1.0 - t; wt[1] = 0.0; wt[2] = t;
        return;
    }
    const double va = d3 * d6 - d5 * d4;
    if (va <= 0.0 && (d4 - d3) >= 0.0 && (d5 - d6) >= 0.0) {
        const double t = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        wt[0] = 0.0; wt[1] = 1.0 - t; wt[2] = t;
        return;
    }
    const double inv = 1.0 / (va + vb + vc);
    wt[1] = vb * inv;
    wt[2] = vc * inv;
    wt[0] = 1.0 - wt[1] - wt[2];
}

// Closest points of segments (p0,p1) and (q0,q1): parameters s, t.
__device__ void closest_seg_seg(const double *p0, const double *p1, const double *q0, const double *q1, double &s,
                                double &t)
{
    double d1[3], d2[3], r[3];
    for (int k = 0; k < 3; ++k) { d1[k] = p1[k] - p0[k]; d2[k] = q1[k] - q0[k]; r[k] = p0[k] - q0[k]; }
    const double a = dot3(d1, d1), e = dot3(d2, d2), f = dot3(d2, r);
    if (a <= 0.0 && e <= 0.0) { s = t = 0.0; return; }
    if (a <= 0.0) { s = 0.0; t = clamp01(f / e); return; }
    const double c = dot3(d1, r);
    if (e <= 0.0) { t = 0.0; s = clamp01(-c / a); return; }
    const double b = dot3(d1, d2);
    const double denom = a * e - b * b;
    s = denom > 0.0 ? clamp01((b * f - c * e) / denom) : 0.0;
    t = (b * s + f) / e;
    if (t < 0.0) { t = 0.0; s = clamp01(-c / a); }
    else if (t > 1.0) { t = 1.0; s = clamp01((b - c) / a); }
}

// Stencil geometry: slots [0, na) form the first primitive, [na, ns) the second.
template <int DIM, bool VF>
struct Stencil {
    static constexpr int ns = DIM + 1;
    static constexpr int na = VF ? 1 : 2;
    double x0[ns][DIM], D[ns][DIM];
};

// Distance at time t, with the closest-point weights (signed: + first
// primitive, - second), unit separation n and f_t.
template <int DIM, bool VF>
__device__ void eval(const Stencil<DIM, VF> &S, double t, double &d, double (&w)[DIM + 1], double (&n)[DIM],
                     double &ft)
{
    constexpr int ns = DIM + 1;
    double x[ns][3];
#pragma unroll
    for (int i = 0; i < ns; ++i) {
#pragma unroll
        for (int k = 0; k < DIM; ++k) x[i][k] = S.x0[i][k] + t * S.D[i][k];
        if (DIM == 2) x[i][2] = 0.0;
    }
    if constexpr (DIM == 2) {
        double e[3] = {x[2][0] - x[1][0], x[2][1] - x[1][1], 0.0}, pe[3] = {x[0][0] - x[1][0], x[0][1] - x[1][1], 0.0};
        const double len2 = dot3(e, e);
        const double s = len2 > 0.0 ? clamp01(dot3(pe, e) / len2) : 0.0;
        w[0] = 1.0; w[1] = -(1.0 - s); w[2] = -s;
    } else if constexpr (VF) {
        double wt[3];
        closest_pt_tri(x[0], x[1], x[2], x[3], wt);
        w[0] = 1.0; w[1] = -wt[0]; w[2] = -wt[1]; w[3] = -wt[2];
    } else {
        double s, u;
        closest_seg_seg(x[0], x[1], x[2], x[3], s, u);
        w[0] = 1.0 - s; w[1] = s; w[2] = -(1.0 - u); w[3] = -u;
    }
    double sep[DIM], vel[DIM];
#pragma unroll
    for (int k = 0; k < DIM; ++k) { sep[k] = 0.0; vel[k] = 0.0; }
#pragma unroll
    for (int i = 0; i < ns; ++i)
#pragma unroll
        for (int k = 0; k < DIM; ++k) { sep[k] += w[i] * x[i][k]; vel[k] += w[i] * S.D[i][k]; }
    double d2 = 0.0;
#pragma unroll
    for (int k = 0; k < DIM; ++k) d2 += sep[k] * sep[k];
    d = sqrt(d2);
    const double inv = d > 0.0 ? 1.0 / d : 0.0;
    ft = 0.0;
#pragma unroll
    for (int k = 0; k < DIM; ++k) { n[k] = sep[k] * inv; ft += n[k] * vel[k]; }
}

// Contact root and the factors of the Jacobian row for one stencil: on kOk,
// dt*/dV0 of slot i, coordinate k = c0 (w_i n_k) and dt*/dV1 = c1 (w_i n_k)
// (jacobian_entry); otherwise the row is zero.  Returns the status.  The row
// itself is formed by the caller, so its 2 (DIM + 1) DIM values are never
// live during the root search.
template <int DIM, bool VF>
__device__ int toi_gradient(const double (&v0)[DIM + 1][DIM], const double (&v1)[DIM + 1][DIM], double eta,
                            double toi, double &tstar, double (&w)[DIM + 1], double (&n)[DIM], double &c0, double &c1)
{
    constexpr int ns = DIM + 1;
    Stencil<DIM, VF> S;
    constexpr int na = Stencil<DIM, VF>::na;
#pragma unroll
    for (int i = 0; i < ns; ++i)
#pragma unroll
        for (int k = 0; k < DIM; ++k) {
            S.x0[i][k] = v0[i][k];
            S.D[i][k] = v1[i][k] - v0[i][k];
        }
    // Lipschitz bound of the distance in t: the closest points' relative
    // velocity is a convex combination of the vertex pairs' D_a - D_b.
    double lmax = 0.0;
#pragma unroll
    for (int a = 0; a < na; ++a)
#pragma unroll
        for (int b = na; b < ns; ++b) {
            double q = 0.0;
#pragma unroll
            for (int k = 0; k < DIM; ++k) q += (S.D[a][k] - S.D[b][k]) * (S.D[a][k] - S.D[b][k]);
            lmax = fmax(lmax, q);
        }
    const double l = sqrt(lmax) * (1.0 + 1e-12);
    c0 = c1 = 0.0;
    tstar = toi;
    if (toi == 0.0) return kToiZero;
    if (!(toi > 0.0) || !(toi <= 1.0) || !(l > 0.0) || !isfinite(l)) return kBadToi;

    double d, ft;
    double t = toi;
    eval<DIM, VF>(S, t, d, w, n, ft);
    double f = d - eta;
    if (!(f >= 0.0)) {
        // The reference's distance can exceed the true one (its off-closest
        // point_on_triangle branch), so ACCD may step past the true contact:
        // then search from t = 0.
        t = 0.0;
        eval<DIM, VF>(S, t, d, w, n, ft);
        f = d - eta;
        if (!(f > 0.0)) return kBadToi;
    }
    // Advancement along the separating direction n at t: every vertex moves
    // linearly, so the support gap along n, min_a n.x_a(tau) - max_b n.x_b(tau),
    // is bounded below by each pair's linear n.(x_a - x_b)(tau) and never
    // exceeds the distance.  The largest tau keeping every pair at >= eta is
    // therefore a step that passes no root; it is at least the Lipschitz step
    // f / l and, near a contact, the Newton step, so the iterates rise to the
    // first root quadratically.  A step beyond t = 1 proves there is none.
    bool converged = false;
    for (int it = 0; it < 512; ++it) {
        if (!(f > 0.0)) { converged = true; break; }
        double tau = INFINITY;
#pragma unroll
        for (int a = 0; a < na; ++a)
#pragma unroll
            for (int b = na; b < ns; ++b) {
                double c = 0.0, v = 0.0;
#pragma unroll
                for (int k = 0; k < DIM; ++k) {
                    c += n[k] * ((S.x0[a][k] + t * S.D[a][k]) - (S.x0[b][k] + t * S.D[b][k]));
                    v += n[k] * (S.D[a][k] - S.D[b][k]);
                }
                if (v < 0.0) tau = fmin(tau, (c - eta) / -v);
            }
        const double step = fmax(tau, f / l);   // both are root-free; rounding can only shrink tau
        if (t + step > 1.0) return kNoContact;
        if (!(step > 4e-16 * fmax(1.0, t))) { converged = true; break; }
        t = t + step;
        eval<DIM, VF>(S, t, d, w, n, ft);
        f = d - eta;
    }
    tstar = t;
    if (!converged) return kNoConverge;
    if (!(ft < -1e-12 * l)) return kGrazing;   // not a transversal crossing
    c0 = -(1.0 - t) / ft;
    c1 = -t / ft;
    return kOk;
}

template <int DIM>
__device__ __forceinline__ bool gather_a(const int *s, const double *__restrict__ V0, const double *__restrict__ V1,
                                         int nv, double (&x0)[DIM + 1][DIM], double (&x1)[DIM + 1][DIM])
{
    bool ok = true;
#pragma unroll
    for (int i = 0; i < DIM + 1; ++i) {
        int v = s[i];
        if (v < 0 || v >= nv) { ok = false; v = 0; }
#pragma unroll
        for (int k = 0; k < DIM; ++k) {
            x0[i][k] = V0[(size_t)v * DIM + k];
            x1[i][k] = V1[(size_t)v * DIM + k];
        }
    }
    return ok;
}

// One thread per hit: row, t*, status, and g * row scattered into dV0 / dV1.
template <int DIM>
__global__ void __launch_bounds__(128, 4)
k_vjp_toi(const int *__restrict__ sten, const unsigned char *__restrict__ is_vf, const double *__restrict__ toi,
          const double *__restrict__ g, long long n, const double *__restrict__ V0, const double *__restrict__ V1,
          int nv, double vf_eta, double ee_eta, double *__restrict__ dV0, double *__restrict__ dV1,
          double *__restrict__ t_star, int *__restrict__ status, double *__restrict__ rows,
          unsigned long long *n_ok)
{
    constexpr int ns = DIM + 1;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long h = (long long)blockIdx.x * blockDim.x + threadIdx.x; h < n; h += stride) {
        const int s[4] = {sten[4 * h], sten[4 * h + 1], sten[4 * h + 2], sten[4 * h + 3]};
        double w[ns], nn[DIM], c0 = 0.0, c1 = 0.0, ts = toi[h];
        int st;
        {
            double x0[ns][DIM], x1[ns][DIM];
            if (!gather_a<DIM>(s, V0, V1, nv, x0, x1)) st = kBadIndex;
            else if (DIM == 3 && !is_vf[h]) st = toi_gradient<DIM, false>(x0, x1, ee_eta, toi[h], ts, w, nn, c0, c1);
            else st = toi_gradient<DIM, true>(x0, x1, vf_eta, toi[h], ts, w, nn, c0, c1);
        }
        if (t_star) t_star[h] = ts;
        if (status) status[h] = st;
        const bool ok = st == kOk;
        // row entries: c (w_i n_k), zero unless ok
        if (rows)
#pragma unroll
            for (int i = 0; i < ns; ++i)
#pragma unroll
                for (int k = 0; k < DIM; ++k) {
                    const double gx = ok ? w[i] * nn[k] : 0.0;
                    rows[h * 2 * ns * DIM + i * DIM + k] = ok ? c0 * gx : 0.0;
                    rows[h * 2 * ns * DIM + ns * DIM + i * DIM + k] = ok ? c1 * gx : 0.0;
                }
        if (ok) {
            if (n_ok) {   // one atomic per warp
                const unsigned m = __activemask();
                if ((int)lane_id() == __ffs(m) - 1) atomicAdd(n_ok, (unsigned long long)__popc(m));
            }
            const double gh = g ? g[h] : 0.0;
            if (gh != 0.0 && dV0 && dV1)
#pragma unroll
                for (int i = 0; i < ns; ++i)
#pragma unroll
                    for (int k = 0; k < DIM; ++k) {
                        const double gx = w[i] * nn[k];
                        atomicAdd(dV0 + (size_t)s[i] * DIM + k, gh * (c0 * gx));
                        atomicAdd(dV1 + (size_t)s[i] * DIM + k, gh * (c1 * gx));
                    }
        }
    }
}

} // namespace adj

void launch_vjp_toi(int dim, const int *sten, const unsigned char *is_vf, const double *toi, const double *g,
                    long long n, const double *V0, const double *V1, int nv, double vf_eta, double ee_eta,
                    double *dV0, double *dV1, double *t_star, int *status, double *rows, unsigned long long *n_ok,
                    cudaStream_t st)
{
    if (n <= 0) return;
    long long grid = (n + 127) / 128;
    if (grid > 148 * 16) grid = 148 * 16;
    if (dim == 3)
        adj::k_vjp_toi<3><<<(int)grid, 128, 0, st>>>(sten, is_vf, toi, g, n, V0, V1, nv, vf_eta, ee_eta, dV0, dV1,
                                                     t_star, status, rows, n_ok);
    else
        adj::k_vjp_toi<2><<<(int)grid, 128, 0, st>>>(sten, is_vf, toi, g, n, V0, V1, nv, vf_eta, ee_eta, dV0, dV1,
                                                     t_star, status, rows, n_ok);
}

} // namespace mclccd
