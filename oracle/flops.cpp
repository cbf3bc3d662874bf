// TEST INFRASTRUCTURE -- the FLOP count of the narrow phase, measured on the
// oracle.  Only bench-side measurement and tests use it; the product never
// links it.
//
// The oracle's distance routines (port_dist.h, the restatement of
// Projection.hpp) run here on a number type that counts every FP64
// operation: add/subtract, multiply, divide and square root are one flop
// each (comparisons, negation and min/max selection are not flops).  The
// narrow phase around them is counted two ways per stencil:
//   * reference: the reference's loop (NarrowPhase.cpp:634-711, as port.c
//     restates it), every operation it performs;
//   * necessary: the same decisions with the work whose results the
//     reference never uses left out -- iteration 0 when its step is an exact
//     zero (x and d unchanged), the distance at an iteration that returns
//     "miss" before a break is possible, the break threshold of a stencil
//     that misses, and the zero step itself -- and l_p from the larger
//     squared norm (two square roots).  That is the algorithm the device
//     kernels run (mclccd_b200/csrc/geom.cuh), so "necessary" is the FP64
//     work per stencil the roofline divides.  Both forms must return the same
//     (hit, toi) as port_accd; oracle/count_flops.py checks it.
#include <cmath>
#include <cstring>

namespace {

long long g_add, g_mul, g_div, g_sqrt;

struct Cd {
    double v;
    Cd() : v(0) {}
    Cd(double x) : v(x) {}
    Cd(int x) : v(x) {}
    Cd operator-() const { return Cd(-v); }
    Cd &operator+=(Cd o) { ++g_add; v += o.v; return *this; }
    Cd &operator-=(Cd o) { ++g_add; v -= o.v; return *this; }
    Cd &operator*=(Cd o) { ++g_mul; v *= o.v; return *this; }
};
Cd operator+(Cd a, Cd b) { ++g_add; return Cd(a.v + b.v); }
Cd operator-(Cd a, Cd b) { ++g_add; return Cd(a.v - b.v); }
Cd operator*(Cd a, Cd b) { ++g_mul; return Cd(a.v * b.v); }
Cd operator/(Cd a, Cd b) { ++g_div; return Cd(a.v / b.v); }
bool operator<(Cd a, Cd b) { return a.v < b.v; }
bool operator>(Cd a, Cd b) { return a.v > b.v; }
bool operator<=(Cd a, Cd b) { return a.v <= b.v; }
bool operator>=(Cd a, Cd b) { return a.v >= b.v; }
bool operator==(Cd a, Cd b) { return a.v == b.v; }
bool operator!=(Cd a, Cd b) { return a.v != b.v; }
Cd sqrt(Cd a) { ++g_sqrt; return Cd(std::sqrt(a.v)); }

long long flops() { return g_add + g_mul + g_div + g_sqrt; }

#define double Cd
#include "port_dist.h"
#undef double

Cd pair_distance(int dim, const Cd *x, int is_vf)
{
    if (dim == 2) return port_vf_distance2(x, x + 2, x + 4);
    if (is_vf) return port_vf_distance3(x, x + 3, x + 6, x + 9);
    return port_ee_distance3(x, x + 3, x + 6, x + 9);
}

// The reference loop, as port_additive_ccd runs it.
int counted_accd(int dim, const Cd *v0, const Cd *v1, Cd eta, int is_vf, double *toi_out, long long *dists)
{
    const int ns = dim + 1;
    const Cd s = 1, xsi = eta, t_c = 1;
    Cd p[12], x[12], pbar[3] = {0, 0, 0};
    for (int i = 0; i < ns; ++i)
        for (int k = 0; k < dim; ++k) {
            p[i * dim + k] = v1[i * dim + k] - v0[i * dim + k];
            x[i * dim + k] = v0[i * dim + k];
            pbar[k] += (Cd(1.0) / (Cd)ns) * p[i * dim + k];
        }
    for (int i = 0; i < ns; ++i)
        for (int k = 0; k < dim; ++k) p[i * dim + k] -= pbar[k];
    Cd lf = 0, ls = 0;
    for (int i = 0; i < ns; ++i) {
        Cd sq = 0;
        for (int k = 0; k < dim; ++k) sq = (k == 0) ? p[i * dim] * p[i * dim] : sq + p[i * dim + k] * p[i * dim + k];
        const Cd nrm = sqrt(sq);
        const int first = is_vf ? i == 0 : i <= 1;
        if (first) lf = lf < nrm ? nrm : lf;
        else ls = ls < nrm ? nrm : ls;
    }
    const Cd l_p = lf + ls;
    *toi_out = -1.0;
    if (l_p <= 0) return 0;
    Cd d = pair_distance(dim, x, is_vf);
    ++*dists;
    const Cd g = s * (d * d - xsi * xsi) / (d - xsi);
    Cd toi = 0;
    Cd t_l = (Cd(1) - s) * (d * d - xsi * xsi) / ((d + xsi) * l_p);
    if (d <= xsi) { *toi_out = 0.0; return 1; }
    for (int iter = 0; iter < 1000; ++iter) {
        for (int i = 0; i < ns * dim; ++i) x[i] = x[i] + t_l * p[i];
        d = pair_distance(dim, x, is_vf);
        ++*dists;
        const Cd eps = (d * d - xsi * xsi) / (d + xsi);
        if (toi > 0 && iter > 0 && eps < g) break;
        toi += t_l;
        if (toi > t_c) return 0;
        t_l = Cd(0.9) * (d * d - xsi * xsi) / ((d + xsi) * l_p);
    }
    *toi_out = toi.v;
    return 1;
}

// The same decisions with only the work they need (the device form, for
// stencils with finite motion and no -0.0 coordinate, where iteration 0 is
// an exact no-op): relative motion, l_p from the larger squared norms, the
// first distance and step, then -- for a stencil that goes on -- the
// threshold and the loop from iteration 1, with the distance at a miss
// decided before a break is possible left out.
int counted_fast(int dim, const Cd *v0, const Cd *v1, Cd eta, int is_vf, double *toi_out)
{
    const int ns = dim + 1;
    const Cd xsi = eta;
    Cd p[12], x[12], pbar[3] = {0, 0, 0};
    for (int i = 0; i < ns; ++i)
        for (int k = 0; k < dim; ++k) {
            p[i * dim + k] = v1[i * dim + k] - v0[i * dim + k];
            x[i * dim + k] = v0[i * dim + k];
            pbar[k] += (Cd(1.0) / (Cd)ns) * p[i * dim + k];
        }
    Cd lf2 = 0, ls2 = 0;
    for (int i = 0; i < ns; ++i) {
        Cd sq = 0;
        for (int k = 0; k < dim; ++k) {
            p[i * dim + k] -= pbar[k];
            sq = (k == 0) ? p[i * dim] * p[i * dim] : sq + p[i * dim + k] * p[i * dim + k];
        }
        const int first = is_vf ? i == 0 : i <= 1;
        if (first) lf2 = lf2 < sq ? sq : lf2;
        else ls2 = ls2 < sq ? sq : ls2;
    }
    const Cd l_p = sqrt(lf2) + sqrt(ls2);
    *toi_out = -1.0;
    if (l_p <= 0) return 0;
    const Cd d0 = pair_distance(dim, x, is_vf);
    const Cd A = d0 * d0 - xsi * xsi, X = (d0 + xsi) * l_p;
    if (d0 <= xsi) { *toi_out = 0.0; return 1; }
    Cd t_l = Cd(0.9) * A / X;
    if (t_l > 1.0) return 0;
    const Cd g = (Cd(1.0) * A) / (d0 - xsi);
    Cd toi = 0;
    for (int iter = 1; iter < 1000; ++iter) {
        const bool can_break = toi > 0;
        if (!can_break && toi + t_l > 1.0) return 0;
        for (int i = 0; i < ns * dim; ++i) x[i] = x[i] + t_l * p[i];
        const Cd d = pair_distance(dim, x, is_vf);
        const Cd B = d * d - xsi * xsi;
        if (can_break && B / (d + xsi) < g) { *toi_out = toi.v; return 1; }
        toi += t_l;
        if (toi > 1.0) return 0;
        t_l = Cd(0.9) * B / ((d + xsi) * l_p);
    }
    *toi_out = toi.v;
    return 1;
}

} // namespace

extern "C" {

// Flop tallies of the narrow phase over a stencil list (int32 x 4 each):
// out[kind * 4 + j], kind 0 = EE, 1 = VF; j: 0 stencils, 1 reference flops,
// 2 necessary flops, 3 distance evaluations of the reference loop.  hit/toi
// per stencil of both forms are returned so callers can check them against
// port_accd.
void flops_accd(int dim, const double *V0, const double *V1, const int *sten, const unsigned char *is_vf,
                long long n, double vf_eta, double ee_eta, long long *out, int *hit, double *toi, int *hit_fast,
                double *toi_fast)
{
    std::memset(out, 0, sizeof(long long) * 8);
    for (long long s = 0; s < n; ++s) {
        Cd a[12], b[12];
        for (int i = 0; i < dim + 1; ++i)
            for (int k = 0; k < dim; ++k) {
                a[i * dim + k] = V0[(long long)sten[4 * s + i] * dim + k];
                b[i * dim + k] = V1[(long long)sten[4 * s + i] * dim + k];
            }
        const int vf = dim == 2 || is_vf[s];
        long long dists = 0;
        long long f0 = flops();
        hit[s] = counted_accd(dim, a, b, vf ? vf_eta : ee_eta, vf, &toi[s], &dists);
        const long long f_ref = flops() - f0;
        f0 = flops();
        hit_fast[s] = counted_fast(dim, a, b, vf ? vf_eta : ee_eta, vf, &toi_fast[s]);
        const long long f_fast = flops() - f0;
        long long *o = out + 4 * vf;
        o[0] += 1;
        o[1] += f_ref;
        o[2] += f_fast;
        o[3] += dists;
    }
}

} // extern "C"
