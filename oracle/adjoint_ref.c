/* FP64 CPU reference for the adjoint of the time of impact.
 *
 * TEST INFRASTRUCTURE ONLY: used by tests/ as the checker of the device
 * adjoint (mclccd_vjp_toi); never linked into the product.
 *
 * The reference (mclccd) has no adjoint; this restates the mathematics the
 * device kernel implements, with deliberately different algorithms so the
 * two are independent:
 *   - contact time t* = first root t >= toi of f(t) = dist(x(t)) - eta,
 *     x(t) = V0 + t (V1 - V0); found here by plain conservative advancement
 *     (t += f / l, never passing a root since |f'| <= l) followed by Newton
 *     polishing, where the device uses safeguarded Newton throughout;
 *   - closest points by enumeration (interior solution, else the best of the
 *     boundary candidates) where the device uses Voronoi-region case
 *     analysis;
 *   - gradient by the implicit function theorem at t*:
 *     d(t*)/dV0_i = -(1 - t*) w_i n / f_t, d(t*)/dV1_i = -t* w_i n / f_t, with w
 *     the signed closest-point weights and n the unit separation.
 * Status codes match MCLCCD_VJP_* of the public header.
 */
#include <math.h>
#include <string.h>

enum { ADJ_OK = 0, ADJ_TOI_ZERO = 1, ADJ_NO_CONTACT = 2, ADJ_GRAZING = 3, ADJ_NO_CONVERGE = 4, ADJ_BAD_TOI = 5 };

static double dot(const double *a, const double *b, int n)
{
    double s = 0;
    for (int k = 0; k < n; ++k) s += a[k] * b[k];
    return s;
}
static double clampd(double x) { return x < 0 ? 0 : (x > 1 ? 1 : x); }

/* Point p to segment a-b (dim n): parameter of the closest point. */
static double seg_param(const double *p, const double *a, const double *b, int n)
{
    double ab[3], ap[3];
    for (int k = 0; k < n; ++k) { ab[k] = b[k] - a[k]; ap[k] = p[k] - a[k]; }
    const double l2 = dot(ab, ab, n);
    return l2 > 0 ? clampd(dot(ap, ab, n) / l2) : 0.0;
}

static double dist_w(const double x[4][3], const double *w, int ns, int n)
{
    double s[3] = {0, 0, 0};
    for (int i = 0; i < ns; ++i)
        for (int k = 0; k < n; ++k) s[k] += w[i] * x[i][k];
    return sqrt(dot(s, s, n));
}

/* Signed weights w (first primitive +, second -) of the closest pair. */
static void closest(int dim, int is_vf, const double x[4][3], double *w)
{
    if (dim == 2) {
        const double s = seg_param(x[0], x[1], x[2], 2);
        w[0] = 1; w[1] = -(1 - s); w[2] = -s;
        return;
    }
    if (is_vf) {
        /* Interior of the triangle by barycentric coordinates of the plane
         * projection; else the closest of the three edges. */
        double e0[3], e1[3], ap[3];
        for (int k = 0; k < 3; ++k) { e0[k] = x[2][k] - x[1][k]; e1[k] = x[3][k] - x[1][k]; ap[k] = x[0][k] - x[1][k]; }
        const double a = dot(e0, e0, 3), b = dot(e0, e1, 3), c = dot(e1, e1, 3);
        const double d = dot(e0, ap, 3), e = dot(e1, ap, 3), det = a * c - b * b;
        if (det > 0) {
            const double u = (c * d - b * e) / det, v = (a * e - b * d) / det;
            if (u >= 0 && v >= 0 && u + v <= 1) {
                w[0] = 1; w[1] = -(1 - u - v); w[2] = -u; w[3] = -v;
                return;
            }
        }
        double best = INFINITY;
        const int ed[3][2] = {{1, 2}, {2, 3}, {3, 1}};
        for (int j = 0; j < 3; ++j) {
            const double s = seg_param(x[0], x[ed[j][0]], x[ed[j][1]], 3);
            double wt[4] = {1, 0, 0, 0};
            wt[ed[j][0]] = -(1 - s);
            wt[ed[j][1]] -= s;
            const double dd = dist_w(x, wt, 4, 3);
            if (dd < best) { best = dd; memcpy(w, wt, sizeof wt); }
        }
        return;
    }
    /* Edge-edge: interior stationary point if inside [0,1]^2, else the best of
     * the four endpoint-to-segment candidates. */
    double d1[3], d2[3], r[3];
    for (int k = 0; k < 3; ++k) { d1[k] = x[1][k] - x[0][k]; d2[k] = x[3][k] - x[2][k]; r[k] = x[0][k] - x[2][k]; }
    const double a = dot(d1, d1, 3), b = dot(d1, d2, 3), c = dot(d1, r, 3), e = dot(d2, d2, 3), f = dot(d2, r, 3);
    const double den = a * e - b * b;
    if (den > 1e-14 * a * e) {
        const double s = (b * f - c * e) / den, t = (a * f - b * c) / den;
        if (s >= 0 && s <= 1 && t >= 0 && t <= 1) {
            w[0] = 1 - s; w[1] = s; w[2] = -(1 - t); w[3] = -t;
            return;
        }
    }
    double best = INFINITY;
    for (int j = 0; j < 4; ++j) {
        double wt[4];
        if (j < 2) {   /* endpoint of the first segment to the second */
            const double t = seg_param(x[j], x[2], x[3], 3);
            wt[0] = j == 0; wt[1] = j == 1; wt[2] = -(1 - t); wt[3] = -t;
        } else {       /* endpoint of the second segment to the first */
            const double s = seg_param(x[j], x[0], x[1], 3);
            wt[0] = 1 - s; wt[1] = s; wt[2] = -(double)(j == 2); wt[3] = -(double)(j == 3);
        }
        const double dd = dist_w(x, wt, 4, 3);
        if (dd < best) { best = dd; memcpy(w, wt, sizeof wt); }
    }
}

/* f(t) = dist - eta with weights, unit separation and f_t. */
static double eval(int dim, int is_vf, const double *v0, const double *D, double t, double eta, double *w,
                   double *nrm, double *ft)
{
    const int ns = dim + 1;
    double x[4][3] = {{0}};
    for (int i = 0; i < ns; ++i)
        for (int k = 0; k < dim; ++k) x[i][k] = v0[i * dim + k] + t * D[i * dim + k];
    closest(dim, is_vf, x, w);
    double s[3] = {0, 0, 0}, v[3] = {0, 0, 0};
    for (int i = 0; i < ns; ++i)
        for (int k = 0; k < dim; ++k) { s[k] += w[i] * x[i][k]; v[k] += w[i] * D[i * dim + k]; }
    const double d = sqrt(dot(s, s, dim));
    *ft = 0;
    for (int k = 0; k < dim; ++k) { nrm[k] = d > 0 ? s[k] / d : 0; *ft += nrm[k] * v[k]; }
    return d - eta;
}

/* Contact time and the Jacobian row d(t*)/d(V0 slots, then V1 slots). */
int adj_ref_row(int dim, int is_vf, const double *v0, const double *v1, double eta, double toi, double *tstar,
                double *row)
{
    const int ns = dim + 1, na = (dim == 3 && !is_vf) ? 2 : 1, m = ns * dim;
    double D[12], mean[3] = {0, 0, 0}, w[4], nrm[3], ft;
    if (row) memset(row, 0, sizeof(double) * 2 * m);
    *tstar = toi;
    for (int i = 0; i < ns; ++i)
        for (int k = 0; k < dim; ++k) { D[i * dim + k] = v1[i * dim + k] - v0[i * dim + k]; mean[k] += D[i * dim + k] / ns; }
    double la = 0, lb = 0;
    for (int i = 0; i < ns; ++i) {
        double q = 0;
        for (int k = 0; k < dim; ++k) q += (D[i * dim + k] - mean[k]) * (D[i * dim + k] - mean[k]);
        q = sqrt(q);
        if (i < na) la = q > la ? q : la; else lb = q > lb ? q : lb;
    }
    const double l = (la + lb) * (1 + 1e-12);
    if (toi == 0) return ADJ_TOI_ZERO;
    if (!(toi > 0 && toi <= 1) || !(l > 0)) return ADJ_BAD_TOI;
    double t = toi, f = eval(dim, is_vf, v0, D, t, eta, w, nrm, &ft);
    if (f < 0) {
        /* Past the contact: it lies in [0, toi]; advance from 0 instead. */
        t = 0;
        f = eval(dim, is_vf, v0, D, t, eta, w, nrm, &ft);
        if (!(f > 0)) return ADJ_BAD_TOI;
    }
    /* Conservative advancement to within 1e-9 eta (or a quasi-stationary
     * creep), then Newton. */
    int k = 0;
    for (; k < 200000 && f > 1e-9 * eta; ++k) {
        const double tn = t + f / l;
        if (tn > 1) return ADJ_NO_CONTACT;   /* f > l (1 - t): no root in [t, 1] */
        if (tn == t) break;
        t = tn;
        f = eval(dim, is_vf, v0, D, t, eta, w, nrm, &ft);
    }
    if (k >= 200000) return ADJ_NO_CONVERGE;
    for (int j = 0; j < 40; ++j) {
        if (f == 0 || !(ft < 0)) break;
        const double tn = t - f / ft;
        if (!(fabs(tn - t) > 1e-17 * (1 + t))) { t = tn; f = eval(dim, is_vf, v0, D, t, eta, w, nrm, &ft); break; }
        t = tn;
        f = eval(dim, is_vf, v0, D, t, eta, w, nrm, &ft);
    }
    *tstar = t;
    if (!(ft < -1e-12 * l)) return ADJ_GRAZING;
    if (row)
        for (int i = 0; i < ns; ++i)
            for (int kk = 0; kk < dim; ++kk) {
                row[i * dim + kk] = -(1 - t) * w[i] * nrm[kk] / ft;
                row[m + i * dim + kk] = -t * w[i] * nrm[kk] / ft;
            }
    return ADJ_OK;
}

/* Batch over stencils given by vertex indices (sten: n x 4, -1 padded). */
void adj_ref_batch(int dim, const double *V0, const double *V1, const int *sten, const unsigned char *is_vf,
                   const double *toi, long long n, double vf_eta, double ee_eta, double *tstar, int *status,
                   double *rows)
{
    const int ns = dim + 1, m = 2 * ns * dim;
    for (long long h = 0; h < n; ++h) {
        double v0[12], v1[12];
        for (int i = 0; i < ns; ++i)
            for (int k = 0; k < dim; ++k) {
                v0[i * dim + k] = V0[(long long)sten[4 * h + i] * dim + k];
                v1[i * dim + k] = V1[(long long)sten[4 * h + i] * dim + k];
            }
        const int vf = dim == 2 || is_vf[h];
        status[h] = adj_ref_row(dim, vf, v0, v1, vf ? vf_eta : ee_eta, toi[h], &tstar[h], rows ? rows + h * m : 0);
    }
}

/* Central finite differences of t* (this file's root) in every coordinate of
 * one stencil: out[0..m) for V0 slots, out[m..2m) for V1 slots. */
int adj_ref_fd(int dim, int is_vf, const double *v0, const double *v1, double eta, double toi, double h, double *out)
{
    const int ns = dim + 1, m = ns * dim;
    double a[12], b[12], tp, tm;
    for (int j = 0; j < 2 * m; ++j) {
        memcpy(a, v0, sizeof(double) * m);
        memcpy(b, v1, sizeof(double) * m);
        double *x = j < m ? a : b;
        const int c = j < m ? j : j - m;
        const double x0 = x[c];
        x[c] = x0 + h;
        int s1 = adj_ref_row(dim, is_vf, a, b, eta, toi, &tp, 0);
        x[c] = x0 - h;
        int s2 = adj_ref_row(dim, is_vf, a, b, eta, toi, &tm, 0);
        if (s1 != ADJ_OK || s2 != ADJ_OK) return s1 != ADJ_OK ? s1 : s2;
        out[j] = (tp - tm) / (2 * h);
    }
    return ADJ_OK;
}
