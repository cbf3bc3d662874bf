/*
 * TEST INFRASTRUCTURE -- part of the oracle (CPU restatement); see port.c.
 *
 * The distance routines of the restatement (Projection.hpp point_on_triangle,
 * edge_to_edge, point_on_edge, each followed by .norm()), in a header of
 * their own so that oracle/flops.cpp can run the same code on a counting
 * number type.  Written in the common subset of C and C++; include it in one
 * translation unit per library (its functions have external linkage).
 */
#ifndef MCLCCD_ORACLE_PORT_DIST_H
#define MCLCCD_ORACLE_PORT_DIST_H

/* PORT_BRANCH(id) marks the case a routine takes (oracle/dist_err.cpp records
 * it to compare the case taken in FP64 and in higher precision); empty
 * otherwise. */
#ifndef PORT_BRANCH
#define PORT_BRANCH(id)
#endif

/* ---------------------------------------------------------------------- */
/* Distances.                                                                */
/* ---------------------------------------------------------------------- */
static double dot3(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static double clamp_zero_one(double v) { return v < 0 ? 0 : (v > 1 ? 1 : v); }
static double clamp01(double x)
{
    double m = x < 0 ? 0 : x;   /* std::max(x, 0) */
    return m < 1 ? m : 1;       /* std::min(1, m) */
}

/* Projection.hpp:61-145 point_on_triangle, then (point - closest).norm(). */
double port_vf_distance3(const double *pt, const double *p1, const double *p2, const double *p3)
{
    double e0[3], e1[3], v0[3];
    for (int k = 0; k < 3; ++k) { e0[k] = p2[k] - p1[k]; e1[k] = p3[k] - p1[k]; v0[k] = p1[k] - pt[k]; }
    double a = dot3(e0, e0), b = dot3(e0, e1), c = dot3(e1, e1), d = dot3(e0, v0), e = dot3(e1, v0);
    double det = a * c - b * b, s = b * e - c * d, t = b * d - a * e;
    if (s + t < det) {
        if (s < 0) {
            if (t < 0) {
                if (d < 0) { PORT_BRANCH(1); s = clamp_zero_one(-d / a); t = 0; }
                else { PORT_BRANCH(2); s = 0; t = clamp_zero_one(-e / c); }
            } else { PORT_BRANCH(3); s = 0; t = clamp_zero_one(-e / c); }
        } else if (t < 0) { PORT_BRANCH(4); s = clamp_zero_one(-d / a); t = 0; }
        else { PORT_BRANCH(5); double inv = 1.0 / det; s *= inv; t *= inv; }
    } else {
        if (s < 0) {
            double t0 = b + d, t1 = c + e;
            if (t1 > t0) { PORT_BRANCH(6); double num = t1 - t0, den = a - 2.0 * b + c; s = clamp_zero_one(num / den); t = 1 - s; }
            else { PORT_BRANCH(7); t = clamp_zero_one(-e / c); s = 0; }
        } else if (t < 0) {
            if (a + d > b + e) { PORT_BRANCH(8); double num = c + e - b - d, den = a - 2.0 * b + c; s = clamp_zero_one(num / den); t = 1 - s; }
            else { PORT_BRANCH(9); s = clamp_zero_one(-e / c); t = 0; }
        } else {
            PORT_BRANCH(10);
            double num = c + e - b - d, den = a - 2.0 * b + c;
            s = clamp_zero_one(num / den); t = 1 - s;
        }
    }
    double r[3];
    for (int k = 0; k < 3; ++k) r[k] = pt[k] - ((p1[k] + e0[k] * s) + e1[k] * t);
    return sqrt(dot3(r, r));
}

/* Projection.hpp:242-302 edge_to_edge, then .norm(). */
double port_ee_distance3(const double *p0, const double *p1, const double *q0, const double *q1)
{
    double d1[3], d2[3], r[3];
    for (int k = 0; k < 3; ++k) { d1[k] = p1[k] - p0[k]; d2[k] = q1[k] - q0[k]; r[k] = p0[k] - q0[k]; }
    double a = dot3(d1, d1), e = dot3(d2, d2), f = dot3(d2, r);
    double s = 0, t = 0;
    double c = dot3(d1, r), b = dot3(d1, d2);
    double denom = a * e - b * b;
    if (denom != 0) s = clamp01((b * f - c * e) / denom);
    else s = 0;
    double tnom = b * s + f;
    if (tnom < 0 || e == 0) { PORT_BRANCH(denom != 0 ? 11 : 21); t = 0; s = (a == 0) ? 0 : clamp01(-c / a); }
    else if (tnom > e) { PORT_BRANCH(denom != 0 ? 12 : 22); t = 1.0; s = (a == 0) ? 0 : clamp01((b - c) / a); }
    else { PORT_BRANCH(denom != 0 ? 13 : 23); t = tnom / e; }
    double w[3];
    for (int k = 0; k < 3; ++k) w[k] = (q0[k] + t * d2[k]) - (p0[k] + s * d1[k]);
    return sqrt(dot3(w, w));
}

/* Projection.hpp:194-204 point_on_edge (2D), then (point - closest).norm(). */
double port_vf_distance2(const double *p, const double *e0, const double *e1)
{
    double e[2] = {e1[0] - e0[0], e1[1] - e0[1]};
    double len2 = e[0] * e[0] + e[1] * e[1];
    double q[2];
    if (len2 <= 0.0) { q[0] = e0[0]; q[1] = e0[1]; }
    else {
        double pe[2] = {p[0] - e0[0], p[1] - e0[1]};
        double t = (pe[0] * e[0] + pe[1] * e[1]) / len2;
        if (t < 0.0) { q[0] = e0[0]; q[1] = e0[1]; }
        else if (t > 1.0) { q[0] = e1[0]; q[1] = e1[1]; }
        else { q[0] = e0[0] + t * e[0]; q[1] = e0[1] + t * e[1]; }
    }
    double w[2] = {p[0] - q[0], p[1] - q[1]};
    return sqrt(w[0] * w[0] + w[1] * w[1]);
}

#endif
