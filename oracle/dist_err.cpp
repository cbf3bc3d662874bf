// TEST INFRASTRUCTURE -- how far the FP64 distance routines of the oracle
// (port_dist.h, the restatement of Projection.hpp) sit from the same routines
// evaluated in x87 extended precision (64-bit significand), stencil by
// stencil, with the case each evaluation took.  Only tests use it; the
// product never links it.
//
// The FP32-certified narrow phase brackets the value the FP64 routine returns
// and allows DELTA64 = 2^-36 S (S = coordinate magnitude) between that value
// and the exact distance of a well-conditioned problem; tests/
// test_oracle_delta64.py measures the deviation on adversarial stencils.
#include <cmath>
#include <cstring>

namespace {

int g_branch = 0;

}   // namespace

#define PORT_BRANCH(id) (g_branch = (id))

namespace d64 {
using std::sqrt;
#include "port_dist.h"
}   // namespace d64

#undef MCLCCD_ORACLE_PORT_DIST_H

namespace ext {

struct X {
    long double v;
    X() : v(0) {}
    X(long double x) : v(x) {}
    X(double x) : v(x) {}
    X(int x) : v(x) {}
    X operator-() const { return X(-v); }
    X &operator*=(X o) { v *= o.v; return *this; }
};
X operator+(X a, X b) { return X(a.v + b.v); }
X operator-(X a, X b) { return X(a.v - b.v); }
X operator*(X a, X b) { return X(a.v * b.v); }
X operator/(X a, X b) { return X(a.v / b.v); }
bool operator<(X a, X b) { return a.v < b.v; }
bool operator>(X a, X b) { return a.v > b.v; }
bool operator<=(X a, X b) { return a.v <= b.v; }
bool operator>=(X a, X b) { return a.v >= b.v; }
bool operator==(X a, X b) { return a.v == b.v; }
bool operator!=(X a, X b) { return a.v != b.v; }
X sqrt(X a) { return X(sqrtl(a.v)); }

#define double X
#include "port_dist.h"
#undef double

}   // namespace ext

extern "C" {

// For n stencils of four 3D points (12 doubles each): the FP64 distance d64,
// the extended-precision distance dx of the same routine on the same inputs,
// their difference d64 - dx taken in extended precision, and the case each
// evaluation took.  is_vf: point-triangle (1) or edge-edge (0).
void dist_err(long long n, const double *pts, const unsigned char *is_vf, double *d64, double *dx, double *diff,
              int *b64, int *bx)
{
    for (long long i = 0; i < n; ++i) {
        const double *p = pts + 12 * i;
        ext::X q[12];
        for (int k = 0; k < 12; ++k) q[k] = ext::X((long double)p[k]);
        g_branch = 0;
        d64[i] = is_vf[i] ? d64::port_vf_distance3(p, p + 3, p + 6, p + 9)
                          : d64::port_ee_distance3(p, p + 3, p + 6, p + 9);
        b64[i] = g_branch;
        g_branch = 0;
        const ext::X r = is_vf[i] ? ext::port_vf_distance3(q, q + 3, q + 6, q + 9)
                                  : ext::port_ee_distance3(q, q + 3, q + 6, q + 9);
        dx[i] = (double)r.v;
        diff[i] = (double)((long double)d64[i] - r.v);
        bx[i] = g_branch;
    }
}

}   // extern "C"
