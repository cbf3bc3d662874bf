// Host build of the library's ACCD device code (mclccd_b200/csrc/geom.cuh),
// so the CPU tests can compare the exact arithmetic the kernels run with the
// oracle on any input, without a GPU.  Compiled by tests/test_accd_host.py
// with nvcc into a shared library; every function is the one the kernels
// call (host and device share one definition).
#include "../../mclccd_b200/csrc/geom.cuh"

using namespace mclccd;

template <int DIM>
static void gather(const double *V, const int *s, double (&x)[DIM + 1][DIM])
{
    for (int i = 0; i < DIM + 1; ++i)
        for (int k = 0; k < DIM; ++k) x[i][k] = V[(long long)s[i] * DIM + k];
}

extern "C" {

// form 0: accd (fast head, resumed tail), form 1: accd_literal (the
// reference loop step by step).  Per stencil: hit, toi (-1 on a miss), iters.
void host_accd(int dim, int form, const double *V0, const double *V1, const int *sten, const unsigned char *is_vf,
               long long n, double vf_eta, double ee_eta, int *hit, double *toi, int *iters)
{
    for (long long i = 0; i < n; ++i) {
        const int *s = sten + 4 * i;
        double t = -1.0;
        int h = 0, it = 0;
        if (dim == 3) {
            double a[4][3], b[4][3];
            gather<3>(V0, s, a);
            gather<3>(V1, s, b);
            if (is_vf[i]) h = form ? accd_literal<3, true>(a, b, vf_eta, t, it) : accd<3, true>(a, b, vf_eta, t, it);
            else h = form ? accd_literal<3, false>(a, b, ee_eta, t, it) : accd<3, false>(a, b, ee_eta, t, it);
        } else {
            double a[3][2], b[3][2];
            gather<2>(V0, s, a);
            gather<2>(V1, s, b);
            h = form ? accd_literal<2, true>(a, b, vf_eta, t, it) : accd<2, true>(a, b, vf_eta, t, it);
        }
        hit[i] = h;
        toi[i] = h ? t : -1.0;
        if (iters) iters[i] = it;
    }
}

// The distance routines alone: 3D VF (kind 1), 3D EE (kind 0), 2D (dim 2).
void host_distance(int dim, const double *X, const unsigned char *is_vf, long long n, double *out)
{
    for (long long i = 0; i < n; ++i) {
        const double *x = X + i * 4 * dim;
        if (dim == 2) out[i] = vf_distance2(x, x + 2, x + 4);
        else if (is_vf[i]) out[i] = vf_distance3(x, x + 3, x + 6, x + 9);
        else out[i] = ee_distance3(x, x + 3, x + 6, x + 9);
    }
}

} // extern "C"
