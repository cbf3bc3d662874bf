// TEST INFRASTRUCTURE -- the oracle.  Never linked into, or called by, the
// product library.
//
// C ABI around the reference's own, unmodified mcl::BVHTree<double,DIM>
// (include/MCL/BVHTree.cpp, NarrowPhase.cpp, BVHLeaf.cpp, ccd_internal/CTCD.cpp
// of mattoverby/mclccd), compiled against the stand-in Eigen/TBB headers in
// oracle/compat.  It records exactly what the reference hands to its hooks:
//   * candidates : every stencil passed to filter_pair (BVHTree.cpp:345,368,393),
//                  which the reference calls for each stencil before the
//                  narrow phase;
//   * hits       : every append_pair(sten, is_vf, toi) call (BVHTree.cpp:264);
//   * discrete   : every append_discrete(p0, p1) call (BVHTree.cpp:280).
// Hooks run concurrently on the reference's worker threads, so recording goes
// through sharded, mutex-protected buffers.
#include "MCL/BVHTree.hpp"
#include "MCL/NarrowPhase.hpp"
#include "MCL/ccd_internal/rpoly.h"
#include "tbb/parallel_for.h"

#include <atomic>
#include <chrono>
#include <cstring>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

namespace {

struct Candidate { int s[4]; unsigned char is_vf; };
struct Hit { int s[4]; unsigned char is_vf; double toi; };
struct Pair { int a, b; };

template <typename T>
struct Sharded {
    static const int kShards = 64;
    std::mutex mu[kShards];
    std::vector<T> buf[kShards];
    void push(const T &v)
    {
        size_t h = std::hash<std::thread::id>()(std::this_thread::get_id()) % kShards;
        std::lock_guard<std::mutex> lk(mu[h]);
        buf[h].push_back(v);
    }
    std::vector<T> gather()
    {
        std::vector<T> out;
        for (int i = 0; i < kShards; ++i) { out.insert(out.end(), buf[i].begin(), buf[i].end()); buf[i].clear(); }
        return out;
    }
};

struct State {
    std::vector<Candidate> cand;
    std::vector<Hit> hits;
    std::vector<Pair> disc;
    std::vector<double> boxes;   // per leaf: box.min, box.max, t0.min, t0.max, t1.min, t1.max (DIM each)
    std::vector<int> flags;      // per leaf: v[0..2], e[0..2], active
    int dim = 3;
};
State g_state;

enum { F_REPTRI = 1, F_THREADED = 2, F_DISCRETE = 4, F_CONTINUOUS = 8, F_RECORD_CAND = 16, F_ONE_SIDED = 32, F_FLOAT = 64 };

// T = float runs the reference's BVHTree<float, DIM> on the coordinates
// rounded to float (its own float arithmetic throughout).
template <typename T, int DIM>
int run(const double *V0d, const double *V1d, const int *P, int np, int pdim,
        double box_eta, double vf_eta, double ee_eta, int flags, const int *active)
{
    int nv = 0;
    for (long long i = 0; i < (long long)np * pdim; ++i) nv = std::max(nv, P[i] + 1);
    const std::vector<T> V0v(V0d, V0d + (size_t)nv * DIM), V1v(V1d, V1d + (size_t)nv * DIM);
    const T *V0 = V0v.data(), *V1 = V1v.data();
    mcl::BVHTree<T, DIM> tree;
    tree.options.box_eta = box_eta;
    tree.options.vf_ccd_eta = vf_eta;
    tree.options.ee_ccd_eta = ee_eta;
    tree.options.reptri = (flags & F_REPTRI) != 0;
    tree.options.threaded = (flags & F_THREADED) != 0;
    tree.options.discrete = (flags & F_DISCRETE) != 0;
    tree.options.continuous = (flags & F_CONTINUOUS) != 0;
    tree.options.vf_one_sided = (flags & F_ONE_SIDED) != 0;

    Sharded<Candidate> cand;
    Sharded<Hit> hits;
    Sharded<Pair> disc;
    if (flags & F_RECORD_CAND) {
        tree.filter_pair = [&](const Eigen::Vector4i &s, bool is_vf) -> bool {
            Candidate c; for (int i = 0; i < 4; ++i) c.s[i] = s[i]; c.is_vf = is_vf;
            cand.push(c);
            return false;
        };
    }
    tree.append_pair = [&](const Eigen::Vector4i &s, bool is_vf, const T &toi) {
        Hit h; for (int i = 0; i < 4; ++i) h.s[i] = s[i]; h.is_vf = is_vf; h.toi = (double)toi;
        hits.push(h);
    };
    tree.append_discrete = [&](int p0, int p1) -> bool {
        disc.push(Pair{p0, p1});
        return false;
    };

    tree.update(V0, V1, P, np, pdim, active);
    tree.traverse(V0, V1, P);

    g_state.dim = DIM;
    g_state.cand = cand.gather();
    g_state.hits = hits.gather();
    g_state.disc = disc.gather();
    g_state.boxes.assign(size_t(np) * 6 * DIM, 0.0);
    g_state.flags.assign(size_t(np) * 7, 0);
    for (int i = 0; i < (int)tree.leaves.size(); ++i) {
        const auto &L = tree.leaves[i];
        double *b = &g_state.boxes[size_t(i) * 6 * DIM];
        for (int k = 0; k < DIM; ++k) {
            b[0 * DIM + k] = L.box.min()[k]; b[1 * DIM + k] = L.box.max()[k];
            b[2 * DIM + k] = L.box.t0.min()[k]; b[3 * DIM + k] = L.box.t0.max()[k];
            b[4 * DIM + k] = L.box.t1.min()[k]; b[5 * DIM + k] = L.box.t1.max()[k];
        }
        int *f = &g_state.flags[size_t(i) * 7];
        for (int k = 0; k < 3; ++k) { f[k] = L.v[k]; f[3 + k] = L.e[k]; }
        f[6] = L.box.active ? 1 : 0;
    }
    return 0;
}

template <int DIM>
void accd(const double *V0, const double *V1, const int *sten, const unsigned char *is_vf,
          long long n, double vf_eta, double ee_eta, int *hit, double *toi)
{
    typedef typename mcl::NarrowPhaseACCD<double, DIM>::VecType Vec;
    for (long long s = 0; s < n; ++s) {
        Vec x0[DIM + 1], x1[DIM + 1];
        for (int i = 0; i < DIM + 1; ++i)
            for (int k = 0; k < DIM; ++k) {
                x0[i][k] = V0[size_t(sten[4 * s + i]) * DIM + k];
                x1[i][k] = V1[size_t(sten[4 * s + i]) * DIM + k];
            }
        double t = -1;
        int h = is_vf[s] ? mcl::NarrowPhaseACCD<double, DIM>::query_ccd_vf(x0, x1, vf_eta, t)
                         : mcl::NarrowPhaseACCD<double, DIM>::query_ccd_ee(x0, x1, ee_eta, t);
        hit[s] = h;
        toi[s] = h == 1 ? t : -1.0;
    }
}

// NarrowPhaseCTCD::query_ccd_vf (NarrowPhase.cpp:282-333 in 2D, 338-425 in
// 3D) with test_wrong_side = true, as default_narrow_phase calls it when
// vf_one_sided is set (BVHTree.cpp:445-447).  ret: 1 hit, 0 no hit, -1 only
// wrong-side hits; toi = t_impact on a hit, -1 otherwise.
template <int DIM>
void ctcd_vf(const double *V0, const double *V1, const int *sten, long long n, double eta, int *ret, double *toi)
{
    typedef typename mcl::NarrowPhaseCTCD<double, DIM>::VecType Vec;
    for (long long s = 0; s < n; ++s) {
        Vec x0[DIM + 1], x1[DIM + 1];
        for (int i = 0; i < DIM + 1; ++i)
            for (int k = 0; k < DIM; ++k) {
                x0[i][k] = V0[size_t(sten[4 * s + i]) * DIM + k];
                x1[i][k] = V1[size_t(sten[4 * s + i]) * DIM + k];
            }
        double t = -1;
        const int h = mcl::NarrowPhaseCTCD<double, DIM>::query_ccd_vf(x0, x1, eta, true, t);
        ret[s] = h;
        toi[s] = h == 1 ? t : -1.0;
    }
}

} // namespace

extern "C" {

// The reference's polynomial root finder (ccd_internal/rpoly.h, a
// Jenkins-Traub RPOLY), as findIntervals calls it (CTCD.cpp:148): op in
// descending powers (modified in place, as the reference lets it), all
// roots' real and imaginary parts.  Returns its root count.
int ref_rpoly(double *op, int degree, double *re, double *im)
{
    mcl::RootFinder rf;
    return rf.rpoly(op, degree, re, im);
}

void ref_ctcd_vf(int dim, const double *V0, const double *V1, const int *sten, long long n, double eta, int *ret,
                 double *toi)
{
    if (dim == 3) ctcd_vf<3>(V0, V1, sten, n, eta, ret, toi);
    else ctcd_vf<2>(V0, V1, sten, n, eta, ret, toi);
}

// update(V0,V1,P) + traverse(V0,V1,P) with recording hooks.  flags: see F_*.
int ref_run(int dim, const double *V0, const double *V1, const int *P, int np, int pdim,
            double box_eta, double vf_eta, double ee_eta, int flags, const int *active)
{
    if (flags & F_FLOAT) {
        if (dim == 3) return run<float, 3>(V0, V1, P, np, pdim, box_eta, vf_eta, ee_eta, flags, active);
        if (dim == 2) return run<float, 2>(V0, V1, P, np, pdim, box_eta, vf_eta, ee_eta, flags, active);
        return -1;
    }
    if (dim == 3) return run<double, 3>(V0, V1, P, np, pdim, box_eta, vf_eta, ee_eta, flags, active);
    if (dim == 2) return run<double, 2>(V0, V1, P, np, pdim, box_eta, vf_eta, ee_eta, flags, active);
    return -1;
}

long long ref_count(int which)
{
    switch (which) {
    case 0: return (long long)g_state.cand.size();
    case 1: return (long long)g_state.hits.size();
    case 2: return (long long)g_state.disc.size();
    }
    return -1;
}

void ref_copy_candidates(int *sten, unsigned char *is_vf)
{
    for (size_t i = 0; i < g_state.cand.size(); ++i) {
        std::memcpy(sten + 4 * i, g_state.cand[i].s, sizeof(int) * 4);
        is_vf[i] = g_state.cand[i].is_vf;
    }
}

void ref_copy_hits(int *sten, unsigned char *is_vf, double *toi)
{
    for (size_t i = 0; i < g_state.hits.size(); ++i) {
        std::memcpy(sten + 4 * i, g_state.hits[i].s, sizeof(int) * 4);
        is_vf[i] = g_state.hits[i].is_vf;
        toi[i] = g_state.hits[i].toi;
    }
}

void ref_copy_discrete(int *pairs)
{
    for (size_t i = 0; i < g_state.disc.size(); ++i) { pairs[2 * i] = g_state.disc[i].a; pairs[2 * i + 1] = g_state.disc[i].b; }
}

// Leaf data of the last ref_run: boxes (np x 6 x dim) and flags (np x 7).
void ref_copy_leaves(double *boxes, int *flags)
{
    std::memcpy(boxes, g_state.boxes.data(), g_state.boxes.size() * sizeof(double));
    std::memcpy(flags, g_state.flags.data(), g_state.flags.size() * sizeof(int));
}

// NarrowPhaseACCD::query_ccd_vf / query_ccd_ee on caller-given stencils
// (NarrowPhase.cpp:609-631), the reference's own ACCD.
void ref_accd(int dim, const double *V0, const double *V1, const int *sten, const unsigned char *is_vf,
              long long n, double vf_eta, double ee_eta, int *hit, double *toi)
{
    if (dim == 3) accd<3>(V0, V1, sten, is_vf, n, vf_eta, ee_eta, hit, toi);
    else accd<2>(V0, V1, sten, is_vf, n, vf_eta, ee_eta, hit, toi);
}

// NarrowPhase<double,3>::discrete_tri_tri / NarrowPhase<double,2>::discrete_edge_edge
// on V (no shared-vertex rejection: that lives in BVHTree::default_discrete_test).
void ref_discrete(int dim, const double *V, const int *P, const int *pairs, long long n, int *out)
{
    for (long long s = 0; s < n; ++s) {
        const int *p0 = P + size_t(pairs[2 * s]) * dim, *p1 = P + size_t(pairs[2 * s + 1]) * dim;
        if (dim == 3) {
            Eigen::Vector3d a[3], b[3];
            for (int i = 0; i < 3; ++i) for (int k = 0; k < 3; ++k) { a[i][k] = V[size_t(p0[i]) * 3 + k]; b[i][k] = V[size_t(p1[i]) * 3 + k]; }
            out[s] = mcl::NarrowPhase<double, 3>::discrete_tri_tri(a, b) ? 1 : 0;
        } else {
            Eigen::Vector2d a[2], b[2];
            for (int i = 0; i < 2; ++i) for (int k = 0; k < 2; ++k) { a[i][k] = V[size_t(p0[i]) * 2 + k]; b[i][k] = V[size_t(p1[i]) * 2 + k]; }
            out[s] = mcl::NarrowPhase<double, 2>::discrete_edge_edge(a, b) ? 1 : 0;
        }
    }
}

// Timing run of the reference's default path: hooks are no-op atomic
// counters (filter_pair and narrow_phase unset, as in the reference's
// defaults).  Times: first update (builds representative flags), a second
// update with the same P, and traverse.  Returns the number of CCD hits.
long long ref_time(int dim, const double *V0, const double *V1, const double *V1b, const int *P, int np, int pdim,
                   double eta, int threaded, double *ms_update_first, double *ms_update_again,
                   double *ms_traverse, long long *n_discrete)
{
    using clk = std::chrono::steady_clock;
    std::atomic<long long> nh(0), nd(0);
    auto go = [&](auto &tree) {
        tree.options.box_eta = eta; tree.options.vf_ccd_eta = eta; tree.options.ee_ccd_eta = eta;
        tree.options.threaded = threaded != 0;
        tree.append_pair = [&](const Eigen::Vector4i &, bool, const double &) { nh.fetch_add(1, std::memory_order_relaxed); };
        tree.append_discrete = [&](int, int) -> bool { nd.fetch_add(1, std::memory_order_relaxed); return false; };
        auto t0 = clk::now();
        tree.update(V0, V1, P, np, pdim);
        auto t1 = clk::now();
        tree.update(V0, V1b ? V1b : V1, P, np, pdim);
        auto t2 = clk::now();
        nh = 0; nd = 0;
        tree.traverse(V0, V1b ? V1b : V1, P);
        auto t3 = clk::now();
        *ms_update_first = std::chrono::duration<double, std::milli>(t1 - t0).count();
        *ms_update_again = std::chrono::duration<double, std::milli>(t2 - t1).count();
        *ms_traverse = std::chrono::duration<double, std::milli>(t3 - t2).count();
    };
    if (dim == 3) { mcl::BVHTree<double, 3> t; go(t); }
    else { mcl::BVHTree<double, 2> t; go(t); }
    *n_discrete = nd.load();
    return nh.load();
}

// The benchmark step on the reference, repeated: one untimed first update
// (V1a), then per step i update(V0, V1[i % 2], P) with V1[0] = V1b, V1[1] =
// V1a, and traverse; hooks are no-op counters (filter_pair and narrow_phase
// unset, as in the reference's defaults).  ms[i] = update + traverse of step
// i.  stencils[i] = the candidate stencils of that step, counted in an extra
// untimed traverse per draw with a counting filter_pair.
void ref_time_steps(int dim, const double *V0, const double *V1a, const double *V1b, const int *P, int np, int pdim,
                    double eta, int steps, double *ms, long long *stencils)
{
    using clk = std::chrono::steady_clock;
    std::atomic<long long> nh(0), nd(0), nc(0);
    auto go = [&](auto &tree) {
        tree.options.box_eta = eta; tree.options.vf_ccd_eta = eta; tree.options.ee_ccd_eta = eta;
        tree.append_pair = [&](const Eigen::Vector4i &, bool, const double &) { nh.fetch_add(1, std::memory_order_relaxed); };
        tree.append_discrete = [&](int, int) -> bool { nd.fetch_add(1, std::memory_order_relaxed); return false; };
        const double *V1s[2] = {V1b, V1a};
        long long per_draw[2] = {-1, -1};
        tree.update(V0, V1a, P, np, pdim);
        for (int i = 0; i < steps; ++i) {
            const double *V1 = V1s[i % 2];
            auto t0 = clk::now();
            tree.update(V0, V1, P, np, pdim);
            tree.traverse(V0, V1, P);
            auto t1 = clk::now();
            ms[i] = std::chrono::duration<double, std::milli>(t1 - t0).count();
            if (per_draw[i % 2] < 0) {
                nc = 0;
                tree.filter_pair = [&](const Eigen::Vector4i &, bool) -> bool { nc.fetch_add(1, std::memory_order_relaxed); return false; };
                tree.traverse(V0, V1, P);
                tree.filter_pair = nullptr;
                per_draw[i % 2] = nc.load();
            }
            stencils[i] = per_draw[i % 2];
        }
    };
    if (dim == 3) { mcl::BVHTree<double, 3> t; go(t); }
    else { mcl::BVHTree<double, 2> t; go(t); }
}

int ref_threads() { return tbb::compat_thread_count(); }

} // extern "C"
