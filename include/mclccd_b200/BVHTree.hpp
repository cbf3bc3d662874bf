// Drop-in C++ replacement for mclccd's mcl::BVHTree<T, DIM>, T = double or
// float, DIM = 2 or 3 (include/MCL/BVHTree.hpp; instantiations
// BVHTree.cpp:504-507), running the CCD path on the GPU through the C ABI in
// include/mclccd_b200.h.  Link with libmclccd_b200.so.  float trees widen
// their coordinates exactly to double on the device and run the FP64 path;
// their toi is that FP64 toi rounded down to float (never later).
//
// Same members as the reference: Options (same fields and defaults),
// update(), traverse(), and the hooks append_pair, append_discrete,
// filter_pair and narrow_phase.  After traverse() the hooks are called on the
// host, fed from the device result buffers:
//   * append_pair(sten, is_vf, toi) once per CCD hit (toi >= 0);
//   * append_discrete(p0, p1) once per discrete pair until it returns true;
//   * filter_pair / narrow_phase, when set, are applied on the host to the
//     candidate stencils (the default device ACCD scores the survivors when
//     only filter_pair is set).
// With options.threaded (the default, as in the reference, whose TBB
// traversal calls these hooks from its worker threads) append_pair,
// filter_pair and narrow_phase are called from several host threads at once,
// so they must be thread-safe, as the reference requires; an exception
// thrown by one is rethrown by traverse().  With threaded = false every hook
// runs on the calling thread, in order.  append_discrete always runs on the
// calling thread, so that returning true stops the dispatch exactly.
// EE stencils and discrete pairs come with the lower primitive index first.
// Errors throw mcl::CCDError (the reference asserts or silently returns).
//
// traverse(BVHTraverse<T, DIM>*) runs a visitor over a host copy of the
// tree, with the reference's types (BVHTraverse, BVHLeaf, BoundingBox) and
// Eigen's BVIntersect order: a node's child volumes are offered to
// intersectVolume, then its leaves to intersectObject (true stops).
// Volumes are the FP32 node boxes rounded outward (never smaller than the
// reference's merged boxes); leaves carry their exact FP64 boxes.
//
// traverse(V0, V1, P) given the very arrays (the same pointers) of the last
// update reuses their device copies instead of copying them again.
#pragma once

#include "../mclccd_b200.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <exception>
#include <limits>
#include <memory>
#include <mutex>
#include <thread>
#include <type_traits>
#include <functional>
#include <stdexcept>
#include <string>
#include <vector>

#if defined(__has_include)
#if __has_include(<Eigen/Core>)
#include <Eigen/Core>
#define MCLCCD_B200_HAVE_EIGEN 1
#endif
#endif

namespace mcl {

#ifdef MCLCCD_B200_HAVE_EIGEN
typedef Eigen::Vector4i Stencil;
#else
typedef std::array<int, 4> Stencil;
#endif

#ifdef MCLCCD_B200_HAVE_EIGEN
template <typename T, int DIM>
using AlignedBoxT = Eigen::AlignedBox<T, DIM>;
typedef Eigen::Vector3i RepFlags;
inline RepFlags rep_all() { return RepFlags(1, 1, 1); }
#else
// Without Eigen: the part of Eigen::AlignedBox<T, DIM> a visitor uses.
template <typename T, int DIM>
class AlignedBoxT {
public:
    typedef std::array<T, DIM> VectorType;
    AlignedBoxT() { setEmpty(); }
    VectorType &min() { return lo_; }
    VectorType &max() { return hi_; }
    const VectorType &min() const { return lo_; }
    const VectorType &max() const { return hi_; }
    void setEmpty()
    {
        lo_.fill(std::numeric_limits<T>::max());
        hi_.fill(std::numeric_limits<T>::lowest());
    }
    bool isEmpty() const
    {
        for (int k = 0; k < DIM; ++k)
            if (hi_[k] < lo_[k]) return true;
        return false;
    }
    bool contains(const VectorType &p) const
    {
        for (int k = 0; k < DIM; ++k)
            if (p[k] < lo_[k] || hi_[k] < p[k]) return false;
        return true;
    }
    bool intersects(const AlignedBoxT &b) const
    {
        for (int k = 0; k < DIM; ++k)
            if (hi_[k] < b.lo_[k] || b.hi_[k] < lo_[k]) return false;
        return true;
    }

private:
    VectorType lo_, hi_;
};
typedef std::array<int, 3> RepFlags;
inline RepFlags rep_all() { return RepFlags{{1, 1, 1}}; }
#endif

// BVHLeaf.hpp:12-28: the swept box, with the t = 0 and t = 1 boxes and the
// active flag.
template <typename T, int DIM>
class BoundingBox : public AlignedBoxT<T, DIM> {
public:
    bool active = true;
    AlignedBoxT<T, DIM> t0, t1;
    virtual ~BoundingBox() {}
};

// BVHLeaf.hpp:30-52: primitive index, representative vertex / edge flags, box.
template <typename T, int DIM>
class BVHLeaf {
public:
    typedef BoundingBox<T, DIM> BoxType;
    int idx = -1;
    RepFlags v = rep_all(), e = rep_all();
    BoxType box;
    virtual ~BVHLeaf() {}
};

// BVHTree.hpp:17-27: visitor of traverse(BVHTraverse *).
template <typename T, int DIM>
class BVHTraverse {
public:
    typedef BVHLeaf<T, DIM> ObjectType;
    typedef typename BVHLeaf<T, DIM>::BoxType VolumeType;
    virtual ~BVHTraverse() {}
    virtual bool intersectVolume(const VolumeType &) = 0;   // true: descend into this volume
    virtual bool intersectObject(const ObjectType &) = 0;   // true: stop the traversal
};

class CCDError : public std::runtime_error {
public:
    CCDError(int status, const std::string &msg) : std::runtime_error(msg), status(status) {}
    int status;
};

template <typename T, int DIM>
class BVHTree {
    static_assert(DIM == 2 || DIM == 3, "mcl::BVHTree<T, DIM>: DIM must be 2 or 3");
    static_assert(std::is_same<T, double>::value || std::is_same<T, float>::value,
                  "mcl::BVHTree<T, DIM>: T must be double or float");
    static constexpr bool kFloat = std::is_same<T, float>::value;

public:
    struct Options {
        T box_eta = T(1e-6);     // padding of tree boxes
        T vf_ccd_eta = T(1e-6);  // gap for vf narrowphase <= box_eta
        T ee_ccd_eta = T(1e-6);  // gap for ee narrowphase <= box_eta
        bool reptri = true;        // representative triangles
        bool threaded = true;      // accepted; the GPU path is always parallel
        bool discrete = true;      // discrete check ff/ee at V1
        bool continuous = true;    // ccd check from V0 to V1
        bool vf_one_sided = false; // VF narrow phase: CTCD with the wrong-side test
        bool ee_robust = true;     // unused by ACCD, as in the reference
    } options;

    std::function<void(const Stencil &sten, bool is_vf, const T &toi)> append_pair;
    std::function<bool(int p0, int p1)> append_discrete;
    std::function<bool(const Stencil &sten, bool is_vf)> filter_pair;
    std::function<T(const Stencil &sten, bool is_vf)> narrow_phase;

    BVHTree() { check(mclccd_create(DIM, &h_)); }
    ~BVHTree() { if (h_) mclccd_destroy(h_); }
    BVHTree(const BVHTree &) = delete;
    BVHTree &operator=(const BVHTree &) = delete;

    // Reference signature (BVHTree.hpp:81-82).  It carries no vertex count, so
    // the count is taken as 1 + the largest index in P, found on the device
    // (float trees, whose coordinates are staged first, scan P here).
    void update(const T *V0, const T *V1, const int *P, int np, int pdim, const int *active = nullptr)
    {
        int nv = 0;
        if constexpr (kFloat)
            for (long long i = 0; i < (long long)np * pdim; ++i) nv = std::max(nv, P[i] + 1);
        update(V0, V1, nv, P, np, pdim, active, MCLCCD_MEM_HOST);
        upd_V0_ = V0;
        upd_V1_ = V1;
        upd_P_ = P;
    }

    // With an explicit vertex count; mem_kind MCLCCD_MEM_DEVICE takes device
    // pointers (no host copies at all).
    void update(const T *V0, const T *V1, int nv, const int *P, int np, int pdim, const int *active,
                int mem_kind)
    {
        push_options();
        int rc;
        if constexpr (kFloat) rc = mclccd_update_f32(h_, V0, V1, nv, P, np, pdim, active, mem_kind);
        else rc = mclccd_update(h_, V0, V1, nv, P, np, pdim, active, mem_kind);
        pull_options();
        check(rc);
        if (nv == 0) check(mclccd_tree_size(h_, &nv, nullptr, nullptr));
        nv_ = nv;
        np_ = np;
        mem_ = mem_kind;
        upd_V0_ = upd_V1_ = nullptr;
        upd_P_ = nullptr;
        ++rev_;
    }

    // Reference signature (BVHTree.hpp:86).  Runs the device pipeline on the
    // given arrays (same side as the last update), then calls the hooks.
    void traverse(const T *V0, const T *V1, const int *P) const
    {
        // the arrays of the last update: their device copies are current
        if (V0 && V0 == upd_V0_ && V1 == upd_V1_ && P == upd_P_ && mem_ == MCLCCD_MEM_HOST &&
            !(filter_pair && !narrow_phase)) {
            traverse();
            return;
        }
        auto *self = const_cast<BVHTree *>(this);
        self->push_options();
        if constexpr (!kFloat) {
            if (self->streamed(V0, V1, P)) return;
        }
        if constexpr (kFloat) check(mclccd_traverse_f32(h_, V0, V1, nv_, P, mem_));
        else check(mclccd_traverse(h_, V0, V1, nv_, P, mem_));
        self->dispatch(V0, V1);
    }

    // Re-runs traverse on the arrays of the last update (no copies).
    void traverse() const
    {
        auto *self = const_cast<BVHTree *>(this);
        self->push_options();
        if constexpr (!kFloat) {
            if (self->streamed(nullptr, nullptr, nullptr)) return;
        }
        if constexpr (kFloat) check(mclccd_traverse_f32(h_, nullptr, nullptr, 0, nullptr, mem_));
        else check(mclccd_traverse(h_, nullptr, nullptr, 0, nullptr, mem_));
        self->dispatch(nullptr, nullptr);
    }

    // Reference signature (BVHTree.hpp:96, BVHTree.cpp:162-166): the visitor
    // over a host copy of the tree (fetched once per update).
    void traverse(BVHTraverse<T, DIM> *traverser) const
    {
        if (!traverser || np_ < 1) return;
        auto *self = const_cast<BVHTree *>(this);
        self->fetch_tree();
        if (np_ == 1) {
            traverser->intersectObject(self->leaf_object(0));
            return;
        }
        std::vector<int> pending(1, 0);
        while (!pending.empty()) {
            const int node = pending.back();
            pending.pop_back();
            const HostNode &nd = tree_nodes_[node];
            const int split = nd.d[0], meta = nd.d[1];
            for (int side = 0; side < 2; ++side)
                if (!(meta & (1 << side)) && traverser->intersectVolume(node_volume(nd, side)))
                    pending.push_back(split + side);
            for (int side = 0; side < 2; ++side)
                if ((meta & (1 << side)) && traverser->intersectObject(self->leaf_object(split + side))) return;
        }
    }

#ifdef MCLCCD_B200_HAVE_EIGEN
    // Eigen overloads (BVHTree.hpp:151-186).  Where the reference makes
    // RowMajor copies, matrices with contiguous storage in either order
    // (e.g. the default column-major MatrixXd / MatrixXi) are passed as they
    // are, with their layout, and converted on the device
    // (mclccd_update_ex); other expressions are copied to RowMajor first.
    template <typename DerivedV, typename DerivedP>
    void update(const Eigen::MatrixBase<DerivedV> &V0, const Eigen::MatrixBase<DerivedV> &V1,
                const Eigen::MatrixBase<DerivedP> &P, const Eigen::VectorXi &active = Eigen::VectorXi())
    {
        if (V0.rows() != V1.rows()) throw CCDError(MCLCCD_ERR_INVALID, "V0 and V1 row counts differ");
        const int *act = active.size() == V0.rows() ? active.data() : nullptr;
        unsigned f = 0;
        if (direct_layout(V0, V1, P, f)) {
            push_options();
            const int rc = mclccd_update_ex(h_, V0.derived().data(), V1.derived().data(), (int)V0.rows(),
                                            P.derived().data(), (int)P.rows(), (int)P.cols(), act, MCLCCD_MEM_HOST, f);
            pull_options();
            check(rc);
            nv_ = (int)V0.rows();
            np_ = (int)P.rows();
            mem_ = MCLCCD_MEM_HOST;
            return;
        }
        RowV v0 = V0.template cast<T>(), v1 = V1.template cast<T>();
        RowP p = P.template cast<int>();
        update(v0.data(), v1.data(), (int)v0.rows(), p.data(), (int)p.rows(), (int)p.cols(), act, MCLCCD_MEM_HOST);
    }
    template <typename DerivedV, typename DerivedP>
    void traverse(const Eigen::MatrixBase<DerivedV> &V0, const Eigen::MatrixBase<DerivedV> &V1,
                  const Eigen::MatrixBase<DerivedP> &P)
    {
        if (V0.rows() != V1.rows()) throw CCDError(MCLCCD_ERR_INVALID, "V0 and V1 row counts differ");
        unsigned f = 0;
        // a filter_pair without narrow_phase reads V0/V1 on the host as rows
        if (!(filter_pair && !narrow_phase) && direct_layout(V0, V1, P, f)) {
            push_options();
            check(mclccd_traverse_ex(h_, V0.derived().data(), V1.derived().data(), (int)V0.rows(), P.derived().data(),
                                     MCLCCD_MEM_HOST, f));
            dispatch(nullptr, nullptr);
            return;
        }
        RowV v0 = V0.template cast<T>(), v1 = V1.template cast<T>();
        RowP p = P.template cast<int>();
        traverse(v0.data(), v1.data(), p.data());
    }
#endif

    // ---- results of the last traverse, as arrays ---------------------------
    long long num_hits() const { long long n = 0; check(mclccd_counts(h_, &n, nullptr, nullptr, nullptr, nullptr)); return n; }
    long long num_discrete() const { long long n = 0; check(mclccd_counts(h_, nullptr, &n, nullptr, nullptr, nullptr)); return n; }
    void hits(std::vector<int> &sten, std::vector<unsigned char> &is_vf, std::vector<double> &toi) const
    {
        const long long n = num_hits();
        sten.resize(4 * n); is_vf.resize(n); toi.resize(n);
        check(mclccd_get_hits(h_, MCLCCD_MEM_HOST, n, sten.data(), is_vf.data(), toi.data()));
    }
    void discrete(std::vector<int> &pairs) const
    {
        const long long n = num_discrete();
        pairs.resize(2 * n);
        check(mclccd_get_discrete(h_, MCLCCD_MEM_HOST, n, pairs.data()));
    }
    void candidates(std::vector<int> &sten, std::vector<unsigned char> &is_vf) const
    {
        long long nvf = 0, nee = 0;
        check(mclccd_counts(h_, nullptr, nullptr, &nvf, &nee, nullptr));
        sten.resize(4 * (nvf + nee)); is_vf.resize(nvf + nee);
        check(mclccd_get_candidates(h_, MCLCCD_MEM_HOST, nvf + nee, sten.data(), is_vf.data()));
    }
    mclccd_tree *handle() const { return h_; }

private:
#ifdef MCLCCD_B200_HAVE_EIGEN
    typedef Eigen::Matrix<T, Eigen::Dynamic, DIM, Eigen::RowMajor> RowV;
    typedef Eigen::Matrix<int, Eigen::Dynamic, Eigen::Dynamic, Eigen::RowMajor> RowP;

    // 0: contiguous rows, 1: contiguous columns, -1: neither.
    template <typename D>
    static int layout_of(const Eigen::MatrixBase<D> &m)
    {
        const D &d = m.derived();
        if (d.innerStride() != 1) return -1;
        if (D::IsRowMajor) return d.outerStride() == d.cols() ? 0 : -1;
        return d.outerStride() == d.rows() ? 1 : -1;
    }
    // Whether V0, V1 (scalar T, DIM columns, same layout) and P (int) can be
    // passed as they are; f receives the mclccd_update_ex input flags.
    template <typename DV, typename DP>
    static bool direct_layout(const Eigen::MatrixBase<DV> &V0, const Eigen::MatrixBase<DV> &V1,
                              const Eigen::MatrixBase<DP> &P, unsigned &f)
    {
        if constexpr (std::is_same<typename DV::Scalar, T>::value && std::is_same<typename DP::Scalar, int>::value &&
                      (int(DV::Flags) & Eigen::DirectAccessBit) != 0 && (int(DP::Flags) & Eigen::DirectAccessBit) != 0) {
            const int l0 = layout_of(V0), l1 = layout_of(V1), lp = layout_of(P);
            if (V0.cols() != DIM || V1.cols() != DIM || l0 < 0 || l0 != l1 || lp < 0) return false;
            f = (kFloat ? MCLCCD_IN_F32 : 0u) | (l0 == 1 ? MCLCCD_IN_V_COLMAJOR : 0u) |
                (lp == 1 ? MCLCCD_IN_P_COLMAJOR : 0u);
            return true;
        } else {
            (void)V0; (void)V1; (void)P; (void)f;
            return false;
        }
    }
#endif
    mclccd_tree *h_ = nullptr;
    int nv_ = 0, np_ = 0, mem_ = MCLCCD_MEM_HOST;
    const T *upd_V0_ = nullptr, *upd_V1_ = nullptr;   // host arrays of the last update (reference signature)
    const int *upd_P_ = nullptr;
    long long rev_ = 0, tree_rev_ = -1;                // update count / the host tree copy's
    // hit staging for streamed(), page-locked, kept across calls (capacity
    // from the last count)
    struct Pinned {
        void *p = nullptr;
        ~Pinned() { if (p) mclccd_host_free(p); }
    };
    Pinned out_s_, out_v_, out_t_;
    long long out_cap_ = 0;
    // host copy of the tree for visitors
    struct HostNode {
        float l[12], r[12];
        int d[4], pad[4];
    };
    static_assert(sizeof(HostNode) == 128, "node record is 128 bytes");
    std::vector<HostNode> tree_nodes_;
    std::vector<double> tree_box_;
    std::vector<int> tree_prim_;
    std::vector<unsigned char> tree_flags_;

    void fetch_tree()
    {
        if (tree_rev_ == rev_) return;
        tree_nodes_.resize(np_ > 1 ? np_ - 1 : 0);
        tree_box_.resize((size_t)np_ * 4 * DIM);
        tree_prim_.resize(np_);
        tree_flags_.resize(np_);
        check(mclccd_get_tree_host(h_, tree_nodes_.data(), tree_box_.data(), tree_prim_.data(), tree_flags_.data()));
        tree_rev_ = rev_;
    }
    // Child `side` of a node as a volume: FP32 t0 / t1 boxes (outward) and
    // their hull, in T.
    static BoundingBox<T, DIM> node_volume(const HostNode &nd, int side)
    {
        const float *c = side ? nd.r : nd.l;
        float t0lo[DIM], t0hi[DIM], t1lo[DIM], t1hi[DIM];
        if constexpr (DIM == 3) {
            for (int k = 0; k < 3; ++k) { t0lo[k] = c[k]; t1hi[k] = c[9 + k]; }
            t0hi[0] = c[3]; t0hi[1] = c[4]; t0hi[2] = c[5];
            t1lo[0] = c[6]; t1lo[1] = c[7]; t1lo[2] = c[8];
        } else {
            t0lo[0] = c[0]; t0lo[1] = c[1]; t0hi[0] = c[2]; t0hi[1] = c[3];
            t1lo[0] = c[4]; t1lo[1] = c[5]; t1hi[0] = c[6]; t1hi[1] = c[7];
        }
        BoundingBox<T, DIM> b;
        for (int k = 0; k < DIM; ++k) {
            b.t0.min()[k] = (T)t0lo[k]; b.t0.max()[k] = (T)t0hi[k];
            b.t1.min()[k] = (T)t1lo[k]; b.t1.max()[k] = (T)t1hi[k];
            b.min()[k] = (T)std::min(t0lo[k], t1lo[k]);
            b.max()[k] = (T)std::max(t0hi[k], t1hi[k]);
        }
        b.active = ((nd.d[1] >> (side ? 16 : 8)) & 0xff) != 0;
        return b;
    }
    // Sorted leaf k as the reference's leaf object (exact FP64 boxes).
    BVHLeaf<T, DIM> leaf_object(int k) const
    {
        BVHLeaf<T, DIM> o;
        o.idx = tree_prim_[k];
        const unsigned f = tree_flags_[k];
        for (int j = 0; j < 3; ++j) {
            o.v[j] = (f >> j) & 1;
            o.e[j] = (f >> (3 + j)) & 1;
        }
        const double *bx = &tree_box_[(size_t)k * 4 * DIM];   // lo0, hi0, lo1, hi1
        for (int c = 0; c < DIM; ++c) {
            o.box.t0.min()[c] = (T)bx[c];
            o.box.t0.max()[c] = (T)bx[DIM + c];
            o.box.t1.min()[c] = (T)bx[2 * DIM + c];
            o.box.t1.max()[c] = (T)bx[3 * DIM + c];
            o.box.min()[c] = (T)std::min(bx[c], bx[2 * DIM + c]);
            o.box.max()[c] = (T)std::max(bx[DIM + c], bx[3 * DIM + c]);
        }
        o.box.active = (f & (1u << 6)) != 0;
        return o;
    }
    void grow_staging(long long cap)
    {
        Pinned s, v, t;
        check(mclccd_host_alloc(sizeof(int) * 4 * (size_t)cap, &s.p));
        check(mclccd_host_alloc((size_t)cap, &v.p));
        check(mclccd_host_alloc(sizeof(double) * (size_t)cap, &t.p));
        std::swap(out_s_.p, s.p);
        std::swap(out_v_.p, v.p);
        std::swap(out_t_.p, t.p);
        out_cap_ = cap;
    }

    // With only append_pair / append_discrete set: traverse with the hits
    // delivered into host staging (mclccd_traverse_out), so their copy from
    // the device overlaps the rest of the step, then call the hooks.  The
    // staging holds the previous call's count and a quarter more; hits beyond
    // it are fetched after the step.  Returns false when hooks need the
    // general path.
    bool streamed(const double *V0, const double *V1, const int *P)
    {
        if (!append_pair || filter_pair || narrow_phase) return false;
        long long nh = 0, nd = 0;
        int *s = static_cast<int *>(out_s_.p);
        unsigned char *v = static_cast<unsigned char *>(out_v_.p);
        double *t = static_cast<double *>(out_t_.p);
        check(mclccd_traverse_out(h_, V0, V1, nv_, P, mem_, s, v, t, out_cap_, &nh, nullptr, 0, &nd, MCLCCD_MEM_HOST));
        if (nh > out_cap_) {
            grow_staging(nh + nh / 4 + 1024);
            s = static_cast<int *>(out_s_.p);
            v = static_cast<unsigned char *>(out_v_.p);
            t = static_cast<double *>(out_t_.p);
            check(mclccd_get_hits(h_, MCLCCD_MEM_HOST, nh, s, v, t));
        }
        for_each_result(nh, [&](long long i) { append_pair(make_stencil(&s[4 * i]), v[i] != 0, to_toi(t[i])); });
        dispatch_discrete();
        return true;
    }
    // f(i) for i in [0, n): on the calling thread, or with options.threaded
    // over the host's hardware threads in contiguous slices (results of at
    // least kMinPerThread per thread).  The first exception a slice throws is
    // rethrown here after every slice has stopped.
    static constexpr long long kMinPerThread = 1 << 15;
    template <class F>
    void for_each_result(long long n, F &&f) const
    {
        const long long hw = std::max<long long>(1, (long long)std::thread::hardware_concurrency());
        const long long nt = options.threaded ? std::min(hw, n / kMinPerThread) : 1;
        if (nt <= 1) {
            for (long long i = 0; i < n; ++i) f(i);
            return;
        }
        std::exception_ptr err;
        std::mutex err_m;
        auto slice = [&](long long k) {
            try {
                for (long long i = n * k / nt, e = n * (k + 1) / nt; i < e; ++i) f(i);
            } catch (...) {
                std::lock_guard<std::mutex> g(err_m);
                if (!err) err = std::current_exception();
            }
        };
        std::vector<std::thread> th;
        th.reserve((size_t)nt - 1);
        for (long long k = 1; k < nt; ++k) th.emplace_back(slice, k);
        slice(0);
        for (auto &x : th) x.join();
        if (err) std::rethrow_exception(err);
    }
    void dispatch_discrete()
    {
        if (append_discrete && options.discrete) {
            std::vector<int> d;
            discrete(d);
            for (size_t i = 0; i < d.size() / 2; ++i)
                if (append_discrete(d[2 * i], d[2 * i + 1])) break;
        }
    }

    void check(int rc) const
    {
        if (rc != MCLCCD_OK) {
            const char *m = h_ ? mclccd_last_error(h_) : "";
            throw CCDError(rc, std::string(mclccd_status_string(rc)) + (m && *m ? std::string(": ") + m : ""));
        }
    }
    void push_options()
    {
        unsigned f = 0;
        if (options.reptri) f |= MCLCCD_OPT_REPTRI;
        if (options.threaded) f |= MCLCCD_OPT_THREADED;
        if (options.discrete) f |= MCLCCD_OPT_DISCRETE;
        if (options.continuous) f |= MCLCCD_OPT_CONTINUOUS;
        if (options.vf_one_sided) f |= MCLCCD_OPT_VF_ONE_SIDED;
        if (options.ee_robust) f |= MCLCCD_OPT_EE_ROBUST;
        check(mclccd_set_options(h_, (double)options.box_eta, (double)options.vf_ccd_eta, (double)options.ee_ccd_eta,
                                 f));
    }
    void pull_options()
    {
        double b = 0, v = 0, e = 0;
        mclccd_get_options(h_, &b, &v, &e, nullptr);
        options.box_eta = (T)b;
        options.vf_ccd_eta = (T)v;
        options.ee_ccd_eta = (T)e;
    }
    // A device toi (double) as T: float rounds down, so it is never later.
    static T to_toi(double t)
    {
        if constexpr (kFloat) {
            float f = (float)t;
            if ((double)f > t) f = std::nextafter(f, -std::numeric_limits<float>::infinity());
            return f;
        } else {
            return t;
        }
    }
    static Stencil make_stencil(const int *s)
    {
        Stencil t;
        for (int i = 0; i < 4; ++i) t[i] = s[i];
        return t;
    }
    void dispatch(const T *V0, const T *V1)
    {
        if (filter_pair || narrow_phase) {
            std::vector<int> cs;
            std::vector<unsigned char> cv;
            candidates(cs, cv);
            std::vector<unsigned char> skip(cv.size(), 0);
            if (filter_pair)
                for_each_result((long long)cv.size(), [&](long long i) {
                    skip[i] = filter_pair(make_stencil(&cs[4 * i]), cv[i] != 0) ? 1 : 0;
                });
            std::vector<int> ks;
            std::vector<unsigned char> kv;
            for (size_t i = 0; i < cv.size(); ++i) {
                if (skip[i]) continue;
                ks.insert(ks.end(), cs.begin() + 4 * i, cs.begin() + 4 * i + 4);
                kv.push_back(cv[i]);
            }
            std::vector<double> toi(kv.size(), -1.0);
            if (narrow_phase) {
                for_each_result((long long)kv.size(), [&](long long i) {
                    toi[i] = narrow_phase(make_stencil(&ks[4 * i]), kv[i] != 0);
                });
            } else if (!kv.empty()) {
                if (!V0 || mem_ != MCLCCD_MEM_HOST)
                    throw CCDError(MCLCCD_ERR_INVALID, "filter_pair without narrow_phase needs host V0/V1 at traverse");
                std::vector<int> hit(kv.size());
                const double *v0 = nullptr, *v1 = nullptr;
                std::vector<double> w0, w1;
                if constexpr (kFloat) {
                    w0.assign(V0, V0 + (size_t)nv_ * DIM);
                    w1.assign(V1, V1 + (size_t)nv_ * DIM);
                    v0 = w0.data();
                    v1 = w1.data();
                } else {
                    v0 = V0;
                    v1 = V1;
                }
                check(mclccd_narrow_phase_bulk_ex(DIM, v0, v1, nv_, ks.data(), kv.data(), (long long)kv.size(),
                                                  (double)options.vf_ccd_eta, (double)options.ee_ccd_eta, toi.data(),
                                                  hit.data(), MCLCCD_MEM_HOST, nullptr,
                                                  MCLCCD_PREC_FP64 | (options.vf_one_sided ? MCLCCD_BULK_VF_ONE_SIDED : 0),
                                                  nullptr));
            }
            if (append_pair)
                for_each_result((long long)kv.size(), [&](long long i) {
                    if (toi[i] >= 0) append_pair(make_stencil(&ks[4 * i]), kv[i] != 0, to_toi(toi[i]));
                });
        } else if (append_pair) {
            std::vector<int> s;
            std::vector<unsigned char> v;
            std::vector<double> t;
            hits(s, v, t);
            for_each_result((long long)v.size(), [&](long long i) {
                append_pair(make_stencil(&s[4 * i]), v[i] != 0, to_toi(t[i]));
            });
        }
        dispatch_discrete();
    }
};

} // namespace mcl
