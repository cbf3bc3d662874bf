// Bulk narrow phase that never allocates device memory.
//
// mclccd_narrow_phase_bulk needs scratch memory beyond its inputs and
// outputs: a device status word that the kernel sets when a stencil names a
// vertex outside [0, nv), and -- when the caller's arrays are in host memory
// -- device copies of V0, V1, the stencils and the two outputs.  It gets that
// scratch from cudaMallocAsync on every call.  Some callers cannot allocate:
// simulation or real-time loops that run on a fixed device-memory budget
// (cudaMalloc/cudaFree can stall on device-wide synchronisation and fragment
// the budget), processes where another allocator (for example a framework's
// caching allocator) already reserves the device memory, and plugins whose
// host application forbids device allocations from third-party code.  For
// them, mclccd_narrow_phase_bulk_static takes the same arguments and puts the
// scratch in the fixed array below instead.
//
// The array is a file-scope __device__ array of MCLCCD_STATIC_SCRATCH_BYTES
// (32 MiB); every GPU that loads this library holds it until the process
// exits.  All calls share it and it keeps the last call's contents: the
// status word is cleared at the start of each call, and calls that overlap on
// the GPU (two streams, or two host threads) race on it.
#include "../../include/mclccd_b200.h"
#include "kernels.cuh"

#include <mutex>

namespace {

constexpr size_t kScratchBytes = MCLCCD_STATIC_SCRATCH_BYTES;
constexpr size_t kAlign = 256;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_static_scratch[kScratchBytes];

// Device address of g_static_scratch per device.  In host code the symbol is
// only a host-side stand-in, so the address is looked up with
// cudaGetSymbolAddress once per device, with that device current, and kept
// for the life of the process: a reset of the device's primary context
// (cudaDeviceReset) would leave it stale, which the header documents.
std::mutex g_mu;
void *g_addr[kMaxDevices] = {};

int scratch_address(void **out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return MCLCCD_ERR_CUDA;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess || !p) { cudaGetLastError(); return MCLCCD_ERR_CUDA; }
        g_addr[dev] = p;
    }
    *out = g_addr[dev];
    return MCLCCD_OK;
}

size_t up(size_t x) { return (x + kAlign - 1) & ~(kAlign - 1); }

} // namespace

extern "C" int mclccd_narrow_phase_bulk_static(int dim, const double *V0, const double *V1, int nv, const int *sten,
                                               const unsigned char *is_vf, long long n, double vf_ccd_eta,
                                               double ee_ccd_eta, double *out_toi, int *out_hit, int mem_kind,
                                               void *stream)
{
    using mclccd::Counters;
    if ((dim != 2 && dim != 3) || n < 0 || nv < 0) return MCLCCD_ERR_INVALID;
    if (mem_kind != MCLCCD_MEM_HOST && mem_kind != MCLCCD_MEM_DEVICE) return MCLCCD_ERR_INVALID;
    if (!(vf_ccd_eta >= 0) || !(ee_ccd_eta >= 0)) return MCLCCD_ERR_INVALID;
    if (n == 0) return MCLCCD_OK;
    if (!V0 || !V1 || !sten || !is_vf || !out_toi || !out_hit || nv == 0) return MCLCCD_ERR_INVALID;

    // Layout inside the static array: [status word | host-mode staging].
    const size_t vbytes = sizeof(double) * (size_t)nv * dim;
    const size_t off_v0 = up(sizeof(Counters));
    size_t off_v1 = 0, off_s = 0, off_f = 0, off_t = 0, off_h = 0, total = off_v0;
    if (mem_kind == MCLCCD_MEM_HOST) {
        off_v1 = off_v0 + up(vbytes);
        off_s = off_v1 + up(vbytes);
        off_f = off_s + up(sizeof(int) * 4 * (size_t)n);
        off_t = off_f + up((size_t)n);
        off_h = off_t + up(sizeof(double) * (size_t)n);
        total = off_h + up(sizeof(int) * (size_t)n);
    }
    if (total > kScratchBytes) return MCLCCD_ERR_SCRATCH_LIMIT;

    void *base_v = nullptr;
    if (int rc = scratch_address(&base_v)) return rc;
    char *base = static_cast<char *>(base_v);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    Counters *cnt = reinterpret_cast<Counters *>(base);
    const double *dV0 = V0, *dV1 = V1;
    const int *ds = sten;
    const unsigned char *df = is_vf;
    double *dt = out_toi;
    int *dh = out_hit;
    cudaError_t e = cudaMemsetAsync(cnt, 0, sizeof(Counters), st);
    if (e == cudaSuccess && mem_kind == MCLCCD_MEM_HOST) {
        dV0 = reinterpret_cast<const double *>(base + off_v0);
        dV1 = reinterpret_cast<const double *>(base + off_v1);
        ds = reinterpret_cast<const int *>(base + off_s);
        df = reinterpret_cast<const unsigned char *>(base + off_f);
        dt = reinterpret_cast<double *>(base + off_t);
        dh = reinterpret_cast<int *>(base + off_h);
        e = cudaMemcpyAsync((void *)dV0, V0, vbytes, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync((void *)dV1, V1, vbytes, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync((void *)ds, sten, sizeof(int) * 4 * (size_t)n, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync((void *)df, is_vf, (size_t)n, cudaMemcpyHostToDevice, st);
    }
    if (e == cudaSuccess) {
        mclccd::launch_accd_bulk(dim, ds, df, n, dV0, dV1, nv, vf_ccd_eta, ee_ccd_eta, dt, dh, cnt, st);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && mem_kind == MCLCCD_MEM_HOST) {
        e = cudaMemcpyAsync(out_toi, dt, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(out_hit, dh, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, st);
    }
    unsigned err = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&err, &cnt->err, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) { cudaGetLastError(); return MCLCCD_ERR_CUDA; }
    return (err & mclccd::kErrBadIndex) ? MCLCCD_ERR_INVALID : MCLCCD_OK;
}
