// Onesweep LSD radix sort of (uint32 key, int32 value) pairs: one histogram
// pass over all digits, then one kernel per 8-bit digit that ranks its tile
// and scatters in a single sweep, the tile's global offset coming from a
// decoupled look-back over earlier tiles (Adinets & Merrill, "Onesweep: A
// Faster Least Significant Digit Radix Sort for GPUs", 2022).
//
// Tiles take their index from an atomic ticket, so every tile a look-back
// waits on has already started; each wait is still bounded and records
// kErrSortWait instead of spinning forever.
#include "common.cuh"
#include "kernels.cuh"

namespace mclccd {

constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;   // 4096 keys
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kRadix = 256;
constexpr unsigned kFlagAgg = 1u << 30, kFlagPrefix = 2u << 30, kValMask = (1u << 30) - 1;

int sort_num_passes(unsigned key_bits) { return (int)((key_bits + 7) / 8); }

size_t sort_scratch_bytes(int n, int passes)
{
    size_t tiles = (size_t)(n + kSortTile - 1) / kSortTile;
    // global histograms [passes][256] + tile tickets [passes] + look-back [passes][tiles][256]
    return sizeof(unsigned) * ((size_t)passes * kRadix + 32 + (size_t)passes * tiles * kRadix);
}

__global__ void k_sort_hist(const unsigned *__restrict__ keys, int n, int passes, unsigned *__restrict__ ghist)
{
    __shared__ unsigned h[4][kRadix];
    for (int t = threadIdx.x; t < 4 * kRadix; t += blockDim.x) (&h[0][0])[t] = 0;
    __syncthreads();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        unsigned k = keys[i];
        for (int p = 0; p < passes; ++p) atomicAdd(&h[p][(k >> (8 * p)) & 0xff], 1u);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < passes * kRadix; t += blockDim.x) {
        unsigned v = (&h[0][0])[t];
        if (v) atomicAdd(ghist + t, v);
    }
}

__global__ void __launch_bounds__(kSortThreads)
k_sort_pass(const unsigned *__restrict__ kin, const int *__restrict__ vin, unsigned *__restrict__ kout,
            int *__restrict__ vout, int n, int shift, const unsigned *__restrict__ ghist,
            unsigned *__restrict__ lookback, unsigned *__restrict__ ticket, Counters *cnt)
{
    __shared__ unsigned s_warp[kSortWarps][kRadix];   // per-warp digit counts -> warp offsets
    __shared__ unsigned s_base[kRadix];               // global base of this tile, per digit
    __shared__ unsigned s_scan[kRadix];
    __shared__ unsigned s_tile;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) s_tile = atomicAdd(ticket, 1u);
    for (int t = tid; t < kSortWarps * kRadix; t += kSortThreads) (&s_warp[0][0])[t] = 0;
    // exclusive scan of the global histogram of this digit
    {
        unsigned v = ghist[tid];
        s_scan[tid] = v;
        __syncthreads();
        for (int o = 1; o < kRadix; o <<= 1) {
            unsigned add = tid >= o ? s_scan[tid - o] : 0;
            __syncthreads();
            s_scan[tid] += add;
            __syncthreads();
        }
        s_base[tid] = s_scan[tid] - v;
    }
    __syncthreads();
    const unsigned tile = s_tile;
    const long long tbase = (long long)tile * kSortTile + (long long)warp * 32 * kSortItems;

    unsigned key[kSortItems];
    int val[kSortItems];
    unsigned rank[kSortItems];
#pragma unroll
    for (int it = 0; it < kSortItems; ++it) {
        long long idx = tbase + it * 32 + lane;
        bool ok = idx < n;
        key[it] = ok ? kin[idx] : 0u;
        val[it] = ok ? vin[idx] : 0;
        unsigned dig = (key[it] >> shift) & 0xff;
        unsigned peers = __match_any_sync(0xffffffffu, ok ? dig : 0x100u);
        unsigned before = __popc(peers & lanemask_lt());
        unsigned cur = ok ? s_warp[warp][dig] : 0u;
        rank[it] = cur + before;
        __syncwarp();
        if (ok && before == 0) s_warp[warp][dig] = cur + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // per digit: exclusive scan over warps (stable: warp-major order)
    unsigned total = 0;
    {
        const int d = tid;
#pragma unroll
        for (int w = 0; w < kSortWarps; ++w) { unsigned c = s_warp[w][d]; s_warp[w][d] = total; total += c; }
    }
    // decoupled look-back: publish this tile's count, add earlier tiles'
    {
        const int d = tid;
        unsigned *mine = lookback + (size_t)tile * kRadix + d;
        unsigned excl = 0;
        if (tile == 0) {
            atomicExch(mine, kFlagPrefix | (total & kValMask));
        } else {
            atomicExch(mine, kFlagAgg | (total & kValMask));
            for (long long t = (long long)tile - 1; t >= 0; --t) {
                volatile unsigned *src = lookback + (size_t)t * kRadix + d;
                unsigned w = *src;
                unsigned spins = 0;
                while ((w & ~kValMask) == 0) {
                    if (++spins > (1u << 22)) { atomicOr(&cnt->err, kErrSortWait); w = kFlagPrefix; break; }
                    __nanosleep(64);
                    w = *src;
                }
                excl += w & kValMask;
                if ((w & ~kValMask) == kFlagPrefix) break;
            }
            atomicExch(mine, kFlagPrefix | ((excl + total) & kValMask));
        }
        s_base[d] += excl;
    }
    __syncthreads();
#pragma unroll
    for (int it = 0; it < kSortItems; ++it) {
        long long idx = tbase + it * 32 + lane;
        if (idx < n) {
            unsigned dig = (key[it] >> shift) & 0xff;
            unsigned pos = s_base[dig] + s_warp[warp][dig] + rank[it];
            if (pos < (unsigned)n) {   // always true unless a look-back wait gave up
                kout[pos] = key[it];
                vout[pos] = val[it];
            }
        }
    }
}

// Sorts (keys, vals) in place (result ends in keys/vals; alt buffers are
// scratch of the same size).  scratch: sort_scratch_bytes(n, passes) bytes.
void launch_sort_pairs(unsigned *keys, int *vals, unsigned *keys_alt, int *vals_alt, int n, unsigned key_bits,
                       void *scratch, Counters *cnt, cudaStream_t st)
{
    if (n <= 1) return;
    const int passes = sort_num_passes(key_bits);
    const int tiles = (n + kSortTile - 1) / kSortTile;
    unsigned *ghist = reinterpret_cast<unsigned *>(scratch);
    unsigned *tickets = ghist + (size_t)passes * kRadix;
    unsigned *lb = tickets + 32;
    cudaMemsetAsync(scratch, 0, sort_scratch_bytes(n, passes), st);
    int hg = (n + 256 * 8 - 1) / (256 * 8);
    if (hg > 148 * 4) hg = 148 * 4;
    k_sort_hist<<<hg, 256, 0, st>>>(keys, n, passes, ghist);
    unsigned *ki = keys, *ko = keys_alt;
    int *vi = vals, *vo = vals_alt;
    for (int p = 0; p < passes; ++p) {
        k_sort_pass<<<tiles, kSortThreads, 0, st>>>(ki, vi, ko, vo, n, 8 * p, ghist + (size_t)p * kRadix,
                                                  lb + (size_t)p * tiles * kRadix, tickets + p, cnt);
        unsigned *tk = ki; ki = ko; ko = tk;
        int *tv = vi; vi = vo; vo = tv;
    }
    if (ki != keys) {
        cudaMemcpyAsync(keys, ki, sizeof(unsigned) * (size_t)n, cudaMemcpyDeviceToDevice, st);
        cudaMemcpyAsync(vals, vi, sizeof(int) * (size_t)n, cudaMemcpyDeviceToDevice, st);
    }
}

} // namespace mclccd
