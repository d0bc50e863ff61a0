// Exclusive prefix sums for the count -> scan -> fill table builders.
// Three phases per level: tile totals, a scan of the totals (recursing while
// there is more than one tile of totals), and the tile-local scan plus the
// tile offset. Deterministic: integer sums in a fixed order.
#include "dg_internal.h"

namespace dg {
namespace {

constexpr int kThreads = 512;
constexpr int kItems = 8;
constexpr int64_t kTile = int64_t(kThreads) * kItems;

template <typename In>
__device__ __forceinline__ int64_t block_sum(int64_t v) {
    __shared__ int64_t warp_sums[kThreads / 32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) warp_sums[warp] = v;
    __syncthreads();
    int64_t total = 0;
    if (threadIdx.x < 32) {
        int64_t x = threadIdx.x < kThreads / 32 ? warp_sums[threadIdx.x] : 0;
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (threadIdx.x == 0) warp_sums[0] = x;
    }
    __syncthreads();
    total = warp_sums[0];
    __syncthreads();
    return total;
}

template <typename In>
__global__ void tile_totals(const In *__restrict__ in, int64_t n, int64_t *__restrict__ totals) {
    int64_t base = int64_t(blockIdx.x) * kTile;
    int64_t v = 0;
    for (int i = 0; i < kItems; ++i) {
        int64_t k = base + int64_t(i) * kThreads + threadIdx.x;
        if (k < n) v += int64_t(in[k]);
    }
    int64_t t = block_sum<In>(v);
    if (threadIdx.x == 0) totals[blockIdx.x] = t;
}

// Each thread owns kItems consecutive elements; thread totals are scanned
// across the block with warp shuffles, then each element gets its prefix.
template <typename In>
__global__ void tile_scan(const In *__restrict__ in, int64_t *__restrict__ out, int64_t n,
                          const int64_t *__restrict__ tile_offsets) {
    __shared__ int64_t warp_prefix[kThreads / 32];
    int64_t base = int64_t(blockIdx.x) * kTile + int64_t(threadIdx.x) * kItems;
    int64_t vals[kItems];
    int64_t own = 0;
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
        int64_t k = base + i;
        vals[i] = k < n ? int64_t(in[k]) : 0;
        own += vals[i];
    }
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int64_t incl = own;
    for (int o = 1; o < 32; o <<= 1) {
        int64_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) warp_prefix[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        int64_t x = lane < kThreads / 32 ? warp_prefix[lane] : 0;
        int64_t xi = x;
        for (int o = 1; o < 32; o <<= 1) {
            int64_t y = __shfl_up_sync(0xffffffffu, xi, o);
            if (lane >= o) xi += y;
        }
        if (lane < kThreads / 32) warp_prefix[lane] = xi - x;  // exclusive
    }
    __syncthreads();
    int64_t run = tile_offsets[blockIdx.x] + warp_prefix[warp] + (incl - own);
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
        int64_t k = base + i;
        if (k < n) out[k] = run;
        run += vals[i];
    }
}

int64_t n_tiles(int64_t n) { return (n + kTile - 1) / kTile; }

template <typename In>
void scan_impl(const In *in, int64_t *out, int64_t n, int64_t *temp, cudaStream_t stream) {
    if (n <= 0) return;
    int64_t t = n_tiles(n);
    int64_t *totals = temp;
    int64_t *offsets = temp + t;
    tile_totals<In><<<unsigned(t), kThreads, 0, stream>>>(in, n, totals);
    DG_CUDA(cudaGetLastError());
    if (t == 1) {
        DG_CUDA(cudaMemsetAsync(offsets, 0, sizeof(int64_t), stream));
    } else {
        scan_impl<int64_t>(totals, offsets, t, temp + 2 * t, stream);
    }
    tile_scan<In><<<unsigned(t), kThreads, 0, stream>>>(in, out, n, offsets);
    DG_CUDA(cudaGetLastError());
}

}  // namespace

size_t scan_temp_bytes(int64_t n) {
    size_t total = 0;
    while (n > 1) {
        int64_t t = n_tiles(n);
        total += size_t(2 * t) * sizeof(int64_t);
        n = t;
    }
    return total + 64;
}

void exclusive_scan_i32_to_i64(const int32_t *in, int64_t *out, int64_t n, void *temp,
                               cudaStream_t stream) {
    scan_impl<int32_t>(in, out, n, static_cast<int64_t *>(temp), stream);
}

void exclusive_scan_i64(const int64_t *in, int64_t *out, int64_t n, void *temp,
                        cudaStream_t stream) {
    scan_impl<int64_t>(in, out, n, static_cast<int64_t *>(temp), stream);
}

}  // namespace dg
