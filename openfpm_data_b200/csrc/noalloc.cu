// sgb_existing_offsets_noalloc: the per-chunk offsets of existing points
// without any device allocation.
//
// Some callers cannot allocate device memory: applications whose device
// memory is owned by their own pool allocator (they hand the library the
// buffers to use and allow no allocation behind their back), and
// latency-sensitive loops that may not call cudaMalloc, which can
// synchronise the whole device.  This entry point computes what
// sgb_existing_offsets computes, but its scan scratch lives in a fixed
// file-scope device array instead of buffers allocated on first use.
//
// Scratch: kNoAllocMaxTiles int64 tile sums (plus one total), 256-byte
// aligned, held by every GPU that loads the library until the process exits.
// One tile covers kTile chunks, so a grid may have at most
// kNoAllocMaxTiles * kTile = 1,048,576 chunks; larger grids are rejected with
// SGB_ERANGE.  Every call uses the same array and leaves the last call's
// values in it; calls that overlap on the GPU (other streams, other host
// threads) race on it.
#include <cstdio>
#include <mutex>

#include "common.cuh"
#include "internal.h"

namespace sgb {

constexpr int kTile = 2048;                 // chunks per scan tile (256 threads x 8)
constexpr int kNoAllocMaxTiles = 512;
constexpr int64_t kNoAllocMaxChunks = (int64_t)kTile * kNoAllocMaxTiles;

static __device__ __align__(256) long long g_noalloc_scratch[kNoAllocMaxTiles + 1];

// per-chunk EXIST counts written straight into the caller's output
__global__ void k_na_counts(const uint8_t* mask, int64_t n, int bs, long long* out) {
    const int64_t chunk = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (chunk >= n) return;
    const uint8_t* m = mask + (size_t)chunk * bs;
    long long c = 0;
    for (int r = 0; r < bs / 32; ++r) c += __popc(__ballot_sync(0xffffffffu, m[r * 32 + lane] & 1));
    if (lane == 0) out[chunk] = c;
}

__device__ __forceinline__ long long block_scan_excl(long long v, long long* sw, long long* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    long long x = v;
    for (int o = 1; o < 32; o <<= 1) {
        long long y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sw[warp] = x;
    __syncthreads();
    if (warp == 0) {
        long long w = lane < nw ? sw[lane] : 0, s = w;
        for (int o = 1; o < 32; o <<= 1) {
            long long y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < nw) sw[lane] = s - w;
        if (lane == nw - 1) sw[32] = s;
    }
    __syncthreads();
    const long long r = sw[warp] + x - v;
    *total = sw[32];
    __syncthreads();
    return r;
}

// tile sums -> scratch[tile]
__global__ void k_na_tile_sums(const long long* out, int64_t n, long long* scratch) {
    __shared__ long long sw[33];
    const int64_t base = (int64_t)blockIdx.x * kTile + threadIdx.x * 8;
    long long s = 0;
    for (int k = 0; k < 8; ++k)
        if (base + k < n) s += out[base + k];
    long long tot;
    block_scan_excl(s, sw, &tot);
    if (threadIdx.x == 0) scratch[blockIdx.x] = tot;
}

// exclusive scan of the tile sums in place (one CTA); total -> scratch[kNoAllocMaxTiles]
__global__ void k_na_scan_sums(long long* scratch, int ntiles) {
    __shared__ long long sw[33];
    const int t = threadIdx.x;
    const long long v = t < ntiles ? scratch[t] : 0;
    long long tot;
    const long long ex = block_scan_excl(v, sw, &tot);
    if (t < ntiles) scratch[t] = ex;
    if (t == 0) scratch[kNoAllocMaxTiles] = tot;
}

// per tile: exclusive scan of the counts in place plus the tile offset
__global__ void k_na_apply(long long* out, int64_t n, const long long* scratch) {
    __shared__ long long sw[33];
    const int64_t base = (int64_t)blockIdx.x * kTile + threadIdx.x * 8;
    long long v[8], s = 0;
    for (int k = 0; k < 8; ++k) {
        v[k] = base + k < n ? out[base + k] : 0;
        s += v[k];
    }
    long long tot;
    long long pre = block_scan_excl(s, sw, &tot) + scratch[blockIdx.x];
    for (int k = 0; k < 8; ++k) {
        if (base + k < n) out[base + k] = pre;
        pre += v[k];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = scratch[kNoAllocMaxTiles];
}

// device address of the scratch array, looked up once per device
static long long* g_scratch_addr[64];
static std::mutex g_scratch_mu;

static int scratch_for_device(int dev, long long** ptr) {
    if (dev < 0 || dev >= 64) return SGB_EINVAL;
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_status(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
        g_scratch_addr[dev] = static_cast<long long*>(p);
    }
    *ptr = g_scratch_addr[dev];
    return SGB_OK;
}

}  // namespace sgb

using namespace sgb;

extern "C" int sgb_existing_offsets_noalloc(const sgb_grid* g, int64_t* offsets_dev, sgb_stream stream) {
    if (!g || !offsets_dev) return SGB_EINVAL;
    if (g->n > kNoAllocMaxChunks) {
        set_error("sgb_existing_offsets_noalloc handles at most 1048576 chunks; use sgb_existing_offsets");
        return SGB_ERANGE;
    }
    DeviceGuard dg(g->device);
    SGB_CUDA(dg.status);
    long long* scratch = nullptr;
    SGB_TRY(scratch_for_device(g->device, &scratch));
    cudaStream_t s = (cudaStream_t)stream;
    long long* out = reinterpret_cast<long long*>(offsets_dev);
    const int64_t n = g->n;
    if (n == 0) {
        SGB_CUDA(cudaMemsetAsync(out, 0, sizeof(long long), s));
        return SGB_OK;
    }
    const int ntiles = (int)((n + kTile - 1) / kTile);
    k_na_counts<<<(unsigned)((n * 32 + 255) / 256), 256, 0, s>>>(g->mask.as<uint8_t>(), n, g->geo.bs, out);
    k_na_tile_sums<<<ntiles, 256, 0, s>>>(out, n, scratch);
    k_na_scan_sums<<<1, kNoAllocMaxTiles, 0, s>>>(scratch, ntiles);
    k_na_apply<<<ntiles, 256, 0, s>>>(out, n, scratch);
    SGB_CUDA(cudaGetLastError());
    return SGB_OK;
}
