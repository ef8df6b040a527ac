// Device-wide exclusive prefix sum of uint32 (replaces openfpm::scan, a CUB
// DeviceScan::ExclusiveSum wrapper, src/util/cuda/scan_ofp.cuh:31-80).
// Three phases: tile reduce, recursive scan of the tile sums, tile scan.
#include "common.cuh"
#include "internal.h"

namespace sgb {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* smem_warp, uint32_t* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) smem_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < kScanThreads / 32 ? smem_warp[lane] : 0;
        uint32_t s = w;
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < kScanThreads / 32) smem_warp[lane] = s - w;
        if (lane == kScanThreads / 32 - 1) smem_warp[32] = s;
    }
    __syncthreads();
    uint32_t r = smem_warp[warp] + x - v;
    *total = smem_warp[32];
    __syncthreads();
    return r;
}

__global__ void k_scan_reduce(const uint32_t* in, int64_t n, uint32_t* sums) {
    __shared__ uint32_t sw[33];
    const int64_t base = blockIdx.x * (int64_t)kScanTile + threadIdx.x * kScanItems;
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
        if (base + k < n) s += in[base + k];
    uint32_t tot;
    block_exclusive_scan(s, sw, &tot);
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

__global__ void k_scan_tiles(const uint32_t* in, int64_t n, const uint32_t* offsets, uint32_t* out,
                             uint32_t* total_dev) {
    __shared__ uint32_t sw[33];
    const int64_t base = blockIdx.x * (int64_t)kScanTile + threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = base + k < n ? in[base + k] : 0;
        s += v[k];
    }
    uint32_t tot;
    uint32_t pre = block_exclusive_scan(s, sw, &tot) + (offsets ? offsets[blockIdx.x] : 0);
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        if (base + k < n) out[base + k] = pre;
        pre += v[k];
    }
    if (total_dev && blockIdx.x == gridDim.x - 1 && threadIdx.x == kScanThreads - 1) *total_dev = pre;
}

// tmp must provide scratch for the tile sums of every level.
int scan_exclusive_u32(const uint32_t* in, uint32_t* out, int64_t n, uint32_t* total_dev, DevBuf* tmp,
                       cudaStream_t s) {
    if (n <= 0) {
        if (total_dev) SGB_CUDA(cudaMemsetAsync(total_dev, 0, 4, s));
        return SGB_OK;
    }
    const int64_t tiles = (n + kScanTile - 1) / kScanTile;
    if (tiles == 1) {
        k_scan_tiles<<<1, kScanThreads, 0, s>>>(in, n, nullptr, out, total_dev);
        SGB_CUDA(cudaGetLastError());
        return SGB_OK;
    }
    SGB_TRY(tmp->reserve((size_t)tiles * 4 * 2 + 64));
    uint32_t* sums = tmp->as<uint32_t>();
    uint32_t* offs = sums + tiles;
    k_scan_reduce<<<(unsigned)tiles, kScanThreads, 0, s>>>(in, n, sums);
    SGB_CUDA(cudaGetLastError());
    DevBuf sub;  // recursion scratch (only for > kScanTile^2 items)
    int st = scan_exclusive_u32(sums, offs, tiles, nullptr, &sub, s);
    if (st != SGB_OK) return st;
    k_scan_tiles<<<(unsigned)tiles, kScanThreads, 0, s>>>(in, n, offs, out, total_dev);
    cudaError_t e = cudaGetLastError();
    if (sub.p) {
        cudaStreamSynchronize(s);
        sub.release();
    }
    if (e != cudaSuccess) return cuda_status(e, "k_scan_tiles");
    return SGB_OK;
}

}  // namespace sgb
