// Flush of staged point inserts into the sorted block map.
//
// Replaces vector_sparse::flush -> flush_on_gpu_insert (src/Vector/
// map_vector_sparse.hpp:1193-1226): make_continuos + reorder_indexes (CUB
// radix sort) + merge_indexes (Thrust merge) + BlockFunctor::solve_conflicts
// (src/SparseGridGpu/BlockMapGpu_kernels.cuh:701-807).
//
// The reference stages one whole chunk slot per inserted point and reduces
// chunk slots; a chunk slot that carries a single point reduces to a per-point
// fold, so this path stages points only:
//   1. stable LSD radix sort of (point id, insertion index)
//   2. per point: A = first insert, A = op(A, next) in insertion order
//   3. unique chunk ids, looked up in the current index
//   4. when new chunks appear: merged index, old chunks moved to their new
//      positions (128-bit copies), new chunks set to background / empty mask
//   5. per point: A = op(A, old) when the point exists, mask |= EXIST
// One device->host read of three counters sizes the new map.
#include <algorithm>
#include <cstring>

#include "common.cuh"
#include "internal.h"

namespace sgb {

constexpr int kRsWarps = 8;
constexpr int kRsRounds = 16;
constexpr int kRsThreads = kRsWarps * 32;
constexpr int kRsTile = kRsThreads * kRsRounds;  // 4096 keys per CTA

constexpr int kRsMaxBuckets = 1024;  // digits of up to 10 bits

template <typename K>
__global__ void k_rs_hist(const K* keys, int64_t n, int shift, unsigned dmask, int nbuckets, uint32_t* hist,
                          int ntiles) {
    __shared__ uint32_t h[kRsMaxBuckets];
    for (int i = threadIdx.x; i < nbuckets; i += blockDim.x) h[i] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kRsTile;
    for (int k = threadIdx.x; k < kRsTile; k += blockDim.x) {
        int64_t i = base + k;
        if (i < n) atomicAdd(&h[(unsigned)(keys[i] >> shift) & dmask], 1u);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < nbuckets; d += blockDim.x) hist[(size_t)d * ntiles + blockIdx.x] = h[d];
}

// Stable scatter: items keep their order inside each digit.  Tile order is
// (warp, round, lane) == index order; ranks inside a warp come from
// __match_any_sync peer groups, counts across warps from a shared prefix.
// The tile is then staged in shared memory in digit order and written out
// run by run, so that consecutive threads store consecutive positions of a
// digit's output range instead of one scattered 4-byte store per item.
template <typename K>
__host__ __device__ constexpr size_t rs_union_bytes() {
    return (size_t)kRsWarps * kRsMaxBuckets * 4 > (size_t)kRsTile * (sizeof(K) + 4)
               ? (size_t)kRsWarps * kRsMaxBuckets * 4
               : (size_t)kRsTile * (sizeof(K) + 4);
}
template <typename K>
__host__ __device__ constexpr size_t rs_scatter_smem() {
    return rs_union_bytes<K>() + (size_t)kRsMaxBuckets * 4 + kRsWarps * 4;
}

template <typename K>
__global__ void __launch_bounds__(kRsThreads) k_rs_scatter(const K* kin, const uint32_t* vin, K* kout, uint32_t* vout,
                                                            int64_t n, int shift, unsigned dmask, int nbuckets,
                                                            const uint32_t* offs, int ntiles) {
    extern __shared__ __align__(16) unsigned char rs_smem[];
    auto wcnt = reinterpret_cast<uint32_t(*)[kRsMaxBuckets]>(rs_smem);  // [kRsWarps][kRsMaxBuckets]
    K* sk = reinterpret_cast<K*>(rs_smem);                              // the same bytes, once wcnt is done
    uint32_t* sv = reinterpret_cast<uint32_t*>(rs_smem + (size_t)kRsTile * sizeof(K));
    uint32_t* dstart = reinterpret_cast<uint32_t*>(rs_smem + rs_union_bytes<K>());
    uint32_t* wsum = dstart + kRsMaxBuckets;
    for (int i = threadIdx.x; i < kRsWarps * kRsMaxBuckets; i += blockDim.x) (&wcnt[0][0])[i] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t tbase = (int64_t)blockIdx.x * kRsTile;
    const int64_t base = tbase + warp * (32 * kRsRounds);
    K key[kRsRounds];
    uint32_t val[kRsRounds], rank[kRsRounds];
    const unsigned lt = lanemask_lt();
#pragma unroll
    for (int r = 0; r < kRsRounds; ++r) {
        const int64_t i = base + r * 32 + lane;
        const bool valid = i < n;
        key[r] = valid ? kin[i] : K(0);
        val[r] = valid ? (vin ? vin[i] : (uint32_t)i) : 0u;
        const unsigned d = valid ? ((unsigned)(key[r] >> shift) & dmask) : 0x10000u;
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        uint32_t cnt = 0;
        if (valid) cnt = wcnt[warp][d];
        rank[r] = cnt + __popc(peers & lt);
        __syncwarp();
        if (valid && lane == __ffs(peers) - 1) wcnt[warp][d] = cnt + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // per digit: the warps' counts become prefixes; thread t owns digits kPer t .. kPer t + kPer - 1
    constexpr int kPer = kRsMaxBuckets / kRsThreads;
    uint32_t tot[kPer], tsum = 0;
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
        const int d = threadIdx.x * kPer + k;
        uint32_t run = 0;
        if (d < nbuckets)
            for (int w = 0; w < kRsWarps; ++w) {
                const uint32_t c = wcnt[w][d];
                wcnt[w][d] = run;
                run += c;
            }
        tot[k] = run;
        tsum += run;
    }
    // the digits' first positions in the tile: an exclusive scan of the threads' sums
    uint32_t incl = tsum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    uint32_t run = incl - tsum;
    for (int w = 0; w < warp; ++w) run += wsum[w];
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
        const int d = threadIdx.x * kPer + k;
        if (d < nbuckets) dstart[d] = run;
        run += tot[k];
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kRsRounds; ++r) {
        if (base + r * 32 + lane < n) {
            const unsigned d = (unsigned)(key[r] >> shift) & dmask;
            rank[r] += dstart[d] + wcnt[warp][d];  // position in the tile, digit order
        }
    }
    __syncthreads();  // wcnt is read no more: its bytes take the staged tile
#pragma unroll
    for (int r = 0; r < kRsRounds; ++r) {
        if (base + r * 32 + lane < n) {
            sk[rank[r]] = key[r];
            sv[rank[r]] = val[r];
        }
    }
    __syncthreads();
    const int tn = (int)(n - tbase < kRsTile ? n - tbase : kRsTile);
    for (int j = threadIdx.x; j < tn; j += kRsThreads) {
        const K k = sk[j];
        const unsigned d = (unsigned)(k >> shift) & dmask;
        const size_t pos = (size_t)offs[(size_t)d * ntiles + blockIdx.x] + (uint32_t)(j - dstart[d]);
        kout[pos] = k;
        vout[pos] = sv[j];
    }
}

template <typename K>
__global__ void k_make_keys(const int64_t* lin, int64_t n, K* keys) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) keys[i] = (K)lin[i];
}

struct PropSet {
    unsigned char* p[kMaxProps];
    int type[kMaxProps];
    int op[kMaxProps];
    int nprop;
};

template <typename T>
__device__ __forceinline__ T op_apply(int op, T a, T b) {
    switch (op) {
        case SGB_OP_RIGHT: return b;                  // rightOperand_t
        case SGB_OP_LEFT: return a;                   // leftOperand_t
        case SGB_OP_ADD: return a + b;                // plus_t
        case SGB_OP_MAX: return a > b ? a : b;        // maximum_t
        case SGB_OP_MIN: return a < b ? a : b;        // minimum_t
        default: return b;
    }
}

// a = op(a, b) on raw elements of type `type` (both operands exist).
__device__ __forceinline__ void op_raw(int type, int op, unsigned char* a, const unsigned char* b) {
    switch (type) {
        case SGB_F32: *(float*)a = op_apply(op, *(const float*)a, *(const float*)b); break;
        case SGB_F64: *(double*)a = op_apply(op, *(const double*)a, *(const double*)b); break;
        case SGB_I32: {
            int32_t x = *(const int32_t*)a, y = *(const int32_t*)b;
            *(int32_t*)a = op == SGB_OP_OR ? (x | y) : op_apply(op, x, y);
            break;
        }
        default: {
            uint8_t x = *a, y = *b;
            *a = op == SGB_OP_OR ? (uint8_t)(x | y) : op_apply(op, x, y);
        }
    }
}

__device__ __forceinline__ int esz(int t) { return t == SGB_F64 ? 8 : (t == SGB_U8 ? 1 : 4); }

template <typename K>
__global__ void k_heads(const K* sk, int64_t n, int bs_shift, uint32_t* pt_head, uint32_t* blk_head) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const K k = sk[i];
    const bool first = i == 0;
    const K prev = first ? k : sk[i - 1];
    pt_head[i] = first || prev != k;
    blk_head[i] = first || (prev >> bs_shift) != (k >> bs_shift);
}

// Per point: fold its inserts in insertion order (the sort is stable).
template <typename K>
__global__ void k_fold(const K* sk, const uint32_t* sidx, int64_t n, int bs_shift, const uint32_t* pt_head,
                       const uint32_t* pt_seg, const uint32_t* blk_head, const uint32_t* blk_seg, PropSet vals,
                       PropSet upt, int64_t* upt_key, int64_t* ublk_key) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n || !pt_head[i]) return;
    const K k = sk[i];
    const uint32_t u = pt_seg[i];
    upt_key[u] = (int64_t)k;
    if (blk_head[i]) ublk_key[blk_seg[i]] = (int64_t)(k >> bs_shift);
    for (int p = 0; p < vals.nprop; ++p) {
        if (vals.op[p] == SGB_OP_NONE) continue;
        const int t = vals.type[p], es = esz(t);
        alignas(8) unsigned char acc[8];
        const unsigned char* src = vals.p[p] + (size_t)sidx[i] * es;
        for (int b = 0; b < es; ++b) acc[b] = src[b];
        for (int64_t j = i + 1; j < n && sk[j] == k; ++j) op_raw(t, vals.op[p], acc, vals.p[p] + (size_t)sidx[j] * es);
        unsigned char* dst = upt.p[p] + (size_t)u * es;
        for (int b = 0; b < es; ++b) dst[b] = acc[b];
    }
}

__global__ void k_lookup(const int64_t* ublk_key, int64_t nslots, const uint32_t* nb_dev, const int64_t* keys,
                         int64_t n, uint32_t* isnew) {
    int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (b < nslots) isnew[b] = b < (int64_t)*nb_dev ? (find_key(keys, n, ublk_key[b]) < 0) : 0u;
}

__global__ void k_compact_new(const int64_t* ublk_key, int64_t nb, const uint32_t* isnew, const uint32_t* rank,
                              int64_t* newkeys) {
    int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (b < nb && isnew[b]) newkeys[rank[b]] = ublk_key[b];
}

// New position of every old chunk: j + #(new keys below its key).
__global__ void k_old_pos(const int64_t* keys, int64_t n, const int64_t* newkeys, int64_t nnew, int64_t* keys_out,
                          int64_t* newpos) {
    int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= n) return;
    const int64_t k = keys[j];
    const int64_t pos = j + lower_bound_i64(newkeys, nnew, k);
    newpos[j] = pos;
    keys_out[pos] = k;
}

__global__ void k_new_pos(const int64_t* newkeys, int64_t nnew, const int64_t* keys, int64_t n, int64_t* keys_out,
                          int64_t* newpos) {
    int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r >= nnew) return;
    const int64_t k = newkeys[r];
    const int64_t pos = r + lower_bound_i64(keys, n, k);
    newpos[r] = pos;
    keys_out[pos] = k;
}

// Chunk moves as a flat stream of 16-byte words: word i of the old map (of
// chunk i >> cw_shift; a chunk holds 2^cw_shift words) goes to the same word
// of the chunk's merged position.  Four independent copies are in flight per
// thread and the loads are coalesced, whatever a chunk's size.
__global__ void k_move_chunks(const uint4* __restrict__ src, uint4* __restrict__ dst, int64_t nchunks, int cw_shift,
                              const int64_t* __restrict__ newpos) {
    const int64_t total = nchunks << cw_shift, wmask = (int64_t(1) << cw_shift) - 1;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    for (; i + 3 * stride < total; i += 4 * stride) {
        uint4 v[4];
        int64_t d[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int64_t j = i + k * stride;
            v[k] = __ldcs(src + j);  // the old map is read once
            d[k] = (__ldg(newpos + (j >> cw_shift)) << cw_shift) | (j & wmask);
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) dst[d[k]] = v[k];
    }
    for (; i < total; i += stride) dst[(__ldg(newpos + (i >> cw_shift)) << cw_shift) | (i & wmask)] = __ldcs(src + i);
}

// New chunks get the background pattern (or a zero mask), the same flat word stream.
__global__ void k_fill_chunks(uint4* __restrict__ dst, int64_t nnew, int cw_shift, uint4 word,
                              const int64_t* __restrict__ newpos) {
    const int64_t total = nnew << cw_shift, wmask = (int64_t(1) << cw_shift) - 1;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
#pragma unroll 4
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += stride)
        dst[(__ldg(newpos + (i >> cw_shift)) << cw_shift) | (i & wmask)] = word;
}

// The element pattern of es bytes repeated over a 16-byte word.
static uint4 replicate16(uint64_t pattern, int es) {
    unsigned char b[16];
    for (int i = 0; i < 16; ++i) b[i] = (unsigned char)(pattern >> (8 * (i % es)));
    uint4 w;
    std::memcpy(&w, b, 16);
    return w;
}

// Per unique point: reduce with the existing value, write, set EXIST.
__global__ void k_scatter(const int64_t* upt_key, int64_t nu, int bs_shift, const int64_t* keys, int64_t n,
                          PropSet upt, PropSet data, uint8_t* mask, int any_listed) {
    int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (u >= nu) return;
    const int64_t k = upt_key[u];
    const int64_t pos = find_key(keys, n, k >> bs_shift);
    if (pos < 0) return;  // cannot happen: every chunk id was merged in
    const int64_t bsm = (1ll << bs_shift) - 1;
    const size_t idx = (size_t)pos * (bsm + 1) + (size_t)(k & bsm);
    const uint8_t om = mask[idx];
    for (int p = 0; p < data.nprop; ++p) {
        if (data.op[p] == SGB_OP_NONE) continue;
        const int t = data.type[p], es = esz(t);
        alignas(8) unsigned char acc[8];
        const unsigned char* a = upt.p[p] + (size_t)u * es;
        for (int b = 0; b < es; ++b) acc[b] = a[b];
        unsigned char* d = data.p[p] + idx * es;
        if (om & 1) op_raw(t, data.op[p], acc, d);  // op(new, old), BlockMapGpu_kernels.cuh:294-305
        for (int b = 0; b < es; ++b) d[b] = acc[b];
    }
    if (any_listed) mask[idx] = om | 1u;
}

static inline unsigned nblk(int64_t n, int t = 256) { return (unsigned)((n + t - 1) / t); }

template <typename K>
static int radix_sort(sgb_grid* g, int64_t n, int bits, K** keys_out, uint32_t** vals_out, cudaStream_t s) {
    DevBuf& kA = g->scratch[0];
    DevBuf& kB = g->scratch[1];
    DevBuf& vA = g->scratch[2];
    DevBuf& vB = g->scratch[3];
    DevBuf& hist = g->scratch[4];
    DevBuf& hoff = g->scratch[5];
    SGB_TRY(kA.ensure((size_t)n * sizeof(K)));
    SGB_TRY(kB.ensure((size_t)n * sizeof(K)));
    SGB_TRY(vA.ensure((size_t)n * 4));
    SGB_TRY(vB.ensure((size_t)n * 4));
    const int ntiles = (int)((n + kRsTile - 1) / kRsTile);
    // as few passes as digits of at most 10 bits allow, the digit width spread evenly over them
    const int passes = bits <= 0 ? 1 : (bits + 9) / 10;
    const int dbits = bits <= 0 ? 1 : (bits + passes - 1) / passes;
    const int nbuckets = 1 << dbits;
    const unsigned dmask = (unsigned)nbuckets - 1u;
    SGB_TRY(hist.ensure((size_t)ntiles * nbuckets * 4));
    SGB_TRY(hoff.ensure((size_t)ntiles * nbuckets * 4));
    k_make_keys<K><<<nblk(n), 256, 0, s>>>(g->pend_lin.as<int64_t>(), n, kA.as<K>());
    SGB_CUDA(cudaGetLastError());
    K* kin = kA.as<K>();
    K* kout = kB.as<K>();
    uint32_t* vbuf[2] = {vA.as<uint32_t>(), vB.as<uint32_t>()};
    for (int ps = 0; ps < passes; ++ps) {
        const int shift = ps * dbits;
        const uint32_t* vin = ps == 0 ? nullptr : vbuf[ps & 1];  // pass 0 ranks the insertion index itself
        uint32_t* vout = vbuf[(ps + 1) & 1];
        k_rs_hist<K><<<ntiles, 256, 0, s>>>(kin, n, shift, dmask, nbuckets, hist.as<uint32_t>(), ntiles);
        SGB_CUDA(cudaGetLastError());
        SGB_TRY(scan_exclusive_u32(hist.as<uint32_t>(), hoff.as<uint32_t>(), (int64_t)ntiles * nbuckets, nullptr,
                                   &g->scratch[6], s));
        constexpr size_t smem = rs_scatter_smem<K>();
        SGB_CUDA(cudaFuncSetAttribute(k_rs_scatter<K>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_rs_scatter<K><<<ntiles, kRsThreads, smem, s>>>(kin, vin, kout, vout, n, shift, dmask, nbuckets,
                                                         hoff.as<uint32_t>(), ntiles);
        SGB_CUDA(cudaGetLastError());
        K* kt = kin;
        kin = kout;
        kout = kt;
    }
    *vals_out = vbuf[passes & 1];
    *keys_out = kin;
    return SGB_OK;
}

template <typename K>
static int flush_impl(sgb_grid* g, const int* ops, int bits, cudaStream_t s) {
    const int64_t n = g->npend;
    const int bs = g->geo.bs;
    const int bs_shift = bs == 512 ? 9 : 6;
    K* sk = nullptr;
    uint32_t* sidx = nullptr;
    SGB_TRY(radix_sort<K>(g, n, bits, &sk, &sidx, s));

    DevBuf& heads = g->scratch[7];
    DevBuf& segs = g->scratch[8];
    DevBuf& ubuf = g->scratch[9];
    DevBuf& uval = g->scratch[10];
    DevBuf& cnt = g->scratch[11];
    SGB_TRY(heads.ensure((size_t)n * 8));
    SGB_TRY(segs.ensure((size_t)n * 8 + 64));
    SGB_TRY(cnt.ensure(64));
    uint32_t* pt_head = heads.as<uint32_t>();
    uint32_t* blk_head = pt_head + n;
    uint32_t* pt_seg = segs.as<uint32_t>();
    uint32_t* blk_seg = pt_seg + n;
    uint32_t* counters = cnt.as<uint32_t>();  // [0] U, [1] B, [2] NB
    k_heads<K><<<nblk(n), 256, 0, s>>>(sk, n, bs_shift, pt_head, blk_head);
    SGB_CUDA(cudaGetLastError());
    SGB_TRY(scan_exclusive_u32(pt_head, pt_seg, n, counters + 0, &g->scratch[6], s));
    SGB_TRY(scan_exclusive_u32(blk_head, blk_seg, n, counters + 1, &g->scratch[6], s));

    // unique points / chunks: at most n of each
    size_t uval_bytes = 0;
    for (int p = 0; p < g->nprop; ++p) uval_bytes += ((size_t)n * elem_size(g->ptype[p]) + 15) & ~(size_t)15;
    SGB_TRY(uval.ensure(uval_bytes + 64));
    // ubuf: upt_key[n] int64 | ublk_key[n] int64 | isnew[n] u32 | rank[n] u32 | newkeys[n] int64
    SGB_TRY(ubuf.ensure((size_t)n * 32 + 256));
    int64_t* upt_key = ubuf.as<int64_t>();
    int64_t* ublk_key = upt_key + n;
    uint32_t* isnew = (uint32_t*)(ublk_key + n);
    uint32_t* rank = isnew + n;
    int64_t* newkeys = (int64_t*)(rank + n);

    PropSet vals{}, upt{}, data{};
    vals.nprop = upt.nprop = data.nprop = g->nprop;
    size_t off = 0;
    int any_listed = 0;
    for (int p = 0; p < g->nprop; ++p) {
        vals.p[p] = g->pend_val[p].as<unsigned char>();
        upt.p[p] = uval.as<unsigned char>() + off;
        off += ((size_t)n * elem_size(g->ptype[p]) + 15) & ~(size_t)15;
        vals.type[p] = upt.type[p] = data.type[p] = g->ptype[p];
        vals.op[p] = upt.op[p] = data.op[p] = ops[p];
        any_listed |= ops[p] != SGB_OP_NONE;
    }
    k_fold<K><<<nblk(n), 256, 0, s>>>(sk, sidx, n, bs_shift, pt_head, pt_seg, blk_head, blk_seg, vals, upt, upt_key,
                                      ublk_key);
    SGB_CUDA(cudaGetLastError());

    // B is only known on the device: every slot below n is looked up, the
    // ones at or above B report "not new".
    k_lookup<<<nblk(n), 256, 0, s>>>(ublk_key, n, counters + 1, g->keys.as<int64_t>(), g->n, isnew);
    SGB_CUDA(cudaGetLastError());
    SGB_TRY(scan_exclusive_u32(isnew, rank, n, counters + 2, &g->scratch[6], s));
    SGB_TRY(g->hscratch.ensure(64));
    SGB_CUDA(cudaMemcpyAsync(g->hscratch.p, counters, 12, cudaMemcpyDeviceToHost, s));
    SGB_CUDA(cudaStreamSynchronize(s));
    const int64_t U = ((uint32_t*)g->hscratch.p)[0];
    const int64_t B = ((uint32_t*)g->hscratch.p)[1];
    const int64_t NB = ((uint32_t*)g->hscratch.p)[2];

    if (NB > 0) {
        const int64_t nold = g->n, nn_ = nold + NB;
        k_compact_new<<<nblk(B), 256, 0, s>>>(ublk_key, B, isnew, rank, newkeys);
        SGB_CUDA(cudaGetLastError());
        // second buffer set for the new map (contents are rebuilt): kept while it holds the map,
        // otherwise allocated for twice the map, so that a growing map reallocates rarely (each
        // reallocation frees and maps gigabytes and stalls the device)
        int64_t cap2 = std::min<int64_t>((int64_t)(g->keys2.bytes / 8), (int64_t)(g->mask2.bytes / bs) - 1);
        for (int p = 0; p < g->nprop; ++p)
            cap2 = std::min<int64_t>(cap2, (int64_t)(g->data2[p].bytes / ((size_t)bs * elem_size(g->ptype[p]))) - 1);
        if (cap2 < nn_) {
            cap2 = std::max<int64_t>(2 * nn_, 16);
            SGB_TRY(g->keys2.ensure((size_t)cap2 * 8));
            SGB_TRY(g->mask2.ensure((size_t)(cap2 + 1) * bs));
            for (int p = 0; p < g->nprop; ++p)
                SGB_TRY(g->data2[p].ensure((size_t)(cap2 + 1) * bs * elem_size(g->ptype[p])));
        }
        DevBuf& posbuf = g->scratch[5];  // histogram offsets are no longer needed
        SGB_TRY(posbuf.ensure((size_t)(nold + NB) * 8 + 64));
        int64_t* oldpos = posbuf.as<int64_t>();
        int64_t* npos = oldpos + nold;
        if (nold > 0) {
            k_old_pos<<<nblk(nold), 256, 0, s>>>(g->keys.as<int64_t>(), nold, newkeys, NB, g->keys2.as<int64_t>(),
                                                 oldpos);
            SGB_CUDA(cudaGetLastError());
        }
        k_new_pos<<<nblk(NB), 256, 0, s>>>(newkeys, NB, g->keys.as<int64_t>(), nold, g->keys2.as<int64_t>(), npos);
        SGB_CUDA(cudaGetLastError());
        // flat word streams: at most 16 CTAs of 256 threads per SM, no more threads than words
        auto word_grid = [&](int64_t chunks, int cw_shift) {
            const int64_t words = chunks << cw_shift;
            return (unsigned)std::max<int64_t>(1, std::min<int64_t>((int64_t)g->num_sms * 16, (words + 255) / 256));
        };
        auto shift_of = [](int words) {  // chunk sizes in 16-byte words are powers of two
            int sh = 0;
            while ((1 << sh) < words) ++sh;
            return sh;
        };
        const int msh = shift_of(bs / 16);
        if ((1 << msh) != bs / 16) {  // chunk edges are powers of two, so every chunk is 2^k words
            set_error("chunk size is not a power of two 16-byte words");
            return SGB_ENOTSUP;
        }
        for (int p = 0; p < g->nprop; ++p) {
            const int es = elem_size(g->ptype[p]);
            const int sh = shift_of(bs * es / 16);
            if (nold > 0) {
                k_move_chunks<<<word_grid(nold, sh), 256, 0, s>>>(g->data[p].as<uint4>(), g->data2[p].as<uint4>(),
                                                                  nold, sh, oldpos);
                SGB_CUDA(cudaGetLastError());
            }
            uint64_t pat = 0;
            std::memcpy(&pat, g->bck[p], es);
            k_fill_chunks<<<word_grid(NB, sh), 256, 0, s>>>(g->data2[p].as<uint4>(), NB, sh, replicate16(pat, es),
                                                            npos);
            SGB_CUDA(cudaGetLastError());
        }
        if (nold > 0) {
            k_move_chunks<<<word_grid(nold, msh), 256, 0, s>>>(g->mask.as<uint4>(), g->mask2.as<uint4>(), nold, msh,
                                                               oldpos);
            SGB_CUDA(cudaGetLastError());
        }
        k_fill_chunks<<<word_grid(NB, msh), 256, 0, s>>>(g->mask2.as<uint4>(), NB, msh, make_uint4(0, 0, 0, 0), npos);
        SGB_CUDA(cudaGetLastError());
        // swap buffer sets
        std::swap(g->keys, g->keys2);
        std::swap(g->mask, g->mask2);
        for (int p = 0; p < g->nprop; ++p) std::swap(g->data[p], g->data2[p]);
        g->cap = cap2;
        g->n = nn_;
        SGB_TRY(write_background(g, g->n, s, g->data, g->mask));
    }
    for (int p = 0; p < g->nprop; ++p) data.p[p] = g->data[p].as<unsigned char>();
    k_scatter<<<nblk(U), 256, 0, s>>>(upt_key, U, bs_shift, g->keys.as<int64_t>(), g->n, upt, data,
                                      g->mask.as<uint8_t>(), any_listed);
    SGB_CUDA(cudaGetLastError());
    return SGB_OK;
}

}  // namespace sgb

using namespace sgb;

extern "C" int sgb_flush(sgb_grid* g, const int* ops, sgb_stream stream) {
    if (!g || !ops) return SGB_EINVAL;
    for (int p = 0; p < g->nprop; ++p) {
        if (ops[p] < SGB_OP_NONE || ops[p] > SGB_OP_OR) return SGB_EINVAL;
        if (ops[p] == SGB_OP_OR && (g->ptype[p] == SGB_F32 || g->ptype[p] == SGB_F64)) return SGB_EINVAL;
    }
    cudaStream_t s = (cudaStream_t)stream;
    if (g->npend == 0) return SGB_OK;
    // out-of-domain points were flagged at insert time
    SGB_TRY(g->hscratch.ensure(64));
    SGB_CUDA(cudaMemcpyAsync(g->hscratch.p, g->err.p, 4, cudaMemcpyDeviceToHost, s));
    SGB_CUDA(cudaStreamSynchronize(s));
    const unsigned e = *(unsigned*)g->hscratch.p;
    if (e & (kErrOutOfDomain | kErrPoolOverflow)) {
        SGB_CUDA(cudaMemsetAsync(g->err.p, 0, 4, s));
        g->npend = 0;
        set_error((e & kErrOutOfDomain)
                      ? "an inserted point lies outside the grid domain; the staged inserts were dropped"
                      : "an insert pool counted more points than its slots; the staged inserts were dropped");
        return SGB_ERANGE;
    }
    const int64_t maxlin = key_space(g->geo) * g->geo.bs;
    int bits = 0;
    while (bits < 63 && (int64_t(1) << bits) < maxlin) ++bits;
    int st;
    if (bits <= 32) st = flush_impl<uint32_t>(g, ops, bits, s);
    else st = flush_impl<uint64_t>(g, ops, bits, s);
    g->npend = 0;
    g->nn_valid[0] = g->nn_valid[1] = false;
    g->nnhash_ok = false;
    g->bits_valid = false;
    g->epts_valid = false;
    return st;
}
