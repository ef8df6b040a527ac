// findNeighbours, existence bitmaps and tagBoundaries.
#include <vector>

#include "common.cuh"
#include "internal.h"

namespace sgb {

// grid_smb::BlockLinId (src/Grid/Geometry/grid_smb.hpp:280-299): only the
// upper bound is checked, so a block coordinate of -1 along x or y yields the
// id of a block one row (or slice) back -- reproduced on purpose, it decides
// which chunk an NNFull neighbour lookup returns at the low faces.
//
// grid_zmb::BlockLinId (lin_zid, src/util/zmorton.hpp:72-98) checks nothing;
// a negative coordinate there gives an id far above every chunk's, so it is
// absent like one past the upper faces: -1 here.
__device__ __forceinline__ int64_t block_lin_ref(const Geometry& geo, const int64_t* bc) {
    if (geo.zorder) {
        if (bc[0] < 0 || bc[1] < 0 || bc[2] < 0) return -1;
        return block_key(geo, bc[0], bc[1], bc[2]);
    }
    // static indices only (a dynamic one would put the coordinates in local memory)
    int64_t lin = 0;
    bool past = false;
#pragma unroll
    for (int d = 2; d >= 0; --d) {
        if (d < geo.dim) {
            past |= bc[d] >= geo.bsz[d];
            lin = lin * geo.bsz[d] + bc[d];
        }
    }
    return past ? -1 : lin;
}

// findNeighbours (src/SparseGridGpu/SparseGridGpu_kernels.cuh:1014-1035) with
// NNStar::getNNpos (SparseGridGpu_ker_util.hpp:91-112, slots -x,+x,-y,+y,-z,+z,
// two unused) and NNFull::getNNpos (SparseGridGpu.hpp:266-287, slot
// dx+3dy+9dz over {0,1,2}).  Output: data position, -1 when absent.
//
// The keys are distinct sorted integers, so the key bl of a neighbour lies
// within |bl - key| positions of the chunk's own: a near key (an x neighbour
// under x-fastest ids) is searched in that window, one or two probes of
// neighbouring positions; a far one is looked up in a hash of the keys.
__device__ __forceinline__ int64_t find_near(const int64_t* keys, int64_t n, int64_t i, int64_t key, int64_t bl) {
    int64_t lo, hi;
    if (bl > key) {
        lo = i + 1;
        hi = bl - key < n - i ? i + 1 + (bl - key) : n;
    } else {
        hi = i;
        lo = key - bl < i ? i - (key - bl) : 0;
    }
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (keys[mid] < bl) lo = mid + 1;
        else hi = mid;
    }
    return (lo < n && keys[lo] == bl) ? lo : -1;
}

// Open-addressing hash of the chunk keys: linear probing, Fibonacci hashing (the key times
// 2^64 divided by the golden ratio, top bits), at most half full, so every probe sequence ends
// at an empty slot (key -1) within a few steps.  A lookup costs one or two L2 reads where a
// binary search for a y or z neighbour costs up to log2(n) dependent ones.
struct KeyHash {
    int64_t* keys;
    int32_t* pos;
    uint64_t mask;
    int shift;
};

__device__ __forceinline__ uint64_t kh_slot(const KeyHash& h, int64_t key) {
    return ((uint64_t)key * 0x9E3779B97F4A7C15ull) >> h.shift;
}

__global__ void k_kh_build(const int64_t* __restrict__ keys, int64_t n, KeyHash h) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t key = keys[i];
    uint64_t s = kh_slot(h, key);
    for (uint64_t probe = 0; probe <= h.mask; ++probe) {  // keys are distinct: the first empty slot is ours
        const unsigned long long prev =
            atomicCAS(reinterpret_cast<unsigned long long*>(h.keys + s), ~0ull, (unsigned long long)key);
        if (prev == ~0ull) {
            h.pos[s] = (int32_t)i;
            return;
        }
        s = (s + 1) & h.mask;
    }
}

__device__ __forceinline__ int64_t kh_find(const KeyHash& h, int64_t key) {
    uint64_t s = kh_slot(h, key);
    for (uint64_t probe = 0; probe <= h.mask; ++probe) {
        const int64_t k = h.keys[s];
        if (k == key) return h.pos[s];
        if (k == -1) return -1;
        s = (s + 1) & h.mask;
    }
    return -1;
}

__device__ __forceinline__ int64_t locate(const int64_t* keys, int64_t n, int64_t i, int64_t key, int64_t bl,
                                          const KeyHash& h) {
    const int64_t d = bl > key ? bl - key : key - bl;
    return d <= 4 ? find_near(keys, n, i, key, bl) : kh_find(h, bl);
}

__global__ void k_find_nn(const int64_t* keys, int64_t n, Geometry geo, int kind, KeyHash h, int32_t* out) {
    const int nnn = kind == SGB_NN_STAR ? 8 : 27;
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t chunk = t / nnn;
    const int o = (int)(t - chunk * nnn);
    if (chunk >= n) return;
    const int64_t key = keys[chunk];
    int64_t bc[3];
    block_coords(geo, key, bc);
    int64_t pos = -1;
    if (kind == SGB_NN_STAR) {
        if (o < 2 * geo.dim) {
            const int d = o / 2;
            int64_t dpos = 0;
#pragma unroll
            for (int e = 0; e < 3; ++e)
                if (e == d) {
                    dpos = bc[e] + (o % 2) * 2 - 1;
                    bc[e] = dpos;
                }
            if (dpos >= 0) {
                const int64_t bl = block_lin_ref(geo, bc);
                if (bl >= 0 && bl != key) pos = locate(keys, n, chunk, key, bl, h);
                else if (bl == key) pos = chunk;
            }
        }
    } else if (o != nnn / 2) {
        int cnt = o;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            if (d < geo.dim) bc[d] += cnt % 3 - 1;
            cnt /= 3;
        }
        const int64_t bl = block_lin_ref(geo, bc);
        if (bl >= 0 && bl != key) pos = locate(keys, n, chunk, key, bl, h);
        else if (bl == key) pos = chunk;
    }
    out[t] = (int32_t)pos;
}

// Existence bitmap of every chunk: point p of a chunk is bit (p & 63) of
// word (p >> 6).  The chunk size is a multiple of 64, so the points of mask
// bytes [16k, 16k + 16) of the whole map are the 16-bit field k % 4 of bitmap
// word k / 4: one thread per 16 mask bytes, one 16-byte load, one 2-byte store.
__global__ void k_bits(const uint8_t* __restrict__ mask, int64_t n, int bs, uint64_t* bits) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= n * (bs >> 4)) return;
    const uint4 v = __ldg(reinterpret_cast<const uint4*>(mask) + t);
    // bit 0 of each of the four bytes of w, as four bits
    auto four = [](unsigned w) {
        const unsigned x = w & 0x01010101u;
        return (x | x >> 7 | x >> 14 | x >> 21) & 0xfu;
    };
    const unsigned b = four(v.x) | four(v.y) << 4 | four(v.z) << 8 | four(v.w) << 12;
    reinterpret_cast<uint16_t*>(bits)[t] = (uint16_t)b;
}

// tagBoundaries (src/SparseGridGpu/SparseGridGpu_kernels.cuh:676-737) with
// NNStar::isPadding (SparseGridGpu_ker_util.hpp:141-157) for 8^3 chunks: one
// warp per chunk; lanes 0..7 hold the 64-bit z-slices of the existence
// bitmap, neighbours along x/y are word shifts with the facing column / row
// of the adjacent chunk, along z the adjacent lane's word (shuffle) or the
// facing slice of the adjacent chunk.  EXIST points get PADDING set when a
// face neighbour is missing and cleared otherwise; other bytes are untouched.
__global__ void k_tag_star8(const uint64_t* bits, const int32_t* nn, int64_t n, uint8_t* mask) {
    const int64_t chunk = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (chunk >= n) return;
    constexpr uint64_t COL0 = 0x0101010101010101ull, COL7 = COL0 << 7;
    const int z = lane & 7;
    const int32_t* nb = nn + chunk * 8;
    const uint64_t W = bits[chunk * 8 + z];
    const int32_t xm = nb[0], xp = nb[1], ym = nb[2], yp = nb[3], zm = nb[4], zp = nb[5];
    const uint64_t XM = xm >= 0 ? bits[(int64_t)xm * 8 + z] : 0;
    const uint64_t XP = xp >= 0 ? bits[(int64_t)xp * 8 + z] : 0;
    const uint64_t YM = ym >= 0 ? bits[(int64_t)ym * 8 + z] : 0;
    const uint64_t YP = yp >= 0 ? bits[(int64_t)yp * 8 + z] : 0;
    const uint64_t up = __shfl_up_sync(0xffffffffu, W, 1);
    const uint64_t dn = __shfl_down_sync(0xffffffffu, W, 1);
    const uint64_t ZMw = z == 0 ? (zm >= 0 ? bits[(int64_t)zm * 8 + 7] : 0) : up;
    const uint64_t ZPw = z == 7 ? (zp >= 0 ? bits[(int64_t)zp * 8 + 0] : 0) : dn;
    const uint64_t exm = ((W << 1) & ~COL0) | ((XM & COL7) >> 7);
    const uint64_t exp_ = ((W >> 1) & ~COL7) | ((XP & COL0) << 7);
    const uint64_t eym = (W << 8) | (YM >> 56);
    const uint64_t eyp = (W >> 8) | (YP << 56);
    const uint64_t pad = W & ~(exm & exp_ & eym & eyp & ZMw & ZPw);
    // lane l rewrites mask bytes [16l, 16l+16): z-slice l/4, bits 16*(l%4)..
    const uint64_t pw = __shfl_sync(0xffffffffu, pad, lane >> 2);
    const unsigned bits16 = (unsigned)(pw >> (16 * (lane & 3))) & 0xffffu;
    uint4* mp = reinterpret_cast<uint4*>(mask + (size_t)chunk * 512) + lane;
    uint4 v = *mp;
    unsigned w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        unsigned out = 0;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            unsigned m = (w[q] >> (8 * b)) & 0xffu;
            if (m & 1u) m = ((bits16 >> (q * 4 + b)) & 1u) ? (m | 2u) : (m & ~2u);
            out |= m << (8 * b);
        }
        w[q] = out;
    }
    *mp = make_uint4(w[0], w[1], w[2], w[3]);
}

// Generic tagBoundaries for any edge and both neighbourhoods: one CTA per
// chunk, the 27 (or 7) neighbouring existence bitmaps staged in shared
// memory, one thread per point.  NNFull isPadding (SparseGridGpu.hpp:200-228)
// tests the whole 3x3x3 box.
__global__ void k_tag_generic(const uint64_t* bits, const int32_t* nn, int64_t n, int edge, int kind, uint8_t* mask) {
    __shared__ uint64_t nbw[27][8];
    const int64_t chunk = blockIdx.x;
    if (chunk >= n) return;
    const int bs = edge * edge * edge, words = bs / 64;
    for (int t = threadIdx.x; t < 27 * words; t += blockDim.x) {
        const int c = t / words, w = t % words;
        int64_t src = -1;
        if (c == 13) src = chunk;
        else if (kind == SGB_NN_FULL) src = nn[chunk * 27 + c];
        else {
            // faces only: c = (dx+1) + 3(dy+1) + 9(dz+1)
            const int slot = c == 12 ? 0 : c == 14 ? 1 : c == 10 ? 2 : c == 16 ? 3 : c == 4 ? 4 : c == 22 ? 5 : -1;
            src = slot >= 0 ? nn[chunk * 8 + slot] : -1;
        }
        nbw[c][w] = src >= 0 ? bits[src * words + w] : 0;
    }
    __syncthreads();
    for (int p = threadIdx.x; p < bs; p += blockDim.x) {
        uint8_t m = mask[(size_t)chunk * bs + p];
        if (!(m & 1)) continue;
        const int x = p % edge, y = (p / edge) % edge, z = p / (edge * edge);
        bool pad = false;
        for (int q = 0; q < 27 && !pad; ++q) {
            const int dx = q % 3 - 1, dy = (q / 3) % 3 - 1, dz = q / 9 - 1;
            if (kind == SGB_NN_STAR && (dx != 0) + (dy != 0) + (dz != 0) != 1) continue;
            int nx = x + dx, ny = y + dy, nz = z + dz;
            const int c = (nx < 0 ? 0 : nx >= edge ? 2 : 1) + 3 * (ny < 0 ? 0 : ny >= edge ? 2 : 1) +
                          9 * (nz < 0 ? 0 : nz >= edge ? 2 : 1);
            nx = (nx + edge) % edge;
            ny = (ny + edge) % edge;
            nz = (nz + edge) % edge;
            const int l = nx + edge * (ny + edge * nz);
            pad |= !((nbw[c][l >> 6] >> (l & 63)) & 1);
        }
        mask[(size_t)chunk * bs + p] = pad ? (uint8_t)(m | 2u) : (uint8_t)(m & ~2u);
    }
}

int ensure_neighbours(sgb_grid* g, int nn, cudaStream_t s) {
    if (g->nn_valid[nn]) return SGB_OK;
    const int nnn = nn == SGB_NN_STAR ? 8 : 27;
    SGB_TRY(g->nn[nn].grow((size_t)(g->n + 1) * nnn * 4));
    if (g->n > 0) {
        int b = 10;
        while ((int64_t(1) << b) < 2 * g->n) ++b;
        const int64_t cap = int64_t(1) << b;
        // the other table valid means the keys are those the hash was built from
        const bool reuse = g->nnhash_ok && g->nn_valid[1 - nn] && g->nnhash.bytes >= (size_t)cap * 12;
        SGB_TRY(g->nnhash.grow((size_t)cap * 12));
        KeyHash h{g->nnhash.as<int64_t>(), reinterpret_cast<int32_t*>(g->nnhash.as<int64_t>() + cap),
                  (uint64_t)cap - 1, 64 - b};
        if (!reuse) {
            SGB_CUDA(cudaMemsetAsync(h.keys, 0xff, (size_t)cap * 8, s));
            k_kh_build<<<(unsigned)((g->n + 255) / 256), 256, 0, s>>>(g->keys.as<int64_t>(), g->n, h);
            SGB_CUDA(cudaGetLastError());
            g->nnhash_ok = true;
        }
        const int64_t total = g->n * nnn;
        k_find_nn<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(g->keys.as<int64_t>(), g->n, g->geo, nn, h,
                                                                   g->nn[nn].as<int32_t>());
        SGB_CUDA(cudaGetLastError());
    }
    g->nn_valid[nn] = true;
    return SGB_OK;
}

int ensure_bits(sgb_grid* g, cudaStream_t s) {
    if (g->bits_valid) return SGB_OK;
    const int words = g->geo.bs / 64;
    SGB_TRY(g->bits.grow((size_t)(g->n + 1) * words * 8));
    if (g->n > 0) {
        const int64_t threads = g->n * (g->geo.bs / 16);
        k_bits<<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(g->mask.as<uint8_t>(), g->n, g->geo.bs,
                                                                  g->bits.as<uint64_t>());
        SGB_CUDA(cudaGetLastError());
    }
    g->bits_valid = true;
    return SGB_OK;
}

}  // namespace sgb

using namespace sgb;

extern "C" {

int sgb_find_neighbours(sgb_grid* g, int nn, sgb_stream s) {
    if (!g || (nn != SGB_NN_STAR && nn != SGB_NN_FULL)) return SGB_EINVAL;
    g->nn_valid[nn] = false;
    return ensure_neighbours(g, nn, (cudaStream_t)s);
}

int sgb_neighbour_table(sgb_grid* g, int nn, int64_t* out, sgb_stream stream) {
    if (!g || !out || (nn != SGB_NN_STAR && nn != SGB_NN_FULL)) return SGB_EINVAL;
    cudaStream_t s = (cudaStream_t)stream;
    SGB_TRY(ensure_neighbours(g, nn, s));
    const int nnn = nn == SGB_NN_STAR ? 8 : 27;
    std::vector<int32_t> h((size_t)g->n * nnn);
    if (g->n) SGB_CUDA(cudaMemcpyAsync(h.data(), g->nn[nn].p, h.size() * 4, cudaMemcpyDeviceToHost, s));
    SGB_CUDA(cudaStreamSynchronize(s));
    for (size_t i = 0; i < h.size(); ++i) {
        const int o = (int)(i % nnn);
        if (nn == SGB_NN_STAR && o >= 2 * g->geo.dim) out[i] = -1;  // unused NNStar slots
        else out[i] = h[i] < 0 ? g->n : h[i];                      // background position
    }
    return SGB_OK;
}

int sgb_tag_boundaries(sgb_grid* g, int nn, sgb_stream stream) {
    if (!g || (nn != SGB_NN_STAR && nn != SGB_NN_FULL)) return SGB_EINVAL;
    cudaStream_t s = (cudaStream_t)stream;
    if (g->n == 0) return SGB_OK;
    SGB_TRY(ensure_neighbours(g, nn, s));
    SGB_TRY(ensure_bits(g, s));
    if (nn == SGB_NN_STAR && g->geo.edge == 8) {
        const int64_t threads = g->n * 32;
        k_tag_star8<<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(g->bits.as<uint64_t>(), g->nn[0].as<int32_t>(),
                                                                      g->n, g->mask.as<uint8_t>());
    } else {
        k_tag_generic<<<(unsigned)g->n, 128, 0, s>>>(g->bits.as<uint64_t>(), g->nn[nn].as<int32_t>(), g->n,
                                                     g->geo.edge, nn, g->mask.as<uint8_t>());
    }
    SGB_CUDA(cudaGetLastError());
    return SGB_OK;
}

}  // extern "C"
