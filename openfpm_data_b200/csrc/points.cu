// The existing-point list and the point-list ("no shared memory") stencil mode.
//
// tagBoundaries(..., CALCULATE_EXISTING_POINTS) (SparseGridGpu.hpp:2354-2387,
// kernels calc_exist_points / fill_e_points, SparseGridGpu_kernels.cuh:
// 1152-1225) lists every existing point as chunk position * chunk size +
// offset (e_points).  applyStencils in STENCIL_MODE_INPLACE_NO_SHARED
// (SparseGridGpu.hpp:1051-1075 -> applyStencilInPlaceNoShared,
// SparseGridGpu_kernels.cuh:1096-1150) runs one thread per listed point, and
// the stencil reads its neighbours point by point through the NNFull table
// (getNNPoint, SparseGridGpu_ker.cuh:297-327) instead of a shared-memory tile.
// The stencil of that mode in the reference is Conv3x3x3_noshared
// (src/SparseGridGpu/tests/SparseGridGpu_tests.cu:955-1010).
//
// The list here is in (chunk position, offset) order (the reference fills it
// through a shared-memory atomic counter, any order inside a chunk; the
// stencil results do not depend on it) and is rebuilt whenever existence
// changed since it was made.
#include <algorithm>

#include "common.cuh"
#include "internal.h"
#include "stencil.cuh"

namespace sgb {

// The list is read off the existence bitmaps (one bit per point, kept for
// tagBoundaries): 64 bytes per 8^3 chunk instead of its 512 mask bytes.
// Counting: one thread per chunk, the popcount of its bs / 64 words.
__global__ void k_ep_count(const uint64_t* __restrict__ bits, int64_t n, int bs, uint32_t* counts) {
    const int words = bs >> 6;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += stride) {
        uint32_t t = 0;
        for (int k = 0; k < words; ++k) t += (uint32_t)__popcll(__ldg(bits + c * words + k));
        counts[c] = t;
    }
}

// Emission: warp per chunk, lane l owns points [l * P, l * P + P) with P = bs / 32; a warp
// scan of the lanes' counts places each lane's ids, written in point order.  The next chunk's
// bitmap slice and offset are loaded before the current chunk is written out.
__global__ void k_ep_emit(const uint64_t* __restrict__ bits, int64_t n, int bs, const uint32_t* __restrict__ offs,
                          uint32_t* out) {
    constexpr unsigned kAll = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int P = bs >> 5, words = bs >> 6;
    const int first = lane * P, wi = first >> 6, sh = first & 63;
    const uint32_t pmask = P >= 32 ? ~0u : (1u << P) - 1u;
    int64_t c = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    uint32_t m = 0, pos = 0;
    if (c < n) {
        m = (uint32_t)(__ldg(bits + c * words + wi) >> sh) & pmask;
        pos = __ldg(offs + c);
    }
    for (; c < n; c += nw) {
        const int64_t cn = c + nw;
        uint32_t mn = 0, posn = 0;
        if (cn < n) {
            mn = (uint32_t)(__ldg(bits + cn * words + wi) >> sh) & pmask;
            posn = __ldg(offs + cn);
        }
        const uint32_t cnt = __popc(m);
        uint32_t pre = cnt;  // inclusive prefix over the lanes
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t v = __shfl_up_sync(kAll, pre, o);
            if (lane >= o) pre += v;
        }
        uint32_t p = pos + pre - cnt;
        const uint32_t base = (uint32_t)(c * bs) + (uint32_t)first;
        while (m) {
            out[p++] = base + (uint32_t)(__ffs(m) - 1);
            m &= m - 1;
        }
        m = mn;
        pos = posn;
    }
}

int ensure_point_list(sgb_grid* g, cudaStream_t s) {
    if (g->epts_valid) return SGB_OK;
    const int64_t n = g->n, bs = g->geo.bs;
    if ((n + 1) * bs > (int64_t(1) << 32)) {  // ids and the background chunk's points fit 32 bits
        set_error("the existing-point list holds 32-bit point ids: at most 2^32 chunk points");
        return SGB_ERANGE;
    }
    g->nepts = 0;
    if (n > 0) {
        SGB_TRY(g->scratch[1].ensure((size_t)n * 4 + 16));
        SGB_TRY(g->scratch[2].ensure((size_t)(n + 1) * 4 + 16));
        uint32_t* counts = g->scratch[1].as<uint32_t>();
        uint32_t* offs = g->scratch[2].as<uint32_t>();
        const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>((int64_t)g->num_sms * 8, (n + 7) / 8));
        SGB_TRY(ensure_bits(g, s));
        const unsigned cblocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>((int64_t)g->num_sms * 16, (n + 255) / 256));
        k_ep_count<<<cblocks, 256, 0, s>>>(g->bits.as<uint64_t>(), n, (int)bs, counts);
        SGB_CUDA(cudaGetLastError());
        SGB_TRY(scan_exclusive_u32(counts, offs, n, offs + n, &g->scratch[6], s));
        SGB_TRY(g->hscratch.ensure(64));
        SGB_CUDA(cudaMemcpyAsync(g->hscratch.p, offs + n, 4, cudaMemcpyDeviceToHost, s));
        SGB_CUDA(cudaStreamSynchronize(s));
        g->nepts = *(uint32_t*)g->hscratch.p;
        SGB_TRY(g->epts.grow((size_t)g->nepts * 4 + 16));
        k_ep_emit<<<blocks, 256, 0, s>>>(g->bits.as<uint64_t>(), n, (int)bs, offs, g->epts.as<uint32_t>());
        SGB_CUDA(cudaGetLastError());
    }
    g->epts_valid = true;
    return SGB_OK;
}

// Conv3x3x3_noshared over the point list: tot = fma(value, c[i][j][k], tot)
// with the neighbour at (x+k-1, y+j-1, z+i-1), i outermost.  Neighbour values
// are read as stored (the grid keeps the background in non-existing points
// and in the background chunk, where absent neighbours point).
template <int E, bool XOUTER>
__global__ void __launch_bounds__(256) k_box27_points(const float* __restrict__ src, float* __restrict__ dst,
                                                      const uint8_t* __restrict__ mask, const int32_t* __restrict__ nn,
                                                      const int64_t* __restrict__ keys, const uint32_t* __restrict__ pts,
                                                      int64_t npts, int64_t n, Geometry geo, StencilParams prm) {
    constexpr int BS = E * E * E;
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= npts) return;
    const uint32_t id = pts[t];
    const int64_t c = id / BS;
    const int off = (int)(id % BS);
    const uint8_t m = mask[id];
    const int x = off % E, y = (off / E) % E, z = off / (E * E);
    bool act = (m & 1) && !(m & 2);
    if (prm.has_box) {
        int64_t o[3];
        chunk_origin(geo, keys[c], o);
        act = act && in_box(prm, o[0] + x, o[1] + y, o[2] + z);
    }
    if (!act) return;
    // per axis and offset -1 / 0 / +1: the neighbour chunk's component (0, 1, 2) and the local
    // coordinate's contribution to the point offset; ids are below 2^32, so 32-bit arithmetic
    const uint32_t cc = (uint32_t)c;
    int sx[3], sy[3], sz[3];
    uint32_t ox[3], oy[3], oz[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int qx = x + k - 1, qy = y + k - 1, qz = z + k - 1;
        const int px = qx < 0 ? 0 : (qx >= E ? 2 : 1), py = qy < 0 ? 0 : (qy >= E ? 2 : 1),
                  pz = qz < 0 ? 0 : (qz >= E ? 2 : 1);
        sx[k] = px;
        sy[k] = 3 * py;
        sz[k] = 9 * pz;
        ox[k] = (uint32_t)(qx + (1 - px) * E);
        oy[k] = (uint32_t)((qy + (1 - py) * E) * E);
        oz[k] = (uint32_t)((qz + (1 - pz) * E) * E * E);
    }
    const int32_t* row = nn + (int64_t)c * 27;
    float tot = 0.0f;
    auto term = [&](int kx, int jy, int iz, float cf) {
        const int slot = sx[kx] + sy[jy] + sz[iz];
        uint32_t pos = cc;
        if (slot != 13) {
            const int32_t v = __ldg(row + slot);
            pos = v < 0 ? (uint32_t)n : (uint32_t)v;
        }
        tot = __fmaf_rn(__ldg(src + (pos * BS + ox[kx] + oy[jy] + oz[iz])), cf, tot);
    };
    if (XOUTER) {
        // Conv3x3x3 (the shared-tile stencil's order): x offset outermost, z innermost, c[a][b][d]
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b)
#pragma unroll
                for (int d = 0; d < 3; ++d) term(a, b, d, prm.coeff[a * 9 + b * 3 + d]);
    } else {
        // Conv3x3x3_noshared: z offset outermost, x innermost, c[i][j][k]
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j)
#pragma unroll
                for (int k = 0; k < 3; ++k) term(k, j, i, prm.coeff[i * 9 + j * 3 + k]);
    }
    dst[id] = tot;
}

static int launch_points(sgb_grid* g, const int* src, const int* dst, const StencilParams& prm, bool xouter,
                         cudaStream_t s) {
    if (g->n == 0) return SGB_OK;
    SGB_TRY(ensure_neighbours(g, SGB_NN_FULL, s));
    SGB_TRY(ensure_clean(g, src[0], s));
    SGB_TRY(ensure_point_list(g, s));
    if (g->nepts == 0) return SGB_OK;
    const unsigned blocks = (unsigned)((g->nepts + 255) / 256);
    const float* in = g->data[src[0]].as<float>();
    float* out = g->data[dst[0]].as<float>();
#define SGB_PTS(E, X)                                                                                               \
    k_box27_points<E, X><<<blocks, 256, 0, s>>>(in, out, g->mask.as<uint8_t>(), g->nn[SGB_NN_FULL].as<int32_t>(),  \
                                                g->keys.as<int64_t>(), g->epts.as<uint32_t>(), g->nepts, g->n, g->geo, \
                                                prm)
    if (g->geo.edge == 8) {
        if (xouter) SGB_PTS(8, true);
        else SGB_PTS(8, false);
    } else {
        if (xouter) SGB_PTS(4, true);
        else SGB_PTS(4, false);
    }
#undef SGB_PTS
    SGB_CUDA(cudaGetLastError());
    return SGB_OK;
}

int launch_points_box27(sgb_grid* g, const int* src, const int* dst, const StencilParams& prm, cudaStream_t s) {
    return launch_points(g, src, dst, prm, false, s);
}

// Conv3x3x3 over the existing-point list when the chunks are sparse (fewer than an eighth of their
// points exist; measured break-even near a seventh): the same sums in the same order as the
// shared-tile kernels, without the per-chunk tile of mostly empty chunks.  Returns SGB_ENOTSUP
// when the chunks are not sparse.
int launch_points_box27_sparse(sgb_grid* g, const int* src, const int* dst, const StencilParams& prm,
                               cudaStream_t s) {
    if (g->n == 0) return SGB_OK;
    SGB_TRY(ensure_point_list(g, s));
    if (g->nepts * 8 >= g->n * (int64_t)g->geo.bs) return SGB_ENOTSUP;
    return launch_points(g, src, dst, prm, true, s);
}

}  // namespace sgb

using namespace sgb;

extern "C" int sgb_calc_existing_points(sgb_grid* g, int64_t* count, sgb_stream stream) {
    if (!g) return SGB_EINVAL;
    SGB_TRY(ensure_point_list(g, (cudaStream_t)stream));
    if (count) *count = g->nepts;
    return SGB_OK;
}

extern "C" int sgb_existing_point_list(sgb_grid* g, const uint32_t** ids_dev, int64_t* count, sgb_stream stream) {
    if (!g || !ids_dev || !count) return SGB_EINVAL;
    SGB_TRY(ensure_point_list(g, (cudaStream_t)stream));
    *ids_dev = g->epts.as<uint32_t>();
    *count = g->nepts;
    return SGB_OK;
}
