// Ball-union scene builder: the block map of a grid (or of a new batch slot)
// from a union of balls, built on the device.  Used to admit solve requests
// without host-side point lists; no reference counterpart (reference users
// insert points from their own kernels, e.g. insertSphere3D,
// src/SparseGridGpu/tests/utils/SparseGridGpu_testKernels.cuh:144-200).
//
// A point p of the domain exists when |p - c|^2 <= r^2 (double precision) for
// some ball (c, r).  Initial values come from a counter-based hash of
// (seed, linear point id), so they do not depend on how the work is split:
//   SGB_INIT_UNIFORM     field 0 = U[0,1)
//   SGB_INIT_GRAY_SCOTT  u = 1, v = 0, and in the 6^3 cube [floor(c)-3,
//                        floor(c)+3) around each ball centre u = 0.5(1 +
//                        0.01 a), v = 0.25(1 + 0.01 b), a, b ~ U[-1,1)
#include <algorithm>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "internal.h"
#include "stencil.cuh"

namespace sgb {

struct Ball {
    double c[3];
    double r2;
    int64_t lo[3], hi[3];  // bounding box, inclusive
};

constexpr int kMaxBalls = 64;

struct BallSet {
    Ball b[kMaxBalls];
    int n;
};

__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

// U[0,1) with 24 random bits, exact in float32.
__device__ __forceinline__ float hash_unit(uint64_t seed, int64_t lin, uint64_t stream) {
    const uint64_t h = splitmix64(splitmix64(seed ^ (stream * 0xD1B54A32D192ED03ull)) ^ (uint64_t)lin);
    return (float)(h >> 40) * (1.0f / 16777216.0f);
}

// One warp per candidate chunk: the 512 (or 64) points tested against the
// balls, existence bitmap and point count of the chunk.
__global__ void k_ball_chunks(Geometry geo, BallSet balls, int64_t ncand, uint64_t* bits, uint32_t* flag) {
    const int64_t cand = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (cand >= ncand) return;
    const int e = geo.edge, words = geo.bs / 64;
    const int64_t bx = cand % geo.bsz[0], by = (cand / geo.bsz[0]) % geo.bsz[1], bz = cand / (geo.bsz[0] * geo.bsz[1]);
    // chunk / ball bounding-box test
    bool any = false;
    for (int k = 0; k < balls.n; ++k) {
        const Ball& b = balls.b[k];
        any |= bx * e <= b.hi[0] && bx * e + e - 1 >= b.lo[0] && by * e <= b.hi[1] && by * e + e - 1 >= b.lo[1] &&
               bz * e <= b.hi[2] && bz * e + e - 1 >= b.lo[2];
    }
    uint32_t count = 0;
    for (int r = 0; r < geo.bs / 32; ++r) {
        const int p = r * 32 + lane;
        const int64_t x = bx * e + p % e, y = by * e + (p / e) % e, z = bz * e + p / (e * e);
        bool in = false;
        if (any && x < geo.size[0] && y < geo.size[1] && z < geo.size[2]) {
            for (int k = 0; k < balls.n && !in; ++k) {
                const double dx = (double)x - balls.b[k].c[0], dy = (double)y - balls.b[k].c[1],
                             dz = (double)z - balls.b[k].c[2];
                in = dx * dx + dy * dy + dz * dz <= balls.b[k].r2;
            }
        }
        const unsigned w = __ballot_sync(0xffffffffu, in);
        count += __popc(w);
        if (lane == 0) {
            uint64_t* word = bits + cand * words + (r >> 1);
            if (r & 1) *word |= (uint64_t)w << 32;
            else *word = w;
        }
    }
    if (lane == 0) flag[cand] = count > 0;
}

// Emit the non-empty chunks: key, mask bytes, initial values.
__global__ void k_ball_emit(Geometry geo, BallSet balls, int64_t ncand, const uint64_t* bits, const uint32_t* flag,
                            const uint32_t* pos, int64_t base, int64_t* keys, uint8_t* mask, float* f0, float* f1,
                            int init, uint64_t seed, float bck0, float bck1) {
    const int64_t cand = blockIdx.x;
    if (cand >= ncand || !flag[cand]) return;
    const int e = geo.edge, bs = geo.bs, words = bs / 64;
    const int64_t out = base + pos[cand];
    if (threadIdx.x == 0) keys[out] = cand;
    const int64_t bx = cand % geo.bsz[0], by = (cand / geo.bsz[0]) % geo.bsz[1], bz = cand / (geo.bsz[0] * geo.bsz[1]);
    for (int p = threadIdx.x; p < bs; p += blockDim.x) {
        const bool ex = (bits[cand * words + (p >> 6)] >> (p & 63)) & 1;
        const int64_t x = bx * e + p % e, y = by * e + (p / e) % e, z = bz * e + p / (e * e);
        const int64_t lin = cand * bs + p;
        mask[out * bs + p] = ex ? 1 : 0;
        if (init == 0) {
            f0[out * bs + p] = ex ? hash_unit(seed, lin, 0) : bck0;
        } else {
            float u = 1.0f, v = 0.0f;
            bool cube = false;
            for (int k = 0; k < balls.n; ++k) {
                const int64_t cx = (int64_t)floor(balls.b[k].c[0]), cy = (int64_t)floor(balls.b[k].c[1]),
                              cz = (int64_t)floor(balls.b[k].c[2]);
                cube |= x >= cx - 3 && x < cx + 3 && y >= cy - 3 && y < cy + 3 && z >= cz - 3 && z < cz + 3;
            }
            if (cube) {
                u = 0.5f * (1.0f + 0.01f * (2.0f * hash_unit(seed, lin, 1) - 1.0f));
                v = 0.25f * (1.0f + 0.01f * (2.0f * hash_unit(seed, lin, 2) - 1.0f));
            }
            f0[out * bs + p] = ex ? u : bck0;
            f1[out * bs + p] = ex ? v : bck1;
        }
    }
}

int make_balls(const Geometry& geo, int nballs, const float* balls_host, BallSet& bs) {
    if (nballs < 1 || nballs > kMaxBalls || !balls_host) return SGB_EINVAL;
    std::memset(&bs, 0, sizeof(bs));
    bs.n = nballs;
    for (int k = 0; k < nballs; ++k) {
        Ball& b = bs.b[k];
        const double r = balls_host[4 * k + 3];
        for (int d = 0; d < 3; ++d) {
            b.c[d] = balls_host[4 * k + d];
            b.lo[d] = (int64_t)std::floor(b.c[d] - r);
            b.hi[d] = (int64_t)std::ceil(b.c[d] + r);
        }
        b.r2 = r * r;
    }
    (void)geo;
    return SGB_OK;
}

// Count the chunks of a ball set (bits / flags / positions in scratch).
int ball_pass1(const Geometry& geo, const BallSet& balls, DevBuf& bits, DevBuf& flag, DevBuf& pos, DevBuf& tmp,
               uint32_t* total_dev, cudaStream_t s, int64_t* ncand_out) {
    const int64_t ncand = geo.bsz[0] * geo.bsz[1] * geo.bsz[2];
    SGB_TRY(bits.ensure((size_t)ncand * (geo.bs / 64) * 8));
    SGB_TRY(flag.ensure((size_t)ncand * 4 + 16));
    SGB_TRY(pos.ensure((size_t)ncand * 4 + 16));
    k_ball_chunks<<<(unsigned)((ncand * 32 + 255) / 256), 256, 0, s>>>(geo, balls, ncand, bits.as<uint64_t>(),
                                                                        flag.as<uint32_t>());
    SGB_CUDA(cudaGetLastError());
    SGB_TRY(scan_exclusive_u32(flag.as<uint32_t>(), pos.as<uint32_t>(), ncand, total_dev, &tmp, s));
    *ncand_out = ncand;
    return SGB_OK;
}

}  // namespace sgb

using namespace sgb;

extern "C" int sgb_build_balls(sgb_grid* g, int nballs, const float* balls, int init, uint64_t seed, const int* props,
                               sgb_stream stream) {
    if (!g || !props || (init != 0 && init != 1)) return SGB_EINVAL;
    if (g->geo.zorder) {
        set_error("the scene builder writes x-fastest chunk ids");
        return SGB_ENOTSUP;
    }
    const int np = init == 1 ? 2 : 1;
    for (int j = 0; j < np; ++j)
        if (props[j] < 0 || props[j] >= g->nprop || g->ptype[props[j]] != SGB_F32) return SGB_EINVAL;
    cudaStream_t s = (cudaStream_t)stream;
    BallSet bset;
    SGB_TRY(make_balls(g->geo, nballs, balls, bset));
    int64_t ncand = 0;
    SGB_TRY(g->scratch[11].ensure(64));
    uint32_t* total = g->scratch[11].as<uint32_t>();
    SGB_TRY(ball_pass1(g->geo, bset, g->scratch[0], g->scratch[1], g->scratch[2], g->scratch[6], total, s, &ncand));
    SGB_TRY(g->hscratch.ensure(64));
    SGB_CUDA(cudaMemcpyAsync(g->hscratch.p, total, 4, cudaMemcpyDeviceToHost, s));
    SGB_CUDA(cudaStreamSynchronize(s));
    const int64_t n = *(uint32_t*)g->hscratch.p;
    SGB_TRY(grid_reserve(g, n, false));
    g->n = n;
    for (int p = 0; p < g->nprop; ++p) SGB_TRY(fill_background_all(g, p, s));
    float b0, b1;
    std::memcpy(&b0, g->bck[props[0]], 4);
    std::memcpy(&b1, g->bck[props[np - 1]], 4);
    if (ncand > 0)
        k_ball_emit<<<(unsigned)ncand, 256, 0, s>>>(g->geo, bset, ncand, g->scratch[0].as<uint64_t>(),
                                                    g->scratch[1].as<uint32_t>(), g->scratch[2].as<uint32_t>(), 0,
                                                    g->keys.as<int64_t>(), g->mask.as<uint8_t>(),
                                                    g->data[props[0]].as<float>(), g->data[props[np - 1]].as<float>(),
                                                    init, seed, b0, b1);
    SGB_CUDA(cudaGetLastError());
    g->npend = 0;
    SGB_TRY(write_background(g, n, s, g->data, g->mask));
    g->nn_valid[0] = g->nn_valid[1] = false;
    g->nnhash_ok = false;
    g->bits_valid = false;
    g->epts_valid = false;
    return SGB_OK;
}
