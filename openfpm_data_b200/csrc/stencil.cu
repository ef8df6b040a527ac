// Fixed-function stencils over the block map: HEAT7, GS7 and BOX27.
//
// Reference path: applyStencils -> applyStencilInPlace
// (src/SparseGridGpu/SparseGridGpu.hpp:954-1048) -> one 512-thread CTA per
// chunk, loadGhostBlock_impl<1> (SparseGridGpu_ker_util.hpp:487-564) gathers
// the 10^3 tile with one scalar load per point, the user functor computes,
// storeBlock writes back.
//
// Here (8^3 chunks, 7-point): a persistent, warp-specialised kernel.  Each CTA
// owns a contiguous range of chunk positions.  One producer warp streams, per
// chunk, the source tiles and the mask tile with 1-D bulk copies (TMA engine,
// cp.async.bulk) and the four y/z halo faces with cp.async into an S-stage
// shared-memory ring guarded by mbarriers.  The x halo is never fetched: when
// the -x / +x neighbour chunk exists it is the previous / next position of
// the sorted index (its id differs by one), which sits in the ring already,
// so the consumers keep a stage until the chunk after it is done.  Eight
// consumer warps compute from shared memory and store straight to HBM.
//
// The same kernels run a batch of grids concatenated into one block map: a
// per-chunk grid id selects the grid's parameters and its ping-pong buffer
// for global step t (GridInfo); a single grid is a batch of one.
//
// Semantics kept from the reference: a halo or centre value whose mask byte
// is 0 reads the background value; active = EXIST && !PADDING && inside the
// inclusive box; HEAT7 writes every point of the destination chunk (active
// points the update, the others the tile value, as storeBlock does), GS7 and
// BOX27 write active points only.  Arithmetic follows the reference's FP32
// association with nvcc's FMA contraction and flush-to-zero (-use_fast_math,
// src/CMakeLists.txt:158), written with explicit intrinsics so the compiler
// cannot re-associate it.
#include <algorithm>
#include <cstring>

#include "common.cuh"
#include "internal.h"
#include "stencil.cuh"

namespace sgb {

// ------------------------------------------------------------------ 8^3 pipelined kernel
template <int NP>
struct alignas(16) Stage8 {
    float tile[NP][512];
    float ym[NP][64], yp[NP][64], zm[NP][64], zp[NP][64];
    uint8_t mt[512];
    uint8_t mym[64], myp[64], mzm[64], mzp[64];
    GridInfo gi;
    int32_t nn[8];
    int64_t key;
    int32_t par, active;
};

template <int KIND, int NP>
__global__ void __launch_bounds__(kThreads, 2)
    k_stencil7_e8(FieldSet fs, const uint8_t* __restrict__ mask, const int32_t* __restrict__ nn,
                  const int64_t* __restrict__ keys, const int32_t* __restrict__ gid, const GridInfo* __restrict__ grids,
                  GridInfo g0, int64_t n, Geometry geo, StencilParams prm, int64_t t, int S, unsigned* err) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    Stage8<NP>* stage = reinterpret_cast<Stage8<NP>*>(smem_raw);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + (size_t)S * sizeof(Stage8<NP>));
    uint64_t* empty = full + S;

    const int64_t nct = gridDim.x;
    const int64_t c0 = n * blockIdx.x / nct, c1 = n * (blockIdx.x + 1) / nct;
    const int64_t lo = c0 > 0 ? c0 - 1 : 0, hi = c1 + 1 < n ? c1 + 1 : n;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&full[s], 33);               // 32 cp.async arrivals + 1 expect_tx arrival
            mbar_init(&empty[s], kConsumerWarps);  // one arrival per consumer warp
        }
        mbar_fence_init();
    }
    __syncthreads();
    if (c0 >= c1) return;

    if (warp == kConsumerWarps) {
        // ------------------------------------------------------------ producer
        int64_t q = 0;
        bool ok = true;
        for (; q < hi - lo; ++q) {
            const int64_t c = lo + q;
            const int s = (int)(q % S);
            const uint32_t k = (uint32_t)(q / S);
            if (q >= S && !mbar_wait_bounded(&empty[s], (k - 1) & 1u, err)) {
                ok = false;
                break;
            }
            Stage8<NP>& st = stage[s];
            const GridInfo gi = grids ? grids[gid[c]] : g0;
            const bool active = t >= gi.start && t < gi.start + gi.nsteps;
            const int par = (int)((t - gi.start) & 1);
            const int32_t nbv = lane < 8 ? nn[c * 8 + lane] : -1;
            if (lane < 8) st.nn[lane] = nbv;
            if (lane == 0) {
                st.key = keys[c];
                st.gi = gi;
                st.par = par;
                st.active = active;
            }
            const int32_t nby0 = __shfl_sync(0xffffffffu, nbv, 2), nby1 = __shfl_sync(0xffffffffu, nbv, 3),
                          nby2 = __shfl_sync(0xffffffffu, nbv, 4), nby3 = __shfl_sync(0xffffffffu, nbv, 5);
            __syncwarp();
            if (active) {
                const float* s0 = fs.in[par][0];
                const float* s1 = fs.in[par][NP - 1];
                if (lane == 0) {
                    mbar_arrive_expect_tx(&full[s], NP * 2048 + 512);
                    bulk_g2s(st.tile[0], s0 + c * 512, 2048, &full[s]);
                    if (NP == 2) bulk_g2s(st.tile[NP - 1], s1 + c * 512, 2048, &full[s]);
                    bulk_g2s(st.mt, mask + c * 512, 512, &full[s]);
                }
                for (int tk = lane; tk < NP * 64 + 24; tk += 32) {
                    if (tk < NP * 64) {
                        const int p = tk >> 6, r = tk & 63, f = r >> 4, piece = r & 15;
                        const int32_t nb = f == 0 ? nby0 : f == 1 ? nby1 : f == 2 ? nby2 : nby3;
                        if (nb < 0) continue;
                        const float* base = (p == 0 ? s0 : s1) + (int64_t)nb * 512;
                        const int zz = piece >> 1, hh = (piece & 1) * 4;
                        if (f == 0) cp_async16(&st.ym[p][zz * 8 + hh], base + zz * 64 + 56 + hh);
                        else if (f == 1) cp_async16(&st.yp[p][zz * 8 + hh], base + zz * 64 + hh);
                        else if (f == 2) cp_async16(&st.zm[p][piece * 4], base + 448 + piece * 4);
                        else cp_async16(&st.zp[p][piece * 4], base + piece * 4);
                    } else {
                        const int r = tk - NP * 64;
                        const int f = r < 8 ? 0 : r < 16 ? 1 : r < 20 ? 2 : 3;
                        const int32_t nb = f == 0 ? nby0 : f == 1 ? nby1 : f == 2 ? nby2 : nby3;
                        if (nb < 0) continue;
                        const uint8_t* base = mask + (int64_t)nb * 512;
                        if (f == 0) cp_async8(&st.mym[r * 8], base + r * 64 + 56);
                        else if (f == 1) cp_async8(&st.myp[(r - 8) * 8], base + (r - 8) * 64);
                        else if (f == 2) cp_async16(&st.mzm[(r - 16) * 16], base + 448 + (r - 16) * 16);
                        else cp_async16(&st.mzp[(r - 20) * 16], base + (r - 20) * 16);
                    }
                }
            } else if (lane == 0) {
                mbar_arrive(&full[s]);
            }
            cp_async_arrive_noinc(&full[s]);
        }
        if (!ok) {
            // drain own copies in flight before leaving
            cp_async_wait_all();
            for (int64_t r = q - 1; r >= 0 && r >= q - S; --r)
                mbar_wait_bounded(&full[r % S], (uint32_t)(r / S) & 1u, err, 100000000ull);
        }
        return;
    }

    // ---------------------------------------------------------------- consumers
    const int tid = threadIdx.x;
    const int z = tid >> 5, y = (tid >> 2) & 7, x0 = (tid & 3) << 1;
    const int o0 = z * 64 + y * 8 + x0;
    for (int64_t i = c0; i < c1; ++i) {
        const int64_t q = i - lo;
        const int s = (int)(q % S);
        if (!mbar_wait_bounded(&full[s], (uint32_t)(q / S) & 1u, err)) break;
        const bool has_next = i + 1 < hi;
        const int sn = (int)((q + 1) % S);
        if (has_next && !mbar_wait_bounded(&full[sn], (uint32_t)((q + 1) / S) & 1u, err)) break;
        const Stage8<NP>& st = stage[s];
        if (st.active) {
            const Stage8<NP>& pv = stage[(s + S - 1) % S];
            const Stage8<NP>& nx = stage[sn];
            const bool xm_ok = st.nn[0] == (int32_t)(i - 1);
            const bool xp_ok = st.nn[1] == (int32_t)(i + 1);
            const bool ym_ok = st.nn[2] >= 0, yp_ok = st.nn[3] >= 0, zm_ok = st.nn[4] >= 0, zp_ok = st.nn[5] >= 0;
            const float bck[2] = {st.gi.bck[0], st.gi.bck[1]};
            bool act[2];
            {
                int64_t cx = 0, cy = 0, cz = 0;
                if (prm.has_box) {
                    const int64_t key = st.key;
                    cx = (key % geo.bsz[0]) * 8;
                    cy = ((key / geo.bsz[0]) % geo.bsz[1]) * 8;
                    cz = (key / (geo.bsz[0] * geo.bsz[1])) * 8;
                }
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    const uint8_t m = st.mt[o0 + j];
                    act[j] = (m & 1) && !(m & 2);
                    if (prm.has_box) act[j] = act[j] && in_box(prm, cx + x0 + j, cy + y, cz + z);
                }
            }
            const bool need = KIND == SGB_HEAT7 || act[0] || act[1];
            float res[NP][2];
            if (need) {
#pragma unroll
                for (int p = 0; p < NP; ++p) {
                    float cv[2], xmv[2], xpv[2], ymv[2], ypv[2], zmv[2], zpv[2];
#pragma unroll
                    for (int j = 0; j < 2; ++j) {
                        const int x = x0 + j, o = o0 + j;
                        cv[j] = st.mt[o] ? st.tile[p][o] : bck[p];
                        if (x > 0) xmv[j] = st.mt[o - 1] ? st.tile[p][o - 1] : bck[p];
                        else xmv[j] = (xm_ok && pv.mt[o + 7]) ? pv.tile[p][o + 7] : bck[p];
                        if (x < 7) xpv[j] = st.mt[o + 1] ? st.tile[p][o + 1] : bck[p];
                        else xpv[j] = (xp_ok && nx.mt[o - 7]) ? nx.tile[p][o - 7] : bck[p];
                        if (y > 0) ymv[j] = st.mt[o - 8] ? st.tile[p][o - 8] : bck[p];
                        else ymv[j] = (ym_ok && st.mym[z * 8 + x]) ? st.ym[p][z * 8 + x] : bck[p];
                        if (y < 7) ypv[j] = st.mt[o + 8] ? st.tile[p][o + 8] : bck[p];
                        else ypv[j] = (yp_ok && st.myp[z * 8 + x]) ? st.yp[p][z * 8 + x] : bck[p];
                        if (z > 0) zmv[j] = st.mt[o - 64] ? st.tile[p][o - 64] : bck[p];
                        else zmv[j] = (zm_ok && st.mzm[y * 8 + x]) ? st.zm[p][y * 8 + x] : bck[p];
                        if (z < 7) zpv[j] = st.mt[o + 64] ? st.tile[p][o + 64] : bck[p];
                        else zpv[j] = (zp_ok && st.mzp[y * 8 + x]) ? st.zp[p][y * 8 + x] : bck[p];
                    }
#pragma unroll
                    for (int j = 0; j < 2; ++j) {
                        if (KIND == SGB_HEAT7)
                            res[p][j] = act[j] ? heat_update(cv[j], xmv[j], xpv[j], ymv[j], ypv[j], zmv[j], zpv[j],
                                                             st.gi.dt)
                                               : cv[j];
                        else
                            res[p][j] = lap7(cv[j], xmv[j], xpv[j], ymv[j], ypv[j], zmv[j], zpv[j]);
                    }
                }
            }
            const int64_t gidx = i * 512 + o0;
            float* d0 = fs.out[st.par][0];
            if (KIND == SGB_HEAT7) {
                *reinterpret_cast<float2*>(d0 + gidx) = make_float2(res[0][0], res[0][1]);
            } else if (need) {
                float* d1 = fs.out[st.par][NP - 1];
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    if (!act[j]) continue;
                    const float u = st.tile[0][o0 + j], v = st.tile[NP - 1][o0 + j];
                    float un, vn;
                    gs_update(u, v, res[0][j], res[NP - 1][j], st.gi, un, vn);
                    d0[gidx + j] = un;
                    d1[gidx + j] = vn;
                }
            }
        }
        if (i - 1 >= lo) {
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[(s + S - 1) % S]);
        }
    }
}

// ------------------------------------------------------------------ generic tile kernel
// Any edge, any of the three stencils: one CTA per chunk (grid-stride), the
// (edge+2)^3 tile gathered with one load per cell, as the reference's
// loadGhostBlock does, with NNFull edge/corner cells taken from the right
// neighbour.  Used for BOX27, for 4^3 chunks and as a cross-check.
template <int KIND, int E>
__global__ void __launch_bounds__(256) k_stencil_tile(FieldSet fs, const uint8_t* __restrict__ mask,
                                                      const int32_t* __restrict__ nn, const int64_t* __restrict__ keys,
                                                      const int32_t* __restrict__ gid,
                                                      const GridInfo* __restrict__ grids, GridInfo g0, int64_t n,
                                                      Geometry geo, StencilParams prm, int64_t t) {
    constexpr int T = E + 2, TT = T * T * T, BS = E * E * E;
    constexpr int NP = KIND == SGB_GS7 ? 2 : 1;
    constexpr bool FULLNB = KIND == SGB_BOX27;
    __shared__ float tile[NP][TT];
    for (int64_t chunk = blockIdx.x; chunk < n; chunk += gridDim.x) {
        const GridInfo gi = grids ? grids[gid[chunk]] : g0;
        if (!(t >= gi.start && t < gi.start + gi.nsteps)) continue;  // uniform across the CTA
        const int par = (int)((t - gi.start) & 1);
        const float* src[2] = {fs.in[par][0], fs.in[par][NP - 1]};
        for (int cell = threadIdx.x; cell < TT; cell += blockDim.x) {
            const int tx = cell % T, ty = (cell / T) % T, tz = cell / (T * T);
            const int dx = tx == 0 ? -1 : (tx == T - 1 ? 1 : 0);
            const int dy = ty == 0 ? -1 : (ty == T - 1 ? 1 : 0);
            const int dz = tz == 0 ? -1 : (tz == T - 1 ? 1 : 0);
            const int nz = (dx != 0) + (dy != 0) + (dz != 0);
            if (!FULLNB && nz > 1) continue;  // edges/corners unused by 7-point stencils
            int64_t sc = chunk;
            if (nz) {
                if (FULLNB) sc = nn[chunk * 27 + (dx + 1) + 3 * (dy + 1) + 9 * (dz + 1)];
                else sc = nn[chunk * 8 + (dx ? (dx < 0 ? 0 : 1) : dy ? (dy < 0 ? 2 : 3) : (dz < 0 ? 4 : 5))];
            }
            const int lx = (tx - 1 + E) % E, ly = (ty - 1 + E) % E, lz = (tz - 1 + E) % E;
            const int64_t idx = sc * BS + lx + E * (ly + E * lz);
            const bool ex = sc >= 0 && mask[idx] != 0;
#pragma unroll
            for (int p = 0; p < NP; ++p) tile[p][cell] = ex ? src[p][idx] : gi.bck[p];
        }
        __syncthreads();
        int64_t cx = 0, cy = 0, cz = 0;
        if (prm.has_box) {
            const int64_t key = keys[chunk];
            cx = (key % geo.bsz[0]) * E;
            cy = ((key / geo.bsz[0]) % geo.bsz[1]) * E;
            cz = (key / (geo.bsz[0] * geo.bsz[1])) * E;
        }
        float* d0 = fs.out[par][0];
        float* d1 = fs.out[par][NP - 1];
        for (int pnt = threadIdx.x; pnt < BS; pnt += blockDim.x) {
            const int x = pnt % E, y = (pnt / E) % E, z = pnt / (E * E);
            const uint8_t m = mask[chunk * BS + pnt];
            bool act = (m & 1) && !(m & 2);
            if (prm.has_box) act = act && in_box(prm, cx + x, cy + y, cz + z);
            const int c = (x + 1) + T * ((y + 1) + T * (z + 1));
            const int64_t gidx = chunk * BS + pnt;
            if (KIND == SGB_HEAT7) {
                const float cur = tile[0][c];
                d0[gidx] = act ? heat_update(cur, tile[0][c - 1], tile[0][c + 1], tile[0][c - T], tile[0][c + T],
                                             tile[0][c - T * T], tile[0][c + T * T], gi.dt)
                               : cur;
            } else if (KIND == SGB_GS7) {
                if (!act) continue;
                const float u = tile[0][c], v = tile[1][c];
                const float lu = lap7(u, tile[0][c - 1], tile[0][c + 1], tile[0][c - T], tile[0][c + T],
                                      tile[0][c - T * T], tile[0][c + T * T]);
                const float lv = lap7(v, tile[1][c - 1], tile[1][c + 1], tile[1][c - T], tile[1][c + T],
                                      tile[1][c - T * T], tile[1][c + T * T]);
                float un, vn;
                gs_update(u, v, lu, lv, gi, un, vn);
                d0[gidx] = un;
                d1[gidx] = vn;
            } else {
                if (!act) continue;
                // Conv3x3x3: tot += tile[x+i-1][y+j-1][z+k-1] * c[i][j][k], i outermost
                float tot = 0.0f;
#pragma unroll
                for (int a = 0; a < 3; ++a)
#pragma unroll
                    for (int b = 0; b < 3; ++b)
#pragma unroll
                        for (int d = 0; d < 3; ++d)
                            tot = __fmaf_rn(tile[0][c + (a - 1) + T * ((b - 1) + T * (d - 1))],
                                            prm.coeff[a * 9 + b * 3 + d], tot);
                d0[gidx] = tot;
            }
        }
        __syncthreads();
    }
}

int make_params(sgb_grid* g, int kind, const int* src, const int* dst, const float* params, int nparams,
                const int64_t* box, StencilParams& prm) {
    std::memset(&prm, 0, sizeof(prm));
    if (!src || !dst || (nparams > 0 && !params)) return SGB_EINVAL;
    if (kind < SGB_HEAT7 || kind > SGB_BOX27) return SGB_EINVAL;
    const int np = kind == SGB_GS7 ? 2 : 1;
    for (int j = 0; j < np; ++j) {
        if (src[j] < 0 || src[j] >= g->nprop || dst[j] < 0 || dst[j] >= g->nprop) return SGB_EINVAL;
        if (g->ptype[src[j]] != SGB_F32 || g->ptype[dst[j]] != SGB_F32) {
            set_error("stencils operate on float32 properties");
            return SGB_ENOTSUP;
        }
        for (int k = 0; k < np; ++k)
            if (src[j] == dst[k]) {
                set_error("a stencil may not write one of its source properties");
                return SGB_EINVAL;
            }
        std::memcpy(&prm.bck[j], g->bck[src[j]], 4);
    }
    if (np == 2 && (src[0] == src[1] || dst[0] == dst[1])) return SGB_EINVAL;
    if (kind == SGB_HEAT7) {
        if (nparams < 1) return SGB_EINVAL;
        prm.dt = params[0];
    } else if (kind == SGB_GS7) {
        if (nparams < 5) return SGB_EINVAL;
        prm.Du = params[0];
        prm.Dv = params[1];
        prm.F = params[2];
        prm.nFK = -(params[2] + params[3]);
        prm.dt = params[4];
    } else {
        if (nparams < 27) return SGB_EINVAL;
        for (int k = 0; k < 27; ++k) prm.coeff[k] = params[k];
    }
    if (box) {
        prm.has_box = 1;
        for (int d = 0; d < 3; ++d) {
            prm.box_lo[d] = box[d];
            prm.box_hi[d] = box[3 + d];
        }
        // a box covering the whole domain needs no per-point test
        bool all = true;
        for (int d = 0; d < 3; ++d) all &= box[d] <= 0 && box[3 + d] >= g->geo.size[d] - 1;
        if (all) prm.has_box = 0;
    }
    return SGB_OK;
}

GridInfo grid_info_of(const StencilParams& prm) {
    GridInfo gi;
    std::memset(&gi, 0, sizeof(gi));
    gi.start = 0;
    gi.nsteps = 1;
    gi.dt = prm.dt;
    gi.Du = prm.Du;
    gi.Dv = prm.Dv;
    gi.F = prm.F;
    gi.nFK = prm.nFK;
    gi.bck[0] = prm.bck[0];
    gi.bck[1] = prm.bck[1];
    return gi;
}

int launch_fields(const LaunchDesc& L, cudaStream_t s) {
    if (L.n == 0) return SGB_OK;
    const int np = L.kind == SGB_GS7 ? 2 : 1;
    if (L.kind != SGB_BOX27 && L.edge == 8 && !L.use_tile) {
        const int S = L.stages;
        if (np == 2) {
            const size_t smem = (size_t)S * sizeof(Stage8<2>) + 2 * S * 8;
            auto kern = k_stencil7_e8<SGB_GS7, 2>;
            SGB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            kern<<<L.ctas, kThreads, smem, s>>>(L.fs, L.mask, L.nn, L.keys, L.gid, L.grids, L.g0, L.n, L.geo, L.prm,
                                                L.t, S, L.err);
        } else {
            const size_t smem = (size_t)S * sizeof(Stage8<1>) + 2 * S * 8;
            auto kern = k_stencil7_e8<SGB_HEAT7, 1>;
            SGB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            kern<<<L.ctas, kThreads, smem, s>>>(L.fs, L.mask, L.nn, L.keys, L.gid, L.grids, L.g0, L.n, L.geo, L.prm,
                                                L.t, S, L.err);
        }
        SGB_CUDA(cudaGetLastError());
        return SGB_OK;
    }
    const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>(L.n, (int64_t)L.num_sms * 8));
#define SGB_TILE(K, E) \
    k_stencil_tile<K, E><<<blocks, 256, 0, s>>>(L.fs, L.mask, L.nn, L.keys, L.gid, L.grids, L.g0, L.n, L.geo, L.prm, L.t)
    if (L.kind == SGB_HEAT7) {
        if (L.edge == 8) SGB_TILE(SGB_HEAT7, 8);
        else SGB_TILE(SGB_HEAT7, 4);
    } else if (L.kind == SGB_GS7) {
        if (L.edge == 8) SGB_TILE(SGB_GS7, 8);
        else SGB_TILE(SGB_GS7, 4);
    } else {
        if (L.edge == 8) SGB_TILE(SGB_BOX27, 8);
        else SGB_TILE(SGB_BOX27, 4);
    }
#undef SGB_TILE
    SGB_CUDA(cudaGetLastError());
    return SGB_OK;
}

int launch_stencil_impl(sgb_grid* g, int kind, const int* src, const int* dst, const StencilParams& prm,
                        cudaStream_t s, bool use_tile) {
    if (g->n == 0) return SGB_OK;
    const int nnk = kind == SGB_BOX27 ? SGB_NN_FULL : SGB_NN_STAR;
    SGB_TRY(ensure_neighbours(g, nnk, s));
    const int np = kind == SGB_GS7 ? 2 : 1;
    LaunchDesc L;
    std::memset(&L, 0, sizeof(L));
    L.kind = kind;
    L.edge = g->geo.edge;
    L.use_tile = use_tile;
    L.stages = g->stages;
    L.num_sms = g->num_sms;
    L.ctas = (unsigned)std::max<int64_t>(1, std::min<int64_t>(g->n, (int64_t)g->num_sms * g->ctas_per_sm));
    for (int b = 0; b < 2; ++b)
        for (int j = 0; j < 2; ++j) {
            L.fs.in[b][j] = g->data[src[j < np ? j : 0]].as<float>();
            L.fs.out[b][j] = g->data[dst[j < np ? j : 0]].as<float>();
        }
    L.mask = g->mask.as<uint8_t>();
    L.nn = g->nn[nnk].as<int32_t>();
    L.keys = g->keys.as<int64_t>();
    L.gid = nullptr;
    L.grids = nullptr;
    L.g0 = grid_info_of(prm);
    L.n = g->n;
    L.geo = g->geo;
    L.prm = prm;
    L.t = 0;
    L.err = g->err.as<unsigned>();
    return launch_fields(L, s);
}

int launch_stencil(sgb_grid* g, int kind, const int* src, const int* dst, const StencilParams& prm, cudaStream_t s) {
    return launch_stencil_impl(g, kind, src, dst, prm, s, false);
}

}  // namespace sgb

using namespace sgb;

extern "C" {

int sgb_apply_stencil(sgb_grid* g, int kind, const int* src, const int* dst, const float* params, int nparams,
                      const int64_t* box, sgb_stream s) {
    if (!g) return SGB_EINVAL;
    StencilParams prm;
    SGB_TRY(make_params(g, kind, src, dst, params, nparams, box, prm));
    return launch_stencil(g, kind, src, dst, prm, (cudaStream_t)s);
}

// Same as sgb_apply_stencil through the generic one-chunk-per-CTA kernel
// (cross-check of the pipelined kernel; not part of the drop-in surface).
int sgb_apply_stencil_tiled(sgb_grid* g, int kind, const int* src, const int* dst, const float* params, int nparams,
                            const int64_t* box, sgb_stream s) {
    if (!g) return SGB_EINVAL;
    StencilParams prm;
    SGB_TRY(make_params(g, kind, src, dst, params, nparams, box, prm));
    return launch_stencil_impl(g, kind, src, dst, prm, (cudaStream_t)s, true);
}

int sgb_run_steps(sgb_grid* g, int kind, const int* src, const int* dst, const float* params, int nparams, int nsteps,
                  int use_graph, int* final_is_dst, sgb_stream stream) {
    if (!g || nsteps < 0) return SGB_EINVAL;
    cudaStream_t s = (cudaStream_t)stream;
    StencilParams fwd, bwd;
    SGB_TRY(make_params(g, kind, src, dst, params, nparams, nullptr, fwd));
    SGB_TRY(make_params(g, kind, dst, src, params, nparams, nullptr, bwd));
    if (final_is_dst) *final_is_dst = nsteps % 2;
    if (nsteps == 0 || g->n == 0) return SGB_OK;
    SGB_TRY(ensure_neighbours(g, kind == SGB_BOX27 ? SGB_NN_FULL : SGB_NN_STAR, s));
    if (!use_graph) {
        for (int k = 0; k < nsteps; ++k) {
            if (k % 2 == 0) SGB_TRY(launch_stencil(g, kind, src, dst, fwd, s));
            else SGB_TRY(launch_stencil(g, kind, dst, src, bwd, s));
        }
        return SGB_OK;
    }
    return run_graph(
        [&](cudaStream_t cs) -> int {
            for (int k = 0; k < nsteps; ++k) {
                int st = (k % 2 == 0) ? launch_stencil(g, kind, src, dst, fwd, cs)
                                      : launch_stencil(g, kind, dst, src, bwd, cs);
                if (st != SGB_OK) return st;
            }
            return SGB_OK;
        },
        s);
}

}  // extern "C"
