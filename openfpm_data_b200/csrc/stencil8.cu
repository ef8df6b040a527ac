// Pipelined 7-point stencil for 8^3 chunks (HEAT7, GS7).
//
// Reference path: applyStencilInPlace (src/SparseGridGpu/SparseGridGpu.hpp:
// 954-1048) launches one 512-thread CTA per chunk; loadGhostBlock_impl<1>
// (src/SparseGridGpu/SparseGridGpu_ker_util.hpp:487-564) gathers the 10^3
// tile point by point and substitutes the background where a mask byte is 0.
//
// Here: a persistent, warp-specialised kernel.  Each CTA owns a contiguous
// range of chunk positions.  One producer warp streams every chunk into an
// S-stage shared-memory ring with 1-D bulk copies (cp.async.bulk, the TMA
// engine): the source tiles (2 KB per field), the mask tile (512 B), the two
// z faces (256 B each) and the y=7 / y=0 rows of the y neighbours (8 x 32 B
// each); completion is counted in bytes on the stage's mbarrier.  The x halo
// is not fetched: an existing -x / +x neighbour is always the previous / next
// position of the sorted index (ids differ by one), which is in the ring
// already, so consumers keep a stage until the next chunk is done.  Eight
// consumer warps compute from shared memory and store to HBM.
//
// Points with mask byte 0 hold the background value in HBM (grid.cu keeps
// that invariant per property, see sgb_grid::clean), so a neighbour value is
// read as stored; the background is substituted only for neighbour chunks
// that do not exist.  Arithmetic is that of stencil.cuh.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstring>

#include "common.cuh"
#include "internal.h"
#include "stencil.cuh"

namespace sgb {

template <int NP>
struct alignas(128) Stage8 {
    float tile[NP][512];
    float ym[NP][64], yp[NP][64];  // [z*8 + x]: y = 7 row of the -y chunk / y = 0 row of the +y chunk
    float zm[NP][64], zp[NP][64];  // [y*8 + x]: z = 7 slice of the -z chunk / z = 0 slice of the +z chunk
    uint8_t mt[512];
    GridInfo gi;
    int32_t nn[8];
    int64_t key;
    int32_t par, active;
};

// The y faces of a chunk are 8 rows of 32 B, 256 B apart: one 3-D tensor
// copy each.  A field is viewed as a tensor [chunks*8 (z)][8 (y)][8 (x)] of
// float, box {8, 1, 8}; the x coordinate is always 0 (16-byte aligned).
struct TmapSet {
    CUtensorMap yface[2][2];  // [ping-pong buffer][field]
};

__device__ __forceinline__ void tma_yface(void* dst, const CUtensorMap* map, int y, int z, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(0), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

static int encode_yface(CUtensorMap* map, const float* base, int64_t chunks) {
    auto enc = tensor_map_encoder();
    if (!enc) {
        set_error("cuTensorMapEncodeTiled is not available from the driver");
        return SGB_ECUDA;
    }
    const cuuint64_t dims[3] = {8, 8, (cuuint64_t)std::max<int64_t>(chunks, 1) * 8};
    const cuuint64_t strides[2] = {8 * sizeof(float), 64 * sizeof(float)};
    const cuuint32_t box[3] = {8, 1, 8};
    const cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(base), dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error("cuTensorMapEncodeTiled failed");
        return SGB_ECUDA;
    }
    return SGB_OK;
}

template <int KIND, int NP>
__global__ void __launch_bounds__(kThreads, 2)
    k_stencil7_e8(FieldSet fs, const __grid_constant__ TmapSet tm, const uint8_t* __restrict__ mask,
                  const int32_t* __restrict__ nn, const int64_t* __restrict__ keys, const int32_t* __restrict__ gid,
                  const GridInfo* __restrict__ grids, GridInfo g0, int64_t n, Geometry geo, StencilParams prm,
                  int64_t t, int S, unsigned* err) {
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
            mbar_init(&full[s], 1);                // the producer's expect_tx arrival
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
        // Neighbour rows (8 ints per chunk, contiguous) are fetched in windows
        // of 8 chunks, one window ahead: lane l holds entries l and l + 32 of a
        // window, so no chunk waits on a dependent global load.
        const int64_t nnend = hi * 8;
        auto load_win = [&](int64_t first, int32_t& a, int32_t& b) {
            const int64_t e = first * 8 + lane;
            a = e < nnend ? nn[e] : -1;
            b = e + 32 < nnend ? nn[e + 32] : -1;
        };
        int32_t w0, w1, x0v, x1v;
        load_win(lo, w0, w1);
        load_win(lo + 8, x0v, x1v);
        int32_t gid_win = (grids && lo + lane < hi && lane < 8) ? gid[lo + lane] : 0;
        int32_t gid_nxt = (grids && lo + 8 + lane < hi && lane < 8) ? gid[lo + 8 + lane] : 0;
        int32_t g_last = -1;
        GridInfo gi = g0;
        for (; q < hi - lo; ++q) {
            const int64_t c = lo + q;
            const int s = (int)(q % S);
            const int j = (int)(q & 7);
            if (j == 0 && q > 0) {
                w0 = x0v;
                w1 = x1v;
                gid_win = gid_nxt;
                load_win(c + 8, x0v, x1v);
                gid_nxt = (grids && c + 8 + lane < hi && lane < 8) ? gid[c + 8 + lane] : 0;
            }
            const int32_t wsel = j < 4 ? w0 : w1;  // entries j*8 .. j*8+7 of the window
            const int32_t nb_cur = __shfl_sync(0xffffffffu, wsel, ((j & 3) << 3) + (lane & 7));
            if (grids) {
                const int32_t gc = __shfl_sync(0xffffffffu, gid_win, j);
                if (gc != g_last) {  // chunks of one grid are contiguous: one load per grid
                    gi = grids[gc];
                    g_last = gc;
                }
            }
            if (q >= S && !mbar_wait_bounded(&empty[s], (uint32_t)(q / S - 1) & 1u, err)) {
                ok = false;
                break;
            }
            Stage8<NP>& st = stage[s];
            const bool active = t >= gi.start && t < gi.start + gi.nsteps;
            const int par = (int)((t - gi.start) & 1);
            if (lane < 8) st.nn[lane] = nb_cur;
            if (lane == 0) {
                st.key = prm.has_box ? keys[c] : 0;
                st.gi = gi;
                st.par = par;
                st.active = active;
            }
            const int32_t fzm = __shfl_sync(0xffffffffu, nb_cur, 4), fzp = __shfl_sync(0xffffffffu, nb_cur, 5);
            const int32_t fym = __shfl_sync(0xffffffffu, nb_cur, 2), fyp = __shfl_sync(0xffffffffu, nb_cur, 3);
            __syncwarp();
            if (active) {
                const uint32_t faces = (fym >= 0) + (fyp >= 0) + (fzm >= 0) + (fzp >= 0);
                if (lane == 0) mbar_arrive_expect_tx(&full[s], NP * (2048 + 256 * faces) + 512);
                __syncwarp();
                const float* sp[2] = {fs.in[par][0], fs.in[par][NP - 1]};
                // per field: own tile, two z faces (contiguous), two y faces (tensor boxes); then the mask tile
                if (lane < NP * 5 + 1) {
                    const int tk = lane;
                    if (tk == NP * 5) {
                        bulk_g2s(st.mt, mask + c * 512, 512, &full[s]);
                    } else {
                        const int p = tk / 5, r = tk % 5;
                        const float* src = p == 0 ? sp[0] : sp[1];
                        if (r == 0) bulk_g2s(st.tile[p], src + c * 512, 2048, &full[s]);
                        else if (r == 1) { if (fzm >= 0) bulk_g2s(st.zm[p], src + (int64_t)fzm * 512 + 448, 256, &full[s]); }
                        else if (r == 2) { if (fzp >= 0) bulk_g2s(st.zp[p], src + (int64_t)fzp * 512, 256, &full[s]); }
                        else if (r == 3) { if (fym >= 0) tma_yface(st.ym[p], &tm.yface[par][p], 7, fym * 8, &full[s]); }
                        else { if (fyp >= 0) tma_yface(st.yp[p], &tm.yface[par][p], 0, fyp * 8, &full[s]); }
                    }
                }
            } else if (lane == 0) {
                mbar_arrive(&full[s]);
            }
        }
        if (!ok) {
            // let the copies already issued land before the CTA retires
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
            const int32_t n0 = st.nn[0], n1 = st.nn[1], n2 = st.nn[2], n3 = st.nn[3], n4 = st.nn[4], n5 = st.nn[5];
            // an absent neighbour is -1, which must not match position i - 1 of chunk 0
            const bool xm_ok = n0 >= 0 && n0 == (int32_t)(i - 1), xp_ok = n1 >= 0 && n1 == (int32_t)(i + 1);
            const uchar2 m2 = *reinterpret_cast<const uchar2*>(&st.mt[o0]);
            bool act0 = (m2.x & 1) && !(m2.x & 2), act1 = (m2.y & 1) && !(m2.y & 2);
            if (prm.has_box) {
                const int64_t key = st.key;
                const int64_t cx = (key % geo.bsz[0]) * 8 + x0, cy = ((key / geo.bsz[0]) % geo.bsz[1]) * 8 + y,
                              cz = (key / (geo.bsz[0] * geo.bsz[1])) * 8 + z;
                act0 = act0 && in_box(prm, cx, cy, cz);
                act1 = act1 && in_box(prm, cx + 1, cy, cz);
            }
            const bool need = KIND == SGB_HEAT7 || act0 || act1;
            if (need) {
                float2 c2[NP], lap[NP];
#pragma unroll
                for (int p = 0; p < NP; ++p) {
                    const float b = st.gi.bck[p];
                    const float2 c = *reinterpret_cast<const float2*>(&st.tile[p][o0]);
                    const float2 ym = y > 0 ? *reinterpret_cast<const float2*>(&st.tile[p][o0 - 8])
                                            : (n2 >= 0 ? *reinterpret_cast<const float2*>(&st.ym[p][z * 8 + x0]) : make_float2(b, b));
                    const float2 yp = y < 7 ? *reinterpret_cast<const float2*>(&st.tile[p][o0 + 8])
                                            : (n3 >= 0 ? *reinterpret_cast<const float2*>(&st.yp[p][z * 8 + x0]) : make_float2(b, b));
                    const float2 zm = z > 0 ? *reinterpret_cast<const float2*>(&st.tile[p][o0 - 64])
                                            : (n4 >= 0 ? *reinterpret_cast<const float2*>(&st.zm[p][y * 8 + x0]) : make_float2(b, b));
                    const float2 zp = z < 7 ? *reinterpret_cast<const float2*>(&st.tile[p][o0 + 64])
                                            : (n5 >= 0 ? *reinterpret_cast<const float2*>(&st.zp[p][y * 8 + x0]) : make_float2(b, b));
                    const float xm0 = x0 > 0 ? st.tile[p][o0 - 1] : (xm_ok ? pv.tile[p][o0 + 7] : b);
                    const float xp1 = x0 < 6 ? st.tile[p][o0 + 2] : (xp_ok ? nx.tile[p][o0 - 6] : b);
                    c2[p] = c;
                    lap[p].x = lap7(c.x, xm0, c.y, ym.x, yp.x, zm.x, zp.x);
                    lap[p].y = lap7(c.y, c.x, xp1, ym.y, yp.y, zm.y, zp.y);
                }
                const int64_t gidx = i * 512 + o0;
                float* d0 = fs.out[st.par][0];
                if (KIND == SGB_HEAT7) {
                    const float dt = st.gi.dt;
                    float2 r;
                    r.x = act0 ? __fmaf_rn(dt, lap[0].x, c2[0].x) : c2[0].x;
                    r.y = act1 ? __fmaf_rn(dt, lap[0].y, c2[0].y) : c2[0].y;
                    *reinterpret_cast<float2*>(d0 + gidx) = r;
                } else {
                    float* d1 = fs.out[st.par][NP - 1];
                    float2 un, vn;
                    gs_update(c2[0].x, c2[NP - 1].x, lap[0].x, lap[NP - 1].x, st.gi, un.x, vn.x);
                    gs_update(c2[0].y, c2[NP - 1].y, lap[0].y, lap[NP - 1].y, st.gi, un.y, vn.y);
                    if (act0 && act1) {
                        *reinterpret_cast<float2*>(d0 + gidx) = un;
                        *reinterpret_cast<float2*>(d1 + gidx) = vn;
                    } else if (act0) {
                        d0[gidx] = un.x;
                        d1[gidx] = vn.x;
                    } else if (act1) {
                        d0[gidx + 1] = un.y;
                        d1[gidx + 1] = vn.y;
                    }
                }
            }
        }
        if (i - 1 >= lo) {
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[(s + S - 1) % S]);
        }
    }
}

int launch_e8(const LaunchDesc& L, cudaStream_t s) {
    const int S = L.stages;
    const int np = L.kind == SGB_GS7 ? 2 : 1;
    TmapSet tm;
    std::memset(&tm, 0, sizeof(tm));
    for (int b = 0; b < 2; ++b)
        for (int p = 0; p < np; ++p) SGB_TRY(encode_yface(&tm.yface[b][p], L.fs.in[b][p], L.arr_chunks));
    if (L.kind == SGB_GS7) {
        const size_t smem = (size_t)S * sizeof(Stage8<2>) + 2 * S * 8;
        auto kern = k_stencil7_e8<SGB_GS7, 2>;
        SGB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        kern<<<L.ctas, kThreads, smem, s>>>(L.fs, tm, L.mask, L.nn, L.keys, L.gid, L.grids, L.g0, L.n, L.geo, L.prm,
                                            L.t, S, L.err);
    } else {
        const size_t smem = (size_t)S * sizeof(Stage8<1>) + 2 * S * 8;
        auto kern = k_stencil7_e8<SGB_HEAT7, 1>;
        SGB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        kern<<<L.ctas, kThreads, smem, s>>>(L.fs, tm, L.mask, L.nn, L.keys, L.gid, L.grids, L.g0, L.n, L.geo, L.prm,
                                            L.t, S, L.err);
    }
    SGB_CUDA(cudaGetLastError());
    return SGB_OK;
}

}  // namespace sgb
