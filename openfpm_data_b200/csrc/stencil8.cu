// Pipelined 7-point stencil for 8^3 chunks (HEAT7, GS7).
//
// Reference path: applyStencilInPlace (src/SparseGridGpu/SparseGridGpu.hpp:
// 954-1048) launches one 512-thread CTA per chunk; loadGhostBlock_impl<1>
// (src/SparseGridGpu/SparseGridGpu_ker_util.hpp:487-564) gathers the 10^3
// tile point by point and substitutes the background where a mask byte is 0.
//
// Here every warp is an independent pipeline over a contiguous range [a, b)
// of chunk positions.  It streams [lo, hi), the range widened by one chunk on
// each side, through its own R-stage shared-memory ring: per chunk, lanes
// issue 1-D bulk copies (cp.async.bulk, the TMA engine) of the source tiles
// (2 KB per field) and the mask tile (512 B), counted in bytes on the stage's
// mbarrier.  The x halo is not fetched: an existing -x / +x neighbour is
// always the previous / next position of the sorted index, so it sits in the
// neighbouring stage of the same ring.  The y and z faces (256 B each per
// field) are not staged by the ring: each lane loads, one chunk ahead, one
// 16-byte quad of the z face its half of the warp needs and one of a y face
// (lanes 0-15 the -y face, 16-31 the +y face, [z][x quad]); the y faces are
// written once per chunk to a 0.5 / 1 KB per-warp buffer that the y = 0 /
// y = 7 lanes read.  Keeping faces out of the ring makes a stage 2.6 KB
// (heat) / 4.6 KB (Gray-Scott), so more warps fit on an SM.  While chunk q
// is computed, chunks up to q - 2 + R are in flight; after
// it, the stage of chunk q - 1 is refilled with chunk q - 1 + R.  A warp
// waits only on its own barriers, in order, so phase parities are exact and
// no warp ever waits for another.
//
// Compute: lanes 0-15 take z = 0..3 and lanes 16-31 z = 4..7; in each z
// slice a lane owns four x-adjacent points (16-byte loads and stores) of one
// y row and marches its four slices carrying z-1 / z / z+1 in registers.
//
// Points with mask byte 0 hold the background value in HBM (grid.cu keeps
// that invariant per property, see sgb_grid::clean), so a neighbour value is
// read as stored; the background is substituted only for neighbour chunks
// that do not exist.  Arithmetic is that of stencil.cuh.
#include <algorithm>
#include <cstring>

#include "common.cuh"
#include "internal.h"
#include "stencil.cuh"

namespace sgb {

constexpr int kWarps = 2;                  // warps per CTA, each its own pipeline
constexpr int kThreads8 = kWarps * 32;

template <int NP>
struct alignas(128) Stage8 {
    float tile[NP][512];
    uint8_t mt[512];
    GridInfo gi;
    float2 bk[NP];       // background of each source field, twice (read for absent x neighbours)
    int32_t nn[8];
    int32_t cx, cy, cz;  // first point of the chunk (box tests)
    int32_t par, active;
};

// y and z faces of one chunk in registers (see the file comment)
template <int NP>
struct Faces {
    // z face of the lane's half: the lane's own x quad in the z = 7 slice of the -z chunk (lanes 0-15) or
    // the z = 0 slice of the +z chunk (lanes 16-31)
    float4 zf[NP];
    // y face element [z = (lane & 15) / 2][x quad = lane & 1] of the y = 7 row of the -y chunk (lanes 0-15)
    // or the y = 0 row of the +y chunk (lanes 16-31)
    float4 yf[NP];
};

__device__ __forceinline__ float4 ldg_f4(const float* p) {
    return __ldg(reinterpret_cast<const float4*>(p));
}

template <int KIND, int NP, bool BOX>
__global__ void __launch_bounds__(kThreads8, KIND == SGB_GS7 ? 6 : 8)
    k_stencil7_e8(FieldSet fs, const uint8_t* __restrict__ mask, const int32_t* __restrict__ nn,
                  const int64_t* __restrict__ keys, const int32_t* __restrict__ gid,
                  const GridInfo* __restrict__ grids, GridInfo g0, int64_t n, Geometry geo, StencilParams prm,
                  int64_t t, int R, int64_t nwarps, unsigned* err) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    // Programmatic dependent launch: the next step's launch may begin while this one drains; no
    // field is read or written before the previous launch on the stream has completed.
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    Stage8<NP>* ring = reinterpret_cast<Stage8<NP>*>(smem_raw) + (size_t)warp * R;
    uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + (size_t)kWarps * R * sizeof(Stage8<NP>)) + warp * R;
    const int64_t gw = (int64_t)blockIdx.x * kWarps + warp;
    if (gw >= nwarps) return;
    const int64_t a = n * gw / nwarps, b = n * (gw + 1) / nwarps;
    if (a >= b) return;
    const int64_t lo = a > 0 ? a - 1 : 0, hi = b < n ? b + 1 : n;
    const int Q = (int)(hi - lo);
    if (lane == 0) {
        for (int r = 0; r < R; ++r) mbar_init(&full[r], 1);  // the issuing lane's expect_tx arrival
        mbar_fence_init();
    }
    __syncwarp();

    // ------------------------------------------------------------ issue side
    // Neighbour rows (8 ints per chunk, contiguous) are fetched in windows of
    // 8 chunks, one window ahead: lane l holds entries l and l + 32 of a window.
    const int64_t nnend = hi * 8;
    auto load_win = [&](int64_t first, int32_t& wa, int32_t& wb) {
        const int64_t e = first * 8 + lane;
        wa = e < nnend ? nn[e] : -1;
        wb = e + 32 < nnend ? nn[e + 32] : -1;
    };
    int32_t w0, w1, x0v, x1v;
    load_win(lo, w0, w1);
    load_win(lo + 8, x0v, x1v);
    int32_t gid_win = (grids && lo + lane < hi && lane < 8) ? gid[lo + lane] : 0;
    int32_t gid_nxt = (grids && lo + 8 + lane < hi && lane < 8) ? gid[lo + 8 + lane] : 0;
    int32_t g_last = -1;
    GridInfo gi = g0;
    // Fill ring slot `slot` with chunk lo + q; q increases by one per call.
    auto issue = [&](int q, int slot) {
        const int64_t c = lo + q;
        const int j = q & 7;
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
        Stage8<NP>& st = ring[slot];
        uint64_t* bar = &full[slot];
        const bool active = t >= gi.start && t < gi.start + gi.nsteps;
        const int par = (int)((t - gi.start) & 1);
        if (lane < 8) st.nn[lane] = nb_cur;
        if (lane == 0) {
            if (BOX) {
                const int64_t key = keys[c];
                int64_t o[3];
                chunk_origin(geo, key, o);
                st.cx = (int32_t)o[0];
                st.cy = (int32_t)o[1];
                st.cz = (int32_t)o[2];
            }
            st.gi = gi;
#pragma unroll
            for (int p = 0; p < NP; ++p) {
                const float bv = par ? gi.bck[1][p] : gi.bck[0][p];  // no dynamic index into a register struct
                st.bk[p] = make_float2(bv, bv);
            }
            st.par = par;
            st.active = active;
        }
        __syncwarp();
        if (active) {
            if (lane == 0) mbar_arrive_expect_tx(bar, NP * 2048 + 512);
            __syncwarp();
            // lanes 0..NP-1: the field tiles; lane NP: the mask tile
            if (lane <= NP) {
                const float* src = (lane == 0) ? (par ? fs.in[1][0] : fs.in[0][0])
                                               : (par ? fs.in[1][NP - 1] : fs.in[0][NP - 1]);
                if (lane < NP) bulk_g2s(st.tile[lane], src + c * 512, 2048, bar);
                else bulk_g2s(st.mt, mask + c * 512, 512, bar);
            }
        } else if (lane == 0) {
            mbar_arrive(bar);
        }
    };

    const int npro = Q < R ? Q : R;
    for (int q = 0; q < npro; ++q) issue(q, q);
    int issued = npro;

    // ------------------------------------------------------------ compute side
    // Lane l takes z = 4h .. 4h + 3 with h = l / 16 and, in each z slice, the x quad xq = l % 2 of row
    // y = (l % 16) / 2: four points, the z-1 / z / z+1 values carried in registers.
    const int h = lane >> 4, r16 = lane & 15, y = r16 >> 1, xq = r16 & 1, x0 = xq << 2;
    const int zb = h << 2;
    const int o0 = y * 8 + x0;  // the lane's first point in a z slice
    const int fo = (r16 >> 1) * 64 + (xq << 2);  // the lane's element of a y face (z = r16 / 2)
    float* ybuf = reinterpret_cast<float*>(smem_raw + (size_t)kWarps * R * (sizeof(Stage8<NP>) + 8)) +
                  warp * (NP * 2 * 64);  // y faces of the chunk being computed, [field][-y / +y][z * 8 + x]
    // faces of the chunk held in ring slot `st` (its metadata are written at issue time)
    auto load_faces = [&](const Stage8<NP>& st, Faces<NP>& f) {
        const int par = st.par;
        const int32_t fy = h == 0 ? st.nn[2] : st.nn[3], fz = h == 0 ? st.nn[4] : st.nn[5];
#pragma unroll
        for (int p = 0; p < NP; ++p) {
            const float* src = p == 0 ? (par ? fs.in[1][0] : fs.in[0][0]) : (par ? fs.in[1][NP - 1] : fs.in[0][NP - 1]);
            const float b = st.bk[p].x;
            const float4 bk = make_float4(b, b, b, b);
            f.zf[p] = fz >= 0 ? ldg_f4(src + (int64_t)fz * 512 + (h == 0 ? 448 : 0) + o0) : bk;
            f.yf[p] = fy >= 0 ? ldg_f4(src + (int64_t)fy * 512 + (h == 0 ? 56 : 0) + fo) : bk;
        }
    };
    int waited = 0, ws = 0;     // chunks [0, waited) have landed; ws = slot of chunk `waited`
    uint32_t wph = 0;           // phase parity of slot ws for chunk `waited`
    int q = (int)(a - lo);
    int sq = q;                 // slot of chunk q (q < R)
    Faces<NP> fc, fn;           // faces of the chunk being computed / of the next one
    load_faces(ring[sq], fn);
    for (int64_t i = a; i < b; ++i, ++q) {
        const int sp = sq == 0 ? R - 1 : sq - 1, sn = sq + 1 == R ? 0 : sq + 1;
        fc = fn;
        if (i + 1 < b) load_faces(ring[sn], fn);  // one chunk ahead; chunk q + 1's metadata are in slot sn
        const int need = i + 1 < hi ? q + 1 : q;
        bool ok = true;
        while (waited <= need) {
            if (!mbar_wait_bounded(&full[ws], wph, err)) {
                ok = false;
                break;
            }
            if (++ws == R) {
                ws = 0;
                wph ^= 1u;
            }
            ++waited;
        }
        if (!ok) {
            // let the copies already issued land before the warp retires
            for (int r = waited + 1; r < issued; ++r)
                mbar_wait_bounded(&full[r % R], (uint32_t)(r / R) & 1u, err, 100000000ull);
            return;
        }
        const Stage8<NP>& st = ring[sq];
        if (st.active) {
            // the y faces of this chunk to the warp's buffer, read below by the y = 0 / y = 7 lanes
#pragma unroll
            for (int p = 0; p < NP; ++p)
                *reinterpret_cast<float4*>(&ybuf[(p * 2 + h) * 64 + (r16 >> 1) * 8 + x0]) = fc.yf[p];
            __syncwarp();
            const Stage8<NP>& pv = ring[sp];
            const Stage8<NP>& nx = ring[sn];
            const int32_t n0 = st.nn[0], n1 = st.nn[1];
            // an absent neighbour is -1, which must not match position i - 1 of chunk 0
            const bool xm_ok = n0 >= 0 && n0 == (int32_t)(i - 1), xp_ok = n1 >= 0 && n1 == (int32_t)(i + 1);
            // (byte offsets into the dynamic shared array: plain loads through it stay shared-memory loads
            // and leave the scheduler free to batch them)
            auto off = [&](const void* ptr) { return (uint32_t)((const unsigned char*)ptr - smem_raw); };
            auto ld4 = [&](uint32_t o) { return *reinterpret_cast<const float4*>(smem_raw + o); };
            auto ld1 = [&](uint32_t o) { return *reinterpret_cast<const float*>(smem_raw + o); };
            // addresses at the lane's first z (zb) and their steps per z
            uint32_t aC[NP], aXm[NP], aXp[NP], aYm[NP], aYp[NP];
            float4 zmv[NP], cv[NP];
            const uint32_t sYm = y > 0 ? 256u : 32u, sYp = y < 7 ? 256u : 32u;
            const uint32_t sXm = (xq == 1 || xm_ok) ? 256u : 0u, sXp = (xq == 0 || xp_ok) ? 256u : 0u;
#pragma unroll
            for (int p = 0; p < NP; ++p) {
                const uint32_t bk = off(&st.bk[p]);
                aC[p] = off(&st.tile[p][zb * 64 + o0]);
                aYm[p] = y > 0 ? aC[p] - 32 : off(&ybuf[(p * 2 + 0) * 64 + zb * 8 + x0]);
                aYp[p] = y < 7 ? aC[p] + 32 : off(&ybuf[(p * 2 + 1) * 64 + zb * 8 + x0]);
                aXm[p] = xq == 1 ? aC[p] - 4 : (xm_ok ? off(&pv.tile[p][zb * 64 + y * 8 + 7]) : bk);
                aXp[p] = xq == 0 ? aC[p] + 16 : (xp_ok ? off(&nx.tile[p][zb * 64 + y * 8]) : bk);
                if (!(xq == 1 || xm_ok)) aXm[p] = bk;  // step 0 on the background
                if (!(xq == 0 || xp_ok)) aXp[p] = bk;
                // z - 1 of the first slice: the -z face for the lower half, slice 3 for the upper half
                zmv[p] = h == 0 ? fc.zf[p] : ld4(aC[p] - 256);
                cv[p] = ld4(aC[p]);
            }
            const uint32_t aM = off(&st.mt[zb * 64 + o0]);
            const int par = st.par;
            float* d0 = (par ? fs.out[1][0] : fs.out[0][0]) + i * 512 + zb * 64 + o0;
            float* d1 = (par ? fs.out[1][NP - 1] : fs.out[0][NP - 1]) + i * 512 + zb * 64 + o0;
            const GridInfo cgi = st.gi;
            const float bd0 = st.gi.bck[par ^ 1][0], bd1 = st.gi.bck[par ^ 1][NP - 1];  // destination backgrounds
            const int32_t bx = st.cx + x0, by = st.cy + y, bz = st.cz + zb;
#pragma unroll
            for (int zz = 0; zz < 4; ++zz) {
                const uint32_t m4 = *reinterpret_cast<const uint32_t*>(smem_raw + aM + zz * 64);
                float4 lap[NP], cur[NP];
#pragma unroll
                for (int p = 0; p < NP; ++p) {
                    // z + 1: the next slice, or for the upper half's last slice the +z face
                    float4 zp;
                    if (zz < 3) {
                        zp = ld4(aC[p] + (zz + 1) * 256);
                    } else {
                        const float4 t4 = ld4(h == 0 ? aC[p] + 4 * 256 : aC[p]);  // in-stage address for both halves
                        zp = h == 0 ? t4 : fc.zf[p];
                    }
                    const float4 ym = ld4(aYm[p] + zz * sYm);
                    const float4 yp = ld4(aYp[p] + zz * sYp);
                    const float xm = ld1(aXm[p] + zz * sXm);
                    const float xp = ld1(aXp[p] + zz * sXp);
                    const float4 c = cv[p], zm = zmv[p];
                    lap[p].x = lap7k<KIND>(c.x, xm, c.y, ym.x, yp.x, zm.x, zp.x);
                    lap[p].y = lap7k<KIND>(c.y, c.x, c.z, ym.y, yp.y, zm.y, zp.y);
                    lap[p].z = lap7k<KIND>(c.z, c.y, c.w, ym.z, yp.z, zm.z, zp.z);
                    lap[p].w = lap7k<KIND>(c.w, c.z, xp, ym.w, yp.w, zm.w, zp.w);
                    cur[p] = c;
                    zmv[p] = c;
                    cv[p] = zp;
                }
                const uint32_t mb[4] = {m4 & 0xffu, (m4 >> 8) & 0xffu, (m4 >> 16) & 0xffu, m4 >> 24};
                bool act[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    act[k] = (mb[k] & 3u) == 1u;  // EXIST and not PADDING
                    if (BOX) act[k] = act[k] && in_box(prm, bx + k, by, bz + zz);
                }
                if (KIND == SGB_HEAT7) {
                    float4 o;
                    o.x = act[0] ? __fmaf_rn(cgi.dt, lap[0].x, cur[0].x) : (mb[0] ? cur[0].x : bd0);
                    o.y = act[1] ? __fmaf_rn(cgi.dt, lap[0].y, cur[0].y) : (mb[1] ? cur[0].y : bd0);
                    o.z = act[2] ? __fmaf_rn(cgi.dt, lap[0].z, cur[0].z) : (mb[2] ? cur[0].z : bd0);
                    o.w = act[3] ? __fmaf_rn(cgi.dt, lap[0].w, cur[0].w) : (mb[3] ? cur[0].w : bd0);
                    *reinterpret_cast<float4*>(d0 + zz * 64) = o;
                } else {
                    float4 un, vn;
                    gs_update(cur[0].x, cur[NP - 1].x, lap[0].x, lap[NP - 1].x, cgi, un.x, vn.x);
                    gs_update(cur[0].y, cur[NP - 1].y, lap[0].y, lap[NP - 1].y, cgi, un.y, vn.y);
                    gs_update(cur[0].z, cur[NP - 1].z, lap[0].z, lap[NP - 1].z, cgi, un.z, vn.z);
                    gs_update(cur[0].w, cur[NP - 1].w, lap[0].w, lap[NP - 1].w, cgi, un.w, vn.w);
                    // Active points take the update.  Points that do not exist take the destination's
                    // background, which they hold already (the background invariant), so the quad is
                    // written whole with one vector store; only existing inactive points (padding,
                    // outside the box) keep their value, with scalar stores.
                    un.x = act[0] ? un.x : bd0;
                    un.y = act[1] ? un.y : bd0;
                    un.z = act[2] ? un.z : bd0;
                    un.w = act[3] ? un.w : bd0;
                    vn.x = act[0] ? vn.x : bd1;
                    vn.y = act[1] ? vn.y : bd1;
                    vn.z = act[2] ? vn.z : bd1;
                    vn.w = act[3] ? vn.w : bd1;
                    bool all = true;
#pragma unroll
                    for (int k = 0; k < 4; ++k) all = all && (act[k] || mb[k] == 0);
                    if (all) *reinterpret_cast<float4*>(d0 + zz * 64) = un;
                    if (all) *reinterpret_cast<float4*>(d1 + zz * 64) = vn;
                    if (__any_sync(0xffffffffu, !all)) {  // rare: padding or box edges in the quad
                        const float u4[4] = {un.x, un.y, un.z, un.w}, v4[4] = {vn.x, vn.y, vn.z, vn.w};
#pragma unroll
                        for (int k = 0; k < 4; ++k) {
                            if (!all && act[k]) d0[zz * 64 + k] = u4[k];
                            if (!all && act[k]) d1[zz * 64 + k] = v4[k];
                        }
                    }
                }
            }
        }
        __syncwarp();
        if (i > lo && issued < Q) {
            // chunk q - 1 is no longer read: its slot takes chunk q - 1 + R
            fence_proxy_async_smem();
            issue(issued, sp);
            ++issued;
        }
        sq = sn;
    }
}

template <int KIND, int NP, bool BOX>
static int launch_kind(const LaunchDesc& L, cudaStream_t s) {
    // ring depth per warp: at least 3 (chunks q - 1, q, q + 1), within one CTA's shared memory; 0 = the
    // deepest ring (up to 8) with which the requested CTAs per SM stay resident
    const size_t per = sizeof(Stage8<NP>) + 8;
    const size_t yface_bytes = NP * 2 * 64 * sizeof(float);  // per warp
    const int rmax = (int)((227u * 1024u - kWarps * yface_bytes) / (per * kWarps));
    int R = L.stages;
    if (R <= 0) {
        const int64_t per_sm = std::max<int64_t>(1, ((int64_t)L.ctas + L.num_sms - 1) / L.num_sms);
        const int64_t budget = 228 * 1024 / per_sm - 1024;  // 1 KB of every CTA's shared memory is reserved
        R = (int)std::max<int64_t>(3, std::min<int64_t>(8, (budget - (int64_t)(kWarps * yface_bytes)) /
                                                               (int64_t)(per * kWarps)));
    }
    R = std::min(std::max(R, 3), rmax);
    const size_t smem = (size_t)kWarps * (R * per + yface_bytes);
    // warps: CTAs per SM x SMs x kWarps, at most one per chunk (a small grid is latency-bound: one chunk per
    // warp, whose two neighbour chunks are L2 hits, beats a few warps walking several chunks each)
    const int64_t total = (int64_t)L.ctas * kWarps;
    const int64_t nwarps = std::max<int64_t>(1, std::min<int64_t>(total, L.n));
    const unsigned blocks = (unsigned)((nwarps + kWarps - 1) / kWarps);
    auto kern = k_stencil7_e8<KIND, NP, BOX>;
    SGB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    // consecutive steps overlap one launch's ramp-up with the previous one's tail
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(blocks);
    cfg.blockDim = dim3(kThreads8);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    SGB_CUDA(cudaLaunchKernelEx(&cfg, kern, L.fs, L.mask, L.nn, L.keys, L.gid, L.grids, L.g0, L.n, L.geo, L.prm, L.t, R,
                                nwarps, L.err));
    return SGB_OK;
}

int launch_e8(const LaunchDesc& L, cudaStream_t s) {
    const bool box = L.prm.has_box != 0;
    if (L.kind == SGB_GS7) return box ? launch_kind<SGB_GS7, 2, true>(L, s) : launch_kind<SGB_GS7, 2, false>(L, s);
    return box ? launch_kind<SGB_HEAT7, 1, true>(L, s) : launch_kind<SGB_HEAT7, 1, false>(L, s);
}

}  // namespace sgb
