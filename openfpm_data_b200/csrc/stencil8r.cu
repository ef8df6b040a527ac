// Row-sparse pipelined 7-point stencil for one grid of 8^3 chunks (HEAT7,
// GS7, the whole domain): the kernel of applyStencils / sgb_run_steps on a
// single grid.  The batched form and box-limited applications run
// k_stencil7_e8 (stencil8.cu), which this kernel follows in structure.
//
// Reference path: applyStencilInPlace (src/SparseGridGpu/SparseGridGpu.hpp:
// 954-1048) runs one 512-thread CTA per chunk; loadGhostBlock_impl<1>
// (src/SparseGridGpu/SparseGridGpu_ker_util.hpp:487-564) gathers the 10^3
// tile point by point, substituting the background where a mask byte is 0.
//
// Work split: every warp is an independent pipeline over a contiguous range
// [a, b) of chunk positions, streaming [a - 1, b + 1) through its own R-stage
// shared-memory ring.  The -x / +x neighbour of a chunk, when it exists, is
// the previous / next index position, so the x halo is read from the
// neighbouring ring stages; the y and z faces are loaded into registers one
// chunk ahead (the y faces then pass through a 1 KB per-warp buffer).
//
// Traffic: per chunk the warp reads two 64-byte bitmaps (the EXIST points and
// the active points, EXIST and not PADDING, built by neighbours.cu) instead of
// the 512 mask bytes, and fetches a field tile as sixteen 128-byte segments
// (four rows of one z slice): one bulk copy (cp.async.bulk, the TMA engine)
// per segment that holds an existing point, issued by the segment's lane;
// segments without existing points are filled with the background in shared
// memory instead.  Results are written row by row (32 bytes, one sector),
// only for rows that hold an existing point: the other points of the
// destination already hold its background (the library keeps that invariant,
// sgb_grid::clean).  On the 512^3 Gray-Scott benchmark grid this moves ~130 MB
// per step instead of the 165 MB of whole chunks (114 MB algorithmic).
//
// Arithmetic: lanes 0-15 take z = 0..3 and lanes 16-31 z = 4..7; in each z
// slice a lane owns four x-adjacent points of one y row and marches z with
// z-1 / z / z+1 in registers.  The updates run on x-adjacent point pairs with
// the sm_100 packed FP32 instructions (add / sub / mul / fma .f32x2, flush to
// zero), in the association order of stencil.cuh: bit-identical results.
#include <algorithm>
#include <cstring>

#include "common.cuh"
#include "internal.h"
#include "stencil.cuh"

namespace sgb {

constexpr int kRWarps = 2;  // warps per CTA, each its own pipeline
constexpr int kRThreads = kRWarps * 32;

// One ring stage.  Its size is a multiple of 16 bytes (bulk copies and 16-byte loads need 16-byte
// aligned destinations), not of 128: every byte counts for the ring depth.
template <int NP>
struct alignas(16) StageR {
    float tile[NP][512];
    uint64_t ebits[8];  // EXIST bit of point (x, y) of z slice z: word z, bit 8 y + x
    uint64_t abits[8];  // the same for active points (EXIST and not PADDING)
    int32_t nn[8];      // NNStar row: -x, +x, -y, +y, -z, +z positions (-1 absent)
};
static_assert(sizeof(StageR<1>) % 16 == 0 && sizeof(StageR<2>) % 16 == 0, "stage size");

struct RowsArgs {
    const float* in0;
    const float* in1;
    float* out0;
    float* out1;
    const uint64_t* ebits;
    const uint64_t* abits;
    const int32_t* nn;
    int64_t n;
    int64_t nwarps;
    int R;
    float bin0, bin1;    // backgrounds of the source fields
    float bout0, bout1;  // backgrounds of the destination fields
    float dt, Du, Dv, F, nFK;
    unsigned* err;
};

// ---------------------------------------------------------------- packed FP32 pairs
__device__ __forceinline__ float2 add2(float2 a, float2 b) {
    float2 r;
    asm("{\n\t.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "add.rn.ftz.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(r.x), "=f"(r.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return r;
}
__device__ __forceinline__ float2 sub2(float2 a, float2 b) {
    float2 r;
    asm("{\n\t.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "sub.rn.ftz.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(r.x), "=f"(r.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return r;
}
__device__ __forceinline__ float2 mul2(float2 a, float2 b) {
    float2 r;
    asm("{\n\t.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "mul.rn.ftz.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(r.x), "=f"(r.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return r;
}
// a * b + c, one rounding
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) {
    float2 r;
    asm("{\n\t.reg .b64 ra, rb, rc, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "mov.b64 rc, {%6, %7};\n\tfma.rn.ftz.f32x2 rd, ra, rb, rc;\n\tmov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(r.x), "=f"(r.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
    return r;
}
__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 splat2(float a) { return make_float2(a, a); }

// lap7 (stencil.cuh) on two points: (-6 c) + (xm + xp) + (ym + yp) + (zm + zp).  -6 c is formed as
// fma(c, -4, (-2 c)): -2 c is exact, so the fma rounds -6 c once, as the multiply does, and no
// product feeds a separate add that an assembler could contract into a different rounding.
__device__ __forceinline__ float2 lap2(float2 c, float2 xm, float2 xp, float2 ym, float2 yp, float2 zm, float2 zp) {
    float2 m = fma2(c, splat2(-4.0f), mul2(c, splat2(-2.0f)));
    m = add2(m, add2(xm, xp));
    m = add2(m, add2(ym, yp));
    return add2(m, add2(zm, zp));
}

// lap7_heat (stencil.cuh) on two points: fma(-6, c, xm + xp) + (ym + yp) + (zm + zp)
__device__ __forceinline__ float2 lap2_heat(float2 c, float2 xm, float2 xp, float2 ym, float2 yp, float2 zm,
                                            float2 zp) {
    float2 m = fma2(c, splat2(-6.0f), add2(xm, xp));
    m = add2(m, add2(ym, yp));
    return add2(m, add2(zm, zp));
}

template <int KIND>
__device__ __forceinline__ float2 lap2k(float2 c, float2 xm, float2 xp, float2 ym, float2 yp, float2 zm, float2 zp) {
    return KIND == SGB_HEAT7 ? lap2_heat(c, xm, xp, ym, yp, zm, zp) : lap2(c, xm, xp, ym, yp, zm, zp);
}

// gs_update (stencil.cuh) on two points
__device__ __forceinline__ void gs2(float2 u, float2 v, float2 lu, float2 lv, const RowsArgs& A, float2& un,
                                    float2& vn) {
    const float2 uvv = mul2(mul2(u, v), v);
    const float2 nuvv = mul2(uvv, splat2(-1.0f));  // exactly -uvv
    float2 du = fma2(splat2(A.Du), lu, nuvv);
    du = fma2(splat2(A.F), sub2(splat2(1.0f), u), du);
    float2 dv = fma2(splat2(A.Dv), lv, uvv);
    dv = fma2(splat2(A.nFK), v, dv);
    un = fma2(splat2(A.dt), du, u);
    vn = fma2(splat2(A.dt), dv, v);
}

__device__ __forceinline__ float4 ldg4(const float* p) { return __ldg(reinterpret_cast<const float4*>(p)); }

template <int KIND, int NP>
__global__ void __launch_bounds__(kRThreads, 6) k_stencil7_rows(RowsArgs A) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    // programmatic dependent launch: the next step may be scheduled while this one drains; no field is
    // read or written before the previous launch on the stream has completed
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int R = A.R;
    StageR<NP>* ring = reinterpret_cast<StageR<NP>*>(smem_raw) + (size_t)warp * R;
    uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + (size_t)kRWarps * R * sizeof(StageR<NP>)) + warp * R;
    float* ybuf = reinterpret_cast<float*>(smem_raw + (size_t)kRWarps * R * (sizeof(StageR<NP>) + 8)) +
                  warp * (NP * 2 * 64);  // y faces of the chunk being computed, [field][-y / +y][z * 8 + x]
    const int64_t gw = (int64_t)blockIdx.x * kRWarps + warp;
    if (gw >= A.nwarps) return;
    const int64_t n = A.n;
    const int64_t a = n * gw / A.nwarps, b = n * (gw + 1) / A.nwarps;
    if (a >= b) return;
    const int64_t lo = a > 0 ? a - 1 : 0, hi = b < n ? b + 1 : n;
    const int Q = (int)(hi - lo);
    if (lane == 0) {
        for (int r = 0; r < R; ++r) mbar_init(&full[r], 1);  // the issuing lane's expect_tx arrival
        mbar_fence_init();
    }
    __syncwarp();

    // ------------------------------------------------------------ issue side
    // neighbour rows (8 ints per chunk) in windows of 8 chunks, one window ahead: lane l holds entries
    // l and l + 32 of a window
    const int64_t nnend = hi * 8;
    auto load_win = [&](int64_t first, int32_t& wa, int32_t& wb) {
        const int64_t e = first * 8 + lane;
        wa = e < nnend ? A.nn[e] : -1;
        wb = e + 32 < nnend ? A.nn[e + 32] : -1;
    };
    // bitmaps in windows of 2 chunks, one window ahead: lane l holds word l & 7 of the EXIST (l & 8 == 0)
    // or active bitmap of chunk first + (l >> 4)
    auto load_bw = [&](int64_t first) -> uint64_t {
        const int64_t c = first + (lane >> 4);
        if (c >= hi) return 0;
        return __ldg(((lane & 8) ? A.abits : A.ebits) + c * 8 + (lane & 7));
    };
    int32_t w0, w1, x0v, x1v;
    load_win(lo, w0, w1);
    load_win(lo + 8, x0v, x1v);
    uint64_t bw = load_bw(lo), bwn = load_bw(lo + 2);
    const int f = lane >> 4, sgm = lane & 15;  // the lane's field and 128-byte segment (z = sgm / 2)
    const bool has_field = f < NP;
    const float* fsrc = (f == 0 ? A.in0 : A.in1) + sgm * 32;
    const float fbck = f == 0 ? A.bin0 : A.bin1;
    // Fill ring slot `slot` with chunk lo + q; q increases by one per call.
    auto issue = [&](int q, int slot) {
        const int64_t c = lo + q;
        const int j = q & 7;
        if (j == 0 && q > 0) {
            w0 = x0v;
            w1 = x1v;
            load_win(c + 8, x0v, x1v);
        }
        const int jb = q & 1;
        if (jb == 0 && q > 0) {
            bw = bwn;
            bwn = load_bw(c + 2);
        }
        const int32_t wsel = j < 4 ? w0 : w1;
        const int32_t nb_cur = __shfl_sync(0xffffffffu, wsel, ((j & 3) << 3) + (lane & 7));
        const uint64_t ew = __shfl_sync(0xffffffffu, bw, 16 * jb + (sgm >> 1));
        StageR<NP>& st = ring[slot];
        uint64_t* bar = &full[slot];
        if (lane < 8) st.nn[lane] = nb_cur;
        if ((lane >> 4) == jb) {
            if (lane & 8) st.abits[lane & 7] = bw;
            else st.ebits[lane & 7] = bw;
        }
        const uint32_t rows = (sgm & 1) ? (uint32_t)(ew >> 32) : (uint32_t)ew;
        const bool live = has_field && rows != 0u;
        const unsigned liveb = __ballot_sync(0xffffffffu, live);
        if (lane == 0) mbar_arrive_expect_tx(bar, (uint32_t)__popc(liveb) * 128u);
        __syncwarp();
        float* dst = &st.tile[has_field ? f : 0][sgm * 32];
        if (live) {
            bulk_g2s(dst, fsrc + c * 512, 128, bar);
        } else if (has_field) {  // no existing point in these four rows: their values are the background
            const float4 bk = make_float4(fbck, fbck, fbck, fbck);
#pragma unroll
            for (int k = 0; k < 8; ++k) reinterpret_cast<float4*>(dst)[k] = bk;
        }
        __syncwarp();
    };

    const int npro = Q < R ? Q : R;
    for (int q = 0; q < npro; ++q) issue(q, q);
    int issued = npro;

    // ------------------------------------------------------------ compute side
    // Lane l takes z = 4h .. 4h + 3 with h = l / 16 and, in each z slice, the x quad xq = l % 2 of row
    // y = (l % 16) / 2.
    const int h = lane >> 4, r16 = lane & 15, y = r16 >> 1, xq = r16 & 1, x0 = xq << 2;
    const int zb = h << 2;
    const int o0 = y * 8 + x0;                    // the lane's first point in a z slice
    const int fo = (r16 >> 1) * 64 + (xq << 2);  // the lane's element of a y face (z = r16 / 2)
    // z face (the lane's quad of slice 7 of the -z chunk, or of slice 0 of the +z chunk) and y face
    // element of the chunk in ring slot `st`, per field
    const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
    float4 zf0 = z4, yf0 = z4, zf1 = z4, yf1 = z4, nzf0 = z4, nyf0 = z4, nzf1 = z4, nyf1 = z4;
    auto load_faces = [&](const StageR<NP>& st, float4& zf_0, float4& yf_0, float4& zf_1, float4& yf_1) {
        const int32_t fy = h == 0 ? st.nn[2] : st.nn[3], fz = h == 0 ? st.nn[4] : st.nn[5];
        const int zo = (h == 0 ? 448 : 0) + o0, yo = (h == 0 ? 56 : 0) + fo;
        const float4 b0 = make_float4(A.bin0, A.bin0, A.bin0, A.bin0);
        zf_0 = fz >= 0 ? ldg4(A.in0 + (int64_t)fz * 512 + zo) : b0;
        yf_0 = fy >= 0 ? ldg4(A.in0 + (int64_t)fy * 512 + yo) : b0;
        if (NP == 2) {
            const float4 b1 = make_float4(A.bin1, A.bin1, A.bin1, A.bin1);
            zf_1 = fz >= 0 ? ldg4(A.in1 + (int64_t)fz * 512 + zo) : b1;
            yf_1 = fy >= 0 ? ldg4(A.in1 + (int64_t)fy * 512 + yo) : b1;
        }
    };
    int waited = 0, ws = 0;  // chunks [0, waited) have landed; ws = slot of chunk `waited`
    uint32_t wph = 0;        // phase parity of slot ws for chunk `waited`
    int q = (int)(a - lo);
    int sq = q;  // slot of chunk q (q < R)
    load_faces(ring[sq], nzf0, nyf0, nzf1, nyf1);
    for (int64_t i = a; i < b; ++i, ++q) {
        const int sp = sq == 0 ? R - 1 : sq - 1, sn = sq + 1 == R ? 0 : sq + 1;
        zf0 = nzf0, yf0 = nyf0, zf1 = nzf1, yf1 = nyf1;
        if (i + 1 < b) load_faces(ring[sn], nzf0, nyf0, nzf1, nyf1);  // one chunk ahead
        const int need = i + 1 < hi ? q + 1 : q;
        bool ok = true;
        while (waited <= need) {
            if (!mbar_wait_bounded(&full[ws], wph, A.err)) {
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
                mbar_wait_bounded(&full[r % R], (uint32_t)(r / R) & 1u, A.err, 100000000ull);
            return;
        }
        const StageR<NP>& st = ring[sq];
        // the y faces of this chunk to the warp's buffer, read below by the y = 0 / y = 7 lanes
        *reinterpret_cast<float4*>(&ybuf[(0 * 2 + h) * 64 + (r16 >> 1) * 8 + x0]) = yf0;
        if (NP == 2) *reinterpret_cast<float4*>(&ybuf[(1 * 2 + h) * 64 + (r16 >> 1) * 8 + x0]) = yf1;
        __syncwarp();
        const StageR<NP>& pv = ring[sp];
        const StageR<NP>& nx = ring[sn];
        const int32_t n0 = st.nn[0], n1 = st.nn[1];
        // an absent neighbour is -1, which must not match position i - 1 of chunk 0
        const bool xm_ok = n0 >= 0 && n0 == (int32_t)(i - 1), xp_ok = n1 >= 0 && n1 == (int32_t)(i + 1);
        auto off = [&](const void* ptr) { return (uint32_t)((const unsigned char*)ptr - smem_raw); };
        auto ld4 = [&](uint32_t o) { return *reinterpret_cast<const float4*>(smem_raw + o); };
        auto ld1 = [&](uint32_t o) { return *reinterpret_cast<const float*>(smem_raw + o); };
        // shared-memory addresses at the lane's first z (zb) and their steps per z, per field
        uint32_t aC[NP], aXm[NP], aXp[NP], aYm[NP], aYp[NP];
        float4 zmv[NP], cv[NP];
        const uint32_t sYm = y > 0 ? 256u : 32u, sYp = y < 7 ? 256u : 32u;
        const uint32_t sXm = (xq == 1 || xm_ok) ? 256u : 0u, sXp = (xq == 0 || xp_ok) ? 256u : 0u;
        const float4 zfa[2] = {zf0, zf1};
#pragma unroll
        for (int p = 0; p < NP; ++p) {
            aC[p] = off(&st.tile[p][zb * 64 + o0]);
            aYm[p] = y > 0 ? aC[p] - 32 : off(&ybuf[(p * 2 + 0) * 64 + zb * 8 + x0]);
            aYp[p] = y < 7 ? aC[p] + 32 : off(&ybuf[(p * 2 + 1) * 64 + zb * 8 + x0]);
            aXm[p] = xq == 1 ? aC[p] - 4 : off(&pv.tile[p][zb * 64 + y * 8 + 7]);
            aXp[p] = xq == 0 ? aC[p] + 16 : off(&nx.tile[p][zb * 64 + y * 8]);
            zmv[p] = h == 0 ? zfa[p] : ld4(aC[p] - 256);
            cv[p] = ld4(aC[p]);
        }
        // an absent x neighbour chunk: the halo value is the source background
        const bool xm_bk = !(xq == 1 || xm_ok), xp_bk = !(xq == 0 || xp_ok);
        float* d0 = A.out0 + i * 512 + zb * 64 + o0;
        float* d1 = A.out1 + i * 512 + zb * 64 + o0;
#pragma unroll
        for (int zz = 0; zz < 4; ++zz) {
            const int z = zb + zz;
            const uint32_t e8 = (uint32_t)(st.ebits[z] >> (8 * y)) & 0xffu;
            const uint32_t a8 = (uint32_t)(st.abits[z] >> (8 * y)) & 0xffu;
            float2 nA[NP], nB[NP], cA[NP], cB[NP];
#pragma unroll
            for (int p = 0; p < NP; ++p) {
                // z + 1: the next slice, or for the upper half's last slice the +z face
                float4 zp;
                if (zz < 3) {
                    zp = ld4(aC[p] + (zz + 1) * 256);
                } else {
                    const float4 t4 = ld4(h == 0 ? aC[p] + 4 * 256 : aC[p]);  // in-stage address for both halves
                    zp = h == 0 ? t4 : zfa[p];
                }
                const float4 ym = ld4(aYm[p] + zz * sYm);
                const float4 yp = ld4(aYp[p] + zz * sYp);
                const float bk = p == 0 ? A.bin0 : A.bin1;
                const float xm = xm_bk ? bk : ld1(aXm[p] + zz * sXm);
                const float xp = xp_bk ? bk : ld1(aXp[p] + zz * sXp);
                const float4 c = cv[p], zm = zmv[p];
                cA[p] = f2(c.x, c.y);
                cB[p] = f2(c.z, c.w);
                nA[p] = lap2k<KIND>(cA[p], f2(xm, c.x), f2(c.y, c.z), f2(ym.x, ym.y), f2(yp.x, yp.y), f2(zm.x, zm.y),
                             f2(zp.x, zp.y));
                nB[p] = lap2k<KIND>(cB[p], f2(c.y, c.z), f2(c.w, xp), f2(ym.z, ym.w), f2(yp.z, yp.w), f2(zm.z, zm.w),
                             f2(zp.z, zp.w));
                zmv[p] = c;
                cv[p] = zp;
            }
            if (e8 == 0u) continue;  // no existing point in the row: the destination holds its background
            const uint32_t e4 = (e8 >> x0) & 0xfu, a4 = (a8 >> x0) & 0xfu;
            if (KIND == SGB_HEAT7) {
                // HeatStencil's storeBlock writes the whole row: active points the update, other existing
                // points their own value, points that do not exist the destination's background
                const float2 uA = fma2(splat2(A.dt), nA[0], cA[0]), uB = fma2(splat2(A.dt), nB[0], cB[0]);
                float4 o;
                o.x = (a4 & 1u) ? uA.x : ((e4 & 1u) ? cA[0].x : A.bout0);
                o.y = (a4 & 2u) ? uA.y : ((e4 & 2u) ? cA[0].y : A.bout0);
                o.z = (a4 & 4u) ? uB.x : ((e4 & 4u) ? cB[0].x : A.bout0);
                o.w = (a4 & 8u) ? uB.y : ((e4 & 8u) ? cB[0].y : A.bout0);
                *reinterpret_cast<float4*>(d0 + zz * 64) = o;
            } else {
                float2 uA, vA, uB, vB;
                gs2(cA[0], cA[NP - 1], nA[0], nA[NP - 1], A, uA, vA);
                gs2(cB[0], cB[NP - 1], nB[0], nB[NP - 1], A, uB, vB);
                float4 un = make_float4(uA.x, uA.y, uB.x, uB.y), vn = make_float4(vA.x, vA.y, vB.x, vB.y);
                if (a8 == e8) {
                    // no padding in the row: the whole row is written; points that do not exist take the
                    // destination's background, which they hold already
                    un.x = (a4 & 1u) ? un.x : A.bout0;
                    un.y = (a4 & 2u) ? un.y : A.bout0;
                    un.z = (a4 & 4u) ? un.z : A.bout0;
                    un.w = (a4 & 8u) ? un.w : A.bout0;
                    vn.x = (a4 & 1u) ? vn.x : A.bout1;
                    vn.y = (a4 & 2u) ? vn.y : A.bout1;
                    vn.z = (a4 & 4u) ? vn.z : A.bout1;
                    vn.w = (a4 & 8u) ? vn.w : A.bout1;
                    *reinterpret_cast<float4*>(d0 + zz * 64) = un;
                    *reinterpret_cast<float4*>(d1 + zz * 64) = vn;
                } else {  // padding points keep their value: only the active points are stored
                    const float u4[4] = {un.x, un.y, un.z, un.w}, v4[4] = {vn.x, vn.y, vn.z, vn.w};
#pragma unroll
                    for (int k = 0; k < 4; ++k)
                        if (a4 & (1u << k)) {
                            d0[zz * 64 + k] = u4[k];
                            d1[zz * 64 + k] = v4[k];
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

template <int KIND, int NP>
static int launch_rows_kind(const LaunchDesc& L, cudaStream_t s) {
    const size_t per = sizeof(StageR<NP>) + 8;
    const size_t yface_bytes = NP * 2 * 64 * sizeof(float);  // per warp
    const int rmax = (int)((227u * 1024u - kRWarps * yface_bytes) / (per * kRWarps));
    int R = L.stages;
    if (R <= 0) {
        const int64_t per_sm = std::max<int64_t>(1, ((int64_t)L.ctas + L.num_sms - 1) / L.num_sms);
        const int64_t budget = 228 * 1024 / per_sm - 1024;  // 1 KB of every CTA's shared memory is reserved
        R = (int)std::max<int64_t>(3, std::min<int64_t>(8, (budget - (int64_t)(kRWarps * yface_bytes)) /
                                                               (int64_t)(per * kRWarps)));
    }
    R = std::min(std::max(R, 3), rmax);
    const size_t smem = (size_t)kRWarps * (R * per + yface_bytes);
    const int64_t total = (int64_t)L.ctas * kRWarps;
    const int64_t nwarps = std::max<int64_t>(1, std::min<int64_t>(total, L.n));
    const unsigned blocks = (unsigned)((nwarps + kRWarps - 1) / kRWarps);
    RowsArgs A;
    A.in0 = L.fs.in[0][0];
    A.in1 = L.fs.in[0][NP - 1];
    A.out0 = L.fs.out[0][0];
    A.out1 = L.fs.out[0][NP - 1];
    A.ebits = L.ebits;
    A.abits = L.abits;
    A.nn = L.nn;
    A.n = L.n;
    A.nwarps = nwarps;
    A.R = R;
    A.bin0 = L.g0.bck[0][0];
    A.bin1 = L.g0.bck[0][NP - 1];
    A.bout0 = L.g0.bck[1][0];
    A.bout1 = L.g0.bck[1][NP - 1];
    A.dt = L.g0.dt;
    A.Du = L.g0.Du;
    A.Dv = L.g0.Dv;
    A.F = L.g0.F;
    A.nFK = L.g0.nFK;
    A.err = L.err;
    auto kern = k_stencil7_rows<KIND, NP>;
    SGB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(blocks);
    cfg.blockDim = dim3(kRThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    SGB_CUDA(cudaLaunchKernelEx(&cfg, kern, A));
    return SGB_OK;
}

int launch_rows(const LaunchDesc& L, cudaStream_t s) {
    if (L.kind == SGB_GS7) return launch_rows_kind<SGB_GS7, 2>(L, s);
    return launch_rows_kind<SGB_HEAT7, 1>(L, s);
}

}  // namespace sgb
