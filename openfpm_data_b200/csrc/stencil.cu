// Fixed-function stencils over the block map: HEAT7, GS7 and BOX27.
//
// Reference path: applyStencils -> applyStencilInPlace
// (src/SparseGridGpu/SparseGridGpu.hpp:954-1048) -> one 512-thread CTA per
// chunk, loadGhostBlock_impl<1> (SparseGridGpu_ker_util.hpp:487-564) gathers
// the 10^3 tile with one scalar load per point, the user functor computes,
// storeBlock writes back.
//
// Here 7-point stencils on 8^3 chunks run the pipelined kernel of
// stencil8.cu; this file holds the generic one-chunk-per-CTA tile kernel
// (BOX27, 4^3 chunks, cross-checks), parameter handling and dispatch.
//
// The same kernels run a batch of grids concatenated into one block map: a
// per-chunk grid id selects the grid's parameters and its ping-pong buffer
// for global step t (GridInfo); a single grid is a batch of one.
//
// Semantics kept from the reference: a halo or centre value whose mask byte
// is 0 reads the background value; active = EXIST && !PADDING && inside the
// inclusive box; HEAT7 writes every point of the destination chunk (active
// points the update, the others the tile value, as storeBlock does; a point
// whose mask byte is 0 gets the destination's background, which no read can
// tell from the reference's copy of the source background), GS7 and BOX27
// write active points only.  Ping-pong steps take each buffer's own
// background (GridInfo::bck).  Arithmetic follows the reference's FP32
// association with nvcc's FMA contraction and flush-to-zero (-use_fast_math,
// src/CMakeLists.txt:158), written with explicit intrinsics so the compiler
// cannot re-associate it.
#include <algorithm>
#include <cstring>

#include "common.cuh"
#include "internal.h"
#include "stencil.cuh"

namespace sgb {

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
        // selects, not a dynamic index into the parameter struct (which would copy it to local memory)
        const float* src[2] = {par ? fs.in[1][0] : fs.in[0][0], par ? fs.in[1][NP - 1] : fs.in[0][NP - 1]};
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
            for (int p = 0; p < NP; ++p) tile[p][cell] = ex ? src[p][idx] : (par ? gi.bck[1][p] : gi.bck[0][p]);
        }
        __syncthreads();
        int64_t cx = 0, cy = 0, cz = 0;
        if (prm.has_box) {
            int64_t o[3];
            chunk_origin(geo, keys[chunk], o);
            cx = o[0];
            cy = o[1];
            cz = o[2];
        }
        float* d0 = par ? fs.out[1][0] : fs.out[0][0];
        float* d1 = par ? fs.out[1][NP - 1] : fs.out[0][NP - 1];
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
                               : (m ? cur : (par ? gi.bck[0][0] : gi.bck[1][0]));
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

// ------------------------------------------------------------------ Conv3x3x3 on 8^3 chunks
// One warp per chunk at a time (grid-stride over chunks, four independent warps per CTA, no CTA
// barriers), software-pipelined: while chunk i is computed from one 10^3 shared tile, cp.async
// copies fill the warp's other tile with chunk i + 1 (16-byte copies of the chunk's rows, of the z
// and y faces and of the four edges along x; 4-byte copies of the x faces, the other eight edges
// and the corners, from the 26 NNFull neighbours; an absent neighbour's cells get the background
// with plain stores) and its mask bytes.  Tile cell (x, y, z), x, y, z in 0..9, sits at
// z * 120 + y * 12 + x + 3: rows of 12 floats put the chunk's part of every row on a 16-byte
// boundary and spread eight consecutive rows over all 32 banks.
// Lane l owns the x quad q = l % 2 (chunk x = 4q .. 4q + 3) of row y (lanes 0..7 of each half
// take the even rows, 8..15 the odd ones, so the 16-byte row loads of a quarter warp hit
// distinct banks) and the z half l / 16 (z = 0..3 or 4..7).  It marches z holding a 3 x 3 x 6
// window in registers (each row: one 16-byte load, the halo cell, and the partner quad's edge
// cell by a shuffle) and runs the 27 FMAs of each of its four points in Conv3x3x3's order (x
// offset outermost, z innermost), four independent chains.  Results equal the tile kernel's bit
// for bit (the background invariant makes a stored non-existing point read the same as the
// substituted background).
constexpr int kW27Row = 12, kW27Plane = 120, kW27Tile = 1204, kW27Warps = 4;

struct W27Stage {
    float tile[2][kW27Tile];
    uint8_t mt[2][512];
};

// Fill one tile with chunk c (warp-wide; lane l < 27 holds NNFull slot l of chunk c in nbr).
__device__ __noinline__ void w27_fill(float* T, uint8_t* mt, int32_t nbr, const float* __restrict__ src,
                                         const uint8_t* __restrict__ mask, int64_t c, float bck, int l) {
    constexpr unsigned kAll = 0xffffffffu;
    cp_async16(mt + l * 16, mask + c * 512 + l * 16);
    // the chunk's rows: 128 pieces of 16 bytes, piece p = (x half, y, z)
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int p = l + 32 * k, h = p & 1, y = (p >> 1) & 7, z = p >> 4;
        cp_async16(T + (z + 1) * kW27Plane + (y + 1) * kW27Row + 4 + 4 * h, src + c * 512 + p * 4);
    }
    auto piece = [&](float* d, int32_t nb, int off) {
        if (nb >= 0) cp_async16(d, src + (int64_t)nb * 512 + off);
        else *reinterpret_cast<float4*>(d) = make_float4(bck, bck, bck, bck);
    };
    auto cell = [&](float* d, int32_t nb, int off) {
        if (nb >= 0) cp_async4(d, src + (int64_t)nb * 512 + off);
        else *d = bck;
    };
    // z faces and y faces: lanes 0..15 the lower side, 16..31 the upper, one 16-byte piece each
    {
        const int f = l >> 4, h = l & 1, a = (l >> 1) & 7;
        const int32_t nz = __shfl_sync(kAll, nbr, f ? 22 : 4);
        const int32_t ny = __shfl_sync(kAll, nbr, f ? 16 : 10);
        piece(T + (f ? 9 : 0) * kW27Plane + (a + 1) * kW27Row + 4 + 4 * h, nz, (f ? 0 : 7) * 64 + a * 8 + 4 * h);
        piece(T + (a + 1) * kW27Plane + (f ? 9 : 0) * kW27Row + 4 + 4 * h, ny, a * 64 + (f ? 0 : 7) * 8 + 4 * h);
    }
    // x faces: 128 cells, four per lane; odd lanes take the upper face so that one copy
    // instruction writes two bank residues
    {
        const int f = l & 1;
        const int32_t nx = __shfl_sync(kAll, nbr, f ? 14 : 12);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int e = (l >> 1) + 16 * k, y = e & 7, z = e >> 3;
            cell(T + (z + 1) * kW27Plane + (y + 1) * kW27Row + (f ? 12 : 3), nx, z * 64 + y * 8 + (f ? 0 : 7));
        }
    }
    // edges along y (k = 0) and along z (k = 1): x side s & 1, other side s >> 1, position w
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const int w = l & 7, s = l >> 3, sx = s & 1, so = s >> 1;
        const int lx = sx ? 0 : 7, lo = so ? 0 : 7;
        int slot, ty, tz, off;
        if (k == 0) {
            slot = (sx ? 2 : 0) + 3 + 9 * (so ? 2 : 0);
            ty = w + 1;
            tz = so ? 9 : 0;
            off = lo * 64 + w * 8 + lx;
        } else {
            slot = (sx ? 2 : 0) + 3 * (so ? 2 : 0) + 9;
            ty = so ? 9 : 0;
            tz = w + 1;
            off = w * 64 + lo * 8 + lx;
        }
        const int32_t nb = __shfl_sync(kAll, nbr, slot);
        cell(T + tz * kW27Plane + ty * kW27Row + (sx ? 12 : 3), nb, off);
    }
    // edges along x (lanes 0..7, two 16-byte pieces each) and the corners (lanes 8..15)
    {
        const int k = (l >> 1) & 3, h = l & 1, sy = k & 1, sz = k >> 1;
        const int32_t ne = __shfl_sync(kAll, nbr, 1 + 3 * (sy ? 2 : 0) + 9 * (sz ? 2 : 0));
        const int r = l & 7, rx = r & 1, ry = (r >> 1) & 1, rz = r >> 2;
        const int32_t nc = __shfl_sync(kAll, nbr, (rx ? 2 : 0) + 3 * (ry ? 2 : 0) + 9 * (rz ? 2 : 0));
        if (l < 8)
            piece(T + (sz ? 9 : 0) * kW27Plane + (sy ? 9 : 0) * kW27Row + 4 + 4 * h, ne,
                  (sz ? 0 : 7) * 64 + (sy ? 0 : 7) * 8 + 4 * h);
        else if (l < 16)
            cell(T + (rz ? 9 : 0) * kW27Plane + (ry ? 9 : 0) * kW27Row + (rx ? 12 : 3), nc,
                 (rz ? 0 : 7) * 64 + (ry ? 0 : 7) * 8 + (rx ? 0 : 7));
    }
}

__global__ void __launch_bounds__(32 * kW27Warps, 4) k_box27_e8(const float* __restrict__ src, float* __restrict__ dst,
                                                              const uint8_t* __restrict__ mask,
                                                              const int32_t* __restrict__ nn,
                                                              const int64_t* __restrict__ keys, int64_t n,
                                                              Geometry geo, StencilParams prm, float bck) {
    __shared__ __align__(16) W27Stage stage[kW27Warps];
    constexpr unsigned kAll = 0xffffffffu;
    const int warp = threadIdx.x >> 5, l = threadIdx.x & 31;
    W27Stage& S = stage[warp];
    const int64_t stride = (int64_t)gridDim.x * kW27Warps;
    int64_t c = (int64_t)blockIdx.x * kW27Warps + warp;
    if (c >= n) return;  // whole warp
    int32_t nbr = l < 27 ? nn[c * 27 + l] : -1;
    w27_fill(S.tile[0], S.mt[0], nbr, src, mask, c, bck, l);
    cp_async_commit();
    nbr = (l < 27 && c + stride < n) ? nn[(c + stride) * 27 + l] : -1;
    const int q = l & 1, j = (l >> 1) & 7, z0 = (l >> 4) * 4;
    const int y = ((j & 3) << 1) | (j >> 2);
    const int hoff = q ? 12 : 3;
    for (int it = 0; c < n; ++it, c += stride) {
        const int cur = it & 1;
        const int64_t c1 = c + stride;
        if (c1 < n) w27_fill(S.tile[cur ^ 1], S.mt[cur ^ 1], nbr, src, mask, c1, bck, l);
        cp_async_commit();
        nbr = (l < 27 && c1 + stride < n) ? nn[(c1 + stride) * 27 + l] : -1;
        cp_async_wait_group<1>();  // this lane's copies of chunk c have landed
        __syncwarp();              // and every lane's
        const float* T = S.tile[cur];
        int64_t ox = 0, oy = 0, oz = 0;
        if (prm.has_box) {
            int64_t o[3];
            chunk_origin(geo, keys[c], o);
            ox = o[0];
            oy = o[1];
            oz = o[2];
        }
        // win[p][b][e] = tile cell (4q + e, y + b, plane p of the rolling window)
        float win[3][3][6];
        auto load_plane = [&](int tp, float(&pl)[3][6]) {
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                const float* rb = T + tp * kW27Plane + (y + b) * kW27Row;
                const float4 v = *reinterpret_cast<const float4*>(rb + 4 + 4 * q);
                const float hv = rb[hoff];
                const float got = __shfl_xor_sync(kAll, q ? v.x : v.w, 1);
                pl[b][0] = q ? got : hv;
                pl[b][1] = v.x;
                pl[b][2] = v.y;
                pl[b][3] = v.z;
                pl[b][4] = v.w;
                pl[b][5] = q ? hv : got;
            }
        };
        load_plane(z0, win[0]);
        load_plane(z0 + 1, win[1]);
#pragma unroll
        for (int zz = 0; zz < 4; ++zz) {
            load_plane(z0 + zz + 2, win[(zz + 2) % 3]);
            float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
            for (int a = 0; a < 3; ++a)
#pragma unroll
                for (int b = 0; b < 3; ++b)
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        const float cf = prm.coeff[a * 9 + b * 3 + d];
#pragma unroll
                        for (int i = 0; i < 4; ++i) acc[i] = __fmaf_rn(win[(zz + d) % 3][b][i + a], cf, acc[i]);
                    }
            const int z = z0 + zz, po = z * 64 + y * 8 + 4 * q;
            const uint32_t m4 = *reinterpret_cast<const uint32_t*>(S.mt[cur] + po);
            float* d = dst + c * 512 + po;
            if (!prm.has_box && (m4 & 0x03030303u) == 0x01010101u) {
                *reinterpret_cast<float4*>(d) = make_float4(acc[0], acc[1], acc[2], acc[3]);
            } else {
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    bool act = ((m4 >> (8 * i)) & 3u) == 1u;
                    if (prm.has_box) act = act && in_box(prm, ox + 4 * q + i, oy + y, oz + z);
                    if (act) d[i] = acc[i];
                }
            }
        }
        __syncwarp();  // every lane is done with tile[cur] before it is refilled
    }
    cp_async_wait_all();
}

// ------------------------------------------------------------------ many steps of a small grid in one launch
// A grid of a few hundred chunks runs each step in a few microseconds, less
// than a launch costs.  Here every step of a run is done by one cooperative
// launch (all CTAs resident): each CTA takes chunks blockIdx.x + k *
// gridDim.x, gathers the (e+2)^3 tile as k_stencil_tile does, updates, and
// the CTAs meet at a grid barrier (an arrival counter, a bounded wait)
// before the next step reads what the last one wrote.  Field reads bypass
// L1 (other SMs wrote them during the launch).  The arithmetic and the
// written points are those of k_stencil_tile.
template <int KIND, int E>
__global__ void __launch_bounds__(E * E * E < 256 ? 256 : E * E * E) k_steps_coop(FieldSet fs, const uint8_t* __restrict__ mask,
                                                    const int32_t* __restrict__ nn, int64_t n, GridInfo gi, int nsteps,
                                                    unsigned* bar, unsigned* err) {
    constexpr int T = E + 2, TT = T * T * T, BS = E * E * E;
    constexpr int NP = KIND == SGB_GS7 ? 2 : 1;
    __shared__ float tile[NP][TT];
    __shared__ int abort_run;
    if (threadIdx.x == 0) abort_run = 0;
    for (int t = 0; t < nsteps; ++t) {
        const int par = t & 1;
        const float* src[2] = {par ? fs.in[1][0] : fs.in[0][0], par ? fs.in[1][NP - 1] : fs.in[0][NP - 1]};
        float* d0 = par ? fs.out[1][0] : fs.out[0][0];
        float* d1 = par ? fs.out[1][NP - 1] : fs.out[0][NP - 1];
        for (int64_t chunk = blockIdx.x; chunk < n; chunk += gridDim.x) {
            constexpr int THREADS = BS < 256 ? 256 : BS;
            constexpr int ROUNDS = (TT + THREADS - 1) / THREADS;
            // all of the thread's tile cells are loaded before any is stored (the loads overlap)
            float v[ROUNDS][NP];
            int cells[ROUNDS];
#pragma unroll
            for (int r = 0; r < ROUNDS; ++r) {
                const int cell = threadIdx.x + r * THREADS;
                cells[r] = -1;
                if (cell >= TT) continue;
                const int tx = cell % T, ty = (cell / T) % T, tz = cell / (T * T);
                const int dx = tx == 0 ? -1 : (tx == T - 1 ? 1 : 0);
                const int dy = ty == 0 ? -1 : (ty == T - 1 ? 1 : 0);
                const int dz = tz == 0 ? -1 : (tz == T - 1 ? 1 : 0);
                if ((dx != 0) + (dy != 0) + (dz != 0) > 1) continue;  // edges / corners: unused by 7 points
                int64_t sc = chunk;
                if (dx || dy || dz) sc = nn[chunk * 8 + (dx ? (dx < 0 ? 0 : 1) : dy ? (dy < 0 ? 2 : 3) : (dz < 0 ? 4 : 5))];
                const int lx = (tx - 1 + E) % E, ly = (ty - 1 + E) % E, lz = (tz - 1 + E) % E;
                const int64_t idx = sc * BS + lx + E * (ly + E * lz);
                const bool ex = sc >= 0 && mask[idx] != 0;
                cells[r] = cell;
#pragma unroll
                for (int p = 0; p < NP; ++p) v[r][p] = ex ? __ldcg(src[p] + idx) : (par ? gi.bck[1][p] : gi.bck[0][p]);
            }
#pragma unroll
            for (int r = 0; r < ROUNDS; ++r)
                if (cells[r] >= 0)
#pragma unroll
                    for (int p = 0; p < NP; ++p) tile[p][cells[r]] = v[r][p];
            __syncthreads();
            for (int pnt = threadIdx.x; pnt < BS; pnt += blockDim.x) {
                const int x = pnt % E, y = (pnt / E) % E, z = pnt / (E * E);
                const uint8_t m = mask[chunk * BS + pnt];
                const bool act = (m & 1) && !(m & 2);
                const int c = (x + 1) + T * ((y + 1) + T * (z + 1));
                const int64_t gidx = chunk * BS + pnt;
                if (KIND == SGB_HEAT7) {
                    const float cur = tile[0][c];
                    d0[gidx] = act ? heat_update(cur, tile[0][c - 1], tile[0][c + 1], tile[0][c - T], tile[0][c + T],
                                                 tile[0][c - T * T], tile[0][c + T * T], gi.dt)
                                   : (m ? cur : (par ? gi.bck[0][0] : gi.bck[1][0]));
                } else {
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
                }
            }
            __syncthreads();
        }
        if (t + 1 < nsteps) {
            // grid barrier: arrival t + 1 of every CTA; the counter only grows.  Every thread
            // fences its stores of this step before the CTA arrives.
            __threadfence();
            __syncthreads();
            if (threadIdx.x == 0) {
                __threadfence();
                atomicAdd(bar, 1u);
                const unsigned target = (unsigned)(t + 1) * gridDim.x;
                const uint64_t t0 = global_timer_ns();
                for (uint32_t it = 0;; ++it) {
                    if (*reinterpret_cast<volatile unsigned*>(bar) >= target) break;
                    if ((it & 63u) == 63u && global_timer_ns() - t0 > 2000000000ull) {
                        atomicOr(err, kErrWaitTimeout);
                        abort_run = 1;
                        break;
                    }
                }
                __threadfence();
            }
            __syncthreads();
            if (abort_run) return;
        }
    }
}

// Runs nsteps of a HEAT7 / GS7 ping-pong on one grid as one cooperative launch; returns
// SGB_ENOTSUP when the grid is too large for it (the caller then takes the per-step path).
int run_steps_coop(sgb_grid* g, int kind, const int* src, const int* dst, const StencilParams& fwd, int nsteps,
                   cudaStream_t s) {
    if (kind != SGB_HEAT7 && kind != SGB_GS7) return SGB_ENOTSUP;
    if (g->n > (int64_t)g->num_sms * 4 || nsteps < 2) return SGB_ENOTSUP;
    if ((int64_t)nsteps * g->n >= (int64_t(1) << 31)) return SGB_ENOTSUP;  // arrival counter range
    const int np = kind == SGB_GS7 ? 2 : 1;
    FieldSet fs;
    for (int j = 0; j < 2; ++j) {
        fs.in[0][j] = g->data[src[j < np ? j : 0]].as<float>();
        fs.out[0][j] = g->data[dst[j < np ? j : 0]].as<float>();
        fs.in[1][j] = g->data[dst[j < np ? j : 0]].as<float>();
        fs.out[1][j] = g->data[src[j < np ? j : 0]].as<float>();
    }
    GridInfo gi = grid_info_of(fwd);
    const uint8_t* mask = g->mask.as<uint8_t>();
    const int32_t* nnp = g->nn[SGB_NN_STAR].as<int32_t>();
    int64_t n = g->n;
    unsigned* err = g->err.as<unsigned>();
    SGB_TRY(g->scratch[11].ensure(64));
    unsigned* bar = g->scratch[11].as<unsigned>();
    SGB_CUDA(cudaMemsetAsync(bar, 0, 4, s));
    void* kern = nullptr;
    const int e = g->geo.edge;
    if (kind == SGB_HEAT7) kern = e == 8 ? (void*)k_steps_coop<SGB_HEAT7, 8> : (void*)k_steps_coop<SGB_HEAT7, 4>;
    else kern = e == 8 ? (void*)k_steps_coop<SGB_GS7, 8> : (void*)k_steps_coop<SGB_GS7, 4>;
    const int threads = e == 8 ? 512 : 256;  // one thread per chunk point (8^3), 256 for 4^3
    int per_sm = 0;
    SGB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, 0));
    if (per_sm < 1) return SGB_ENOTSUP;
    const int64_t blocks = std::min<int64_t>(n, (int64_t)per_sm * g->num_sms);
    void* args[] = {&fs, &mask, &nnp, &n, &gi, &nsteps, &bar, &err};
    SGB_CUDA(cudaLaunchCooperativeKernel(kern, dim3((unsigned)blocks), dim3(threads), args, 0, s));
    return SGB_OK;
}

int make_params(sgb_grid* g, int kind, const int* src, const int* dst, const float* params, int nparams,
                const int64_t* box, StencilParams& prm) {
    std::memset(&prm, 0, sizeof(prm));
    if (!src || !dst || (nparams > 0 && !params)) return SGB_EINVAL;
    if (kind < SGB_HEAT7 || kind > SGB_BOX27_NS) return SGB_EINVAL;
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
        std::memcpy(&prm.bckd[j], g->bck[dst[j]], 4);
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
    for (int j = 0; j < 2; ++j) {
        gi.bck[0][j] = prm.bck[j];
        gi.bck[1][j] = prm.bckd[j];
    }
    return gi;
}

int launch_fields(const LaunchDesc& L, cudaStream_t s) {
    if (L.n == 0) return SGB_OK;
    // the pipelined kernel takes the x halo from the neighbouring index positions, which hold the
    // x neighbours only under the x-fastest chunk ids
    if (L.kind != SGB_BOX27 && L.edge == 8 && !L.use_tile && !L.geo.zorder) return launch_e8(L, s);
    if (L.kind == SGB_BOX27 && L.edge == 8 && !L.use_tile && !L.grids) {
        // 4 CTAs of four warps per SM are resident (128 registers a thread)
        const int64_t want = (L.n + kW27Warps - 1) / kW27Warps;
        const unsigned nb = (unsigned)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)L.num_sms * 4));
        k_box27_e8<<<nb, 32 * kW27Warps, 0, s>>>(L.fs.in[0][0], L.fs.out[0][0], L.mask, L.nn, L.keys, L.n, L.geo, L.prm,
                                      L.g0.bck[0][0]);
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
    if (kind == SGB_BOX27_NS) return launch_points_box27(g, src, dst, prm, s);
    if (kind == SGB_BOX27 && !use_tile) {  // sparse chunks: the point list
        const int st = launch_points_box27_sparse(g, src, dst, prm, s);
        if (st != SGB_ENOTSUP) return st;
    }
    const int nnk = kind == SGB_BOX27 ? SGB_NN_FULL : SGB_NN_STAR;
    SGB_TRY(ensure_neighbours(g, nnk, s));
    const int np = kind == SGB_GS7 ? 2 : 1;
    for (int j = 0; j < np; ++j) SGB_TRY(ensure_clean(g, src[j], s));
    LaunchDesc L;
    std::memset(&L, 0, sizeof(L));
    L.kind = kind;
    L.edge = g->geo.edge;
    L.use_tile = use_tile;
    L.stages = g->stages;
    L.num_sms = g->num_sms;
    const int cps = g->ctas_per_sm > 0 ? g->ctas_per_sm : auto_ctas_per_sm(kind);
    L.ctas = (unsigned)std::max<int64_t>(1, std::min<int64_t>(g->n, (int64_t)g->num_sms * cps));
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
    L.arr_chunks = g->n + 1;
    L.geo = g->geo;
    L.prm = prm;
    L.t = 0;
    L.err = g->err.as<unsigned>();
    SGB_TRY(launch_fields(L, s));
    if (kind == SGB_HEAT7) g->clean[dst[0]] = true;  // every point of dst was written from the tile
    return SGB_OK;
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
    SGB_TRY(ensure_neighbours(g, kind == SGB_BOX27 || kind == SGB_BOX27_NS ? SGB_NN_FULL : SGB_NN_STAR, s));
    if (kind == SGB_BOX27_NS || kind == SGB_BOX27) SGB_TRY(ensure_point_list(g, s));  // built outside the capture
    // both halves of the ping-pong are read as sources; no sanitising inside a capture
    for (int j = 0; j < (kind == SGB_GS7 ? 2 : 1); ++j) {
        SGB_TRY(ensure_clean(g, src[j], s));
        SGB_TRY(ensure_clean(g, dst[j], s));
    }
    // a small grid: all steps in one cooperative launch
    {
        const int st = run_steps_coop(g, kind, src, dst, fwd, nsteps, s);
        if (st == SGB_OK) {
            if (kind == SGB_HEAT7) g->clean[nsteps % 2 ? dst[0] : src[0]] = true;
            return SGB_OK;
        }
        if (st != SGB_ENOTSUP) return st;
    }
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
