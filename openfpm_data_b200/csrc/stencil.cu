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
// One chunk at a time per 64-thread CTA (grid-stride), software-pipelined:
// while chunk i is computed from one 10^3 shared tile, the tile of chunk
// i + 1 is being filled in the other by cp.async copies (16-byte copies of
// the chunk's rows, 4-byte copies of the six faces, twelve edges and eight
// corners from the 26 NNFull neighbours; an absent neighbour's cells get the
// background with plain stores) and the chunk's mask bytes alongside.  Tile
// cell (x, y, z), x, y, z in 0..9, sits at z * 240 + y * 24 + x + 3: rows of
// 24 floats put the chunk's part of every row on a 16-byte boundary, and the
// four rows a warp reads at once fall into disjoint banks.  The neighbour rows are read two chunks
// ahead.  Thread t owns the column (x, y) = (t % 8, t / 8) and marches z
// holding the 3 x 3 x 3 window in registers: per point 9 shared loads and
// the 27 FMAs in Conv3x3x3's order (x offset outermost, z innermost).
// Results equal the tile kernel's bit for bit (the background invariant
// makes a stored non-existing point read the same as the substituted
// background).
constexpr int kB27Plane = 240, kB27Row = 24, kB27Tile = 10 * kB27Plane;

__device__ __forceinline__ void box27_fill(float* tile, uint8_t* mt, const int32_t* nb, const float* __restrict__ src,
                                           const uint8_t* __restrict__ mask, int64_t c, float bck, int t) {
    if (t < 32) cp_async16(mt + t * 16, mask + c * 512 + t * 16);
    // interior: row (y, z) = (t % 8, t / 8), two 16-byte copies
    {
        const float* row = src + c * 512 + t * 8;
        float* d = &tile[((t >> 3) + 1) * kB27Plane + ((t & 7) + 1) * kB27Row + 4];
        cp_async16(d, row);
        cp_async16(d + 4, row + 4);
    }
    const int u = t & 7, v = t >> 3;
    auto cell = [&](int ti, int32_t sc, int64_t off) {
        if (sc >= 0) cp_async4(&tile[ti], src + (int64_t)sc * 512 + off);
        else tile[ti] = bck;
    };
    // faces: cell (u, v) of each; slot = px + 3 py + 9 pz
    auto at = [](int x, int y, int z) { return z * kB27Plane + y * kB27Row + x + 3; };
    cell(at(0, u + 1, v + 1), nb[12], v * 64 + u * 8 + 7);
    cell(at(9, u + 1, v + 1), nb[14], v * 64 + u * 8 + 0);
    cell(at(u + 1, 0, v + 1), nb[10], v * 64 + 7 * 8 + u);
    cell(at(u + 1, 9, v + 1), nb[16], v * 64 + 0 * 8 + u);
    cell(at(u + 1, v + 1, 0), nb[4], 7 * 64 + v * 8 + u);
    cell(at(u + 1, v + 1, 9), nb[22], 0 * 64 + v * 8 + u);
    // edges (12 x 8 cells) and corners (8)
    for (int e = t; e < 104; e += 64) {
        int tx, ty, tz;
        if (e < 96) {
            const int k = e >> 3, w = (e & 7) + 1;  // edge k, position w along it
            const int a = (k & 1) ? 9 : 0, b = (k & 2) ? 9 : 0;
            if (k < 4) { tx = w; ty = a; tz = b; }          // edges along x
            else if (k < 8) { tx = a; ty = w; tz = b; }     // along y
            else { tx = a; ty = b; tz = w; }                // along z
        } else {
            const int k = e - 96;
            tx = (k & 1) ? 9 : 0;
            ty = (k & 2) ? 9 : 0;
            tz = (k & 4) ? 9 : 0;
        }
        const int px = tx == 0 ? 0 : (tx == 9 ? 2 : 1), py = ty == 0 ? 0 : (ty == 9 ? 2 : 1),
                  pz = tz == 0 ? 0 : (tz == 9 ? 2 : 1);
        const int lx = (tx + 7) & 7, ly = (ty + 7) & 7, lz = (tz + 7) & 7;
        cell(at(tx, ty, tz), nb[px + 3 * py + 9 * pz], lz * 64 + ly * 8 + lx);
    }
}

__global__ void __launch_bounds__(64, 10) k_box27_e8(const float* __restrict__ src, float* __restrict__ dst,
                                                 const uint8_t* __restrict__ mask, const int32_t* __restrict__ nn,
                                                 const int64_t* __restrict__ keys, int64_t n, Geometry geo,
                                                 StencilParams prm, float bck) {
    __shared__ __align__(16) float tile[2][kB27Tile];
    __shared__ __align__(16) uint8_t mt[2][512];
    __shared__ int32_t nbs[2][28];
    const int t = threadIdx.x;
    const int cx = t & 7, cy = t >> 3;
    const int64_t stride = gridDim.x;
    int64_t c = blockIdx.x;
    if (c >= n) return;
    // neighbour rows: of the first chunk now, of the second in a register
    if (t < 27) nbs[0][t] = t == 13 ? (int32_t)c : nn[c * 27 + t];
    int32_t nb_next = -1;
    if (t < 27 && c + stride < n) nb_next = t == 13 ? (int32_t)(c + stride) : nn[(c + stride) * 27 + t];
    __syncthreads();
    box27_fill(tile[0], mt[0], nbs[0], src, mask, c, bck, t);
    cp_async_commit();
    for (int it = 0; c < n; ++it, c += stride) {
        const int cur = it & 1, nxt = cur ^ 1;
        const int64_t c1 = c + stride;
        // the next chunk's neighbour row to shared memory, the one after it to a register
        if (t < 27) nbs[nxt][t] = nb_next;
        if (t < 27 && c1 + stride < n) nb_next = t == 13 ? (int32_t)(c1 + stride) : nn[(c1 + stride) * 27 + t];
        __syncthreads();  // nbs[nxt] visible; every thread is done with tile[nxt] (chunk it - 1)
        if (c1 < n) box27_fill(tile[nxt], mt[nxt], nbs[nxt], src, mask, c1, bck, t);
        cp_async_commit();
        cp_async_wait_group<1>();  // this thread's copies of chunk c have landed
        __syncthreads();           // and everyone's
        const float* T0 = tile[cur];
        int64_t ox = 0, oy = 0, oz = 0;
        if (prm.has_box) {
            int64_t o[3];
            chunk_origin(geo, keys[c], o);
            ox = o[0];
            oy = o[1];
            oz = o[2];
        }
        // window w[a][b][d] = tile[z + d][y + b][x + a] (a, b in 0..2, d in 0..3, tile coordinates):
        // two points (z, z + 1) per step, their two FMA chains interleaved
        float w[3][3][4];
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                w[a][b][0] = T0[0 * kB27Plane + (cy + b) * kB27Row + (cx + a) + 3];
                w[a][b][1] = T0[1 * kB27Plane + (cy + b) * kB27Row + (cx + a) + 3];
            }
#pragma unroll
        for (int z = 0; z < 8; z += 2) {
#pragma unroll
            for (int a = 0; a < 3; ++a)
#pragma unroll
                for (int b = 0; b < 3; ++b) {
                    w[a][b][2] = T0[(z + 2) * kB27Plane + (cy + b) * kB27Row + (cx + a) + 3];
                    w[a][b][3] = T0[(z + 3) * kB27Plane + (cy + b) * kB27Row + (cx + a) + 3];
                }
            float tot0 = 0.0f, tot1 = 0.0f;
#pragma unroll
            for (int a = 0; a < 3; ++a)
#pragma unroll
                for (int b = 0; b < 3; ++b)
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        const float cf = prm.coeff[a * 9 + b * 3 + d];
                        tot0 = __fmaf_rn(w[a][b][d], cf, tot0);
                        tot1 = __fmaf_rn(w[a][b][d + 1], cf, tot1);
                    }
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int zz = z + h;
                const uint8_t m = mt[cur][zz * 64 + cy * 8 + cx];
                bool act = (m & 3) == 1;
                if (prm.has_box) act = act && in_box(prm, ox + cx, oy + cy, oz + zz);
                if (act) dst[c * 512 + zz * 64 + cy * 8 + cx] = h ? tot1 : tot0;
            }
#pragma unroll
            for (int a = 0; a < 3; ++a)
#pragma unroll
                for (int b = 0; b < 3; ++b) {
                    w[a][b][0] = w[a][b][2];
                    w[a][b][1] = w[a][b][3];
                }
        }
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
        // 10 CTAs of 64 threads per SM are resident (20 KB of shared memory each)
        const unsigned nb = (unsigned)std::max<int64_t>(1, std::min<int64_t>(L.n, (int64_t)L.num_sms * 10));
        k_box27_e8<<<nb, 64, 0, s>>>(L.fs.in[0][0], L.fs.out[0][0], L.mask, L.nn, L.keys, L.n, L.geo, L.prm,
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
