// CPU restatement of openfpm_data's SparseGridGpu hot path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the parity oracle: tests/, the smoke
// check and bench.py's CPU-baseline leg call it to check (never to produce) the
// results of the CUDA library.  Nothing in the product path links or loads it.
//
// The reference (mosaic-group/openfpm_data) cannot be compiled here: it needs
// Boost MPL/Fusion, Vc and the openfpm_devices sibling repository.  This file
// therefore restates its arithmetic, cited function by function.  Parity of
// the restatement is pinned by tests/test_oracle_golden.py against the
// known-answer tests that the reference ships for this path.
//
// Data model (mirrors the reference's memory_traits_inte SoA layout):
//   keys[n]                 sorted chunk ids (indexT = long)
//   data[p][(n+1)*bs]       one array per property, chunk-major, the chunk
//                           at position n is the background chunk
//   mask[(n+1)*bs]          uint8 per point: bit0 EXIST, bit1 PADDING
//
// Floating point: the reference compiles its kernels with -use_fast_math
// (src/CMakeLists.txt:158), i.e. FMA contraction and flush-to-zero.  Every
// compute entry point below runs with the SSE FTZ|DAZ bits set and writes the
// FMAs that nvcc contracts as explicit fmaf() calls.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <thread>
#include <vector>
#include <xmmintrin.h>

namespace {

enum { T_F32 = 0, T_I32 = 1, T_F64 = 2, T_U8 = 3 };
enum { OP_NONE = 0, OP_RIGHT = 1, OP_LEFT = 2, OP_ADD = 3, OP_MAX = 4, OP_MIN = 5, OP_OR = 6 };
enum { NN_STAR = 0, NN_FULL = 1 };

struct FtzScope {
    unsigned old;
    FtzScope() : old(_mm_getcsr()) { _mm_setcsr(old | 0x8040u); }  // FTZ | DAZ
    ~FtzScope() { _mm_setcsr(old); }
};

int elem_size(int t) { return t == T_F64 ? 8 : (t == T_U8 ? 1 : 4); }

struct Grid {
    int dim = 3, edge = 8, bs = 512;
    bool zorder = false;  // chunk ids: grid_smb (false) or grid_zmb Morton codes (true)
    int64_t sz[3] = {1, 1, 1}, bsz[3] = {1, 1, 1};
    int nprop = 0;
    std::vector<int> ptype;
    std::vector<int64_t> keys;
    std::vector<std::vector<uint8_t>> data;
    std::vector<uint8_t> mask;
    std::vector<std::array<uint8_t, 8>> bck;

    int64_t n() const { return (int64_t)keys.size(); }
    int es(int p) const { return elem_size(ptype[p]); }
    uint8_t* at(int p, int64_t chunk, int off) { return &data[p][((size_t)chunk * bs + off) * es(p)]; }
    void reset_background() {
        // resetBck: re-append the background chunk (map_vector_sparse.hpp:1356-1364,
        // BlockMapGpu.hpp:320-340: data = background value, mask = 0).
        int64_t nc = n();
        for (int p = 0; p < nprop; ++p) {
            data[p].resize((size_t)(nc + 1) * bs * es(p));
            for (int o = 0; o < bs; ++o) std::memcpy(at(p, nc, o), bck[p].data(), es(p));
        }
        mask.resize((size_t)(nc + 1) * bs);
        std::fill(mask.begin() + (size_t)nc * bs, mask.end(), 0);
    }
};

// ---------------------------------------------------------------- grid_zmb
// lin_zid / invlin_zid (src/util/zmorton.hpp:72-135): bit i of the block
// coordinate along d is bit 3i + d of the chunk id (written here bit by bit).
int64_t morton3(const int64_t* bc) {
    uint64_t r = 0;
    for (int i = 0; i < 21; ++i)
        for (int d = 0; d < 3; ++d) r |= (((uint64_t)bc[d] >> i) & 1u) << (3 * i + d);
    return (int64_t)r;
}
void inv_morton3(int64_t key, int64_t* bc) {
    for (int d = 0; d < 3; ++d) {
        bc[d] = 0;
        for (int i = 0; i < 21; ++i) bc[d] |= (int64_t)((((uint64_t)key >> (3 * i + d)) & 1u) << i);
    }
}

// ---------------------------------------------------------------- grid_smb
// grid_smb::LinId (src/Grid/Geometry/grid_smb.hpp:176-190); grid_zmb::LinId
// (grid_zmb.hpp:63-76) for Morton grids
int64_t lin_id(const Grid& g, const int64_t* c) {
    if (g.zorder) {
        const int64_t bc[3] = {c[0] / g.edge, c[1] / g.edge, c[2] / g.edge};
        return morton3(bc) * g.bs + (c[0] % g.edge) + g.edge * ((c[1] % g.edge) + g.edge * (c[2] % g.edge));
    }
    int64_t b = c[g.dim - 1] / g.edge, l = c[g.dim - 1] % g.edge;
    for (int d = g.dim - 2; d >= 0; --d) {
        b = b * g.bsz[d] + c[d] / g.edge;
        l = l * g.edge + c[d] % g.edge;
    }
    return b * g.bs + l;
}

// grid_smb::InvLinId (grid_smb.hpp:263-277)
void inv_lin(const Grid& g, int64_t lin, int64_t* c) {
    int64_t b = lin / g.bs, l = lin % g.bs;
    if (g.zorder) {
        inv_morton3(b, c);
        for (int d = 0; d < 3; ++d) {
            c[d] = c[d] * g.edge + l % g.edge;
            l /= g.edge;
        }
        return;
    }
    for (int d = 0; d < g.dim; ++d) {
        c[d] = (b % g.bsz[d]) * g.edge + l % g.edge;
        b /= g.bsz[d];
        l /= g.edge;
    }
}

// grid_smb::BlockInvLinId (grid_smb.hpp:313-323)
void block_coord(const Grid& g, int64_t b, int64_t* bc) {
    if (g.zorder) {
        inv_morton3(b, bc);
        return;
    }
    for (int d = 0; d < g.dim; ++d) {
        bc[d] = b % g.bsz[d];
        b /= g.bsz[d];
    }
}

// grid_smb::BlockLinId (grid_smb.hpp:280-299).  Only the upper bound is
// checked: a block coordinate of -1 produces a (possibly valid) wrapped id.
// grid_zmb::BlockLinId checks nothing; its id of a negative coordinate lies
// above every chunk's, i.e. absent (-1 here).
int64_t block_lin_ref(const Grid& g, const int64_t* bc) {
    if (g.zorder) return (bc[0] < 0 || bc[1] < 0 || bc[2] < 0) ? -1 : morton3(bc);
    int64_t lin = bc[g.dim - 1];
    if (lin >= g.bsz[g.dim - 1]) return -1;
    for (int d = g.dim - 2; d >= 0; --d) {
        lin *= g.bsz[d];
        int64_t cur = bc[d];
        if (cur >= g.bsz[d]) return -1;
        lin += cur;
    }
    return lin;
}

// vector_sparse_gpu_ker::_branchfree_search (map_vector_sparse_cuda_ker.cuh:75-92):
// position of the key, or the background position n when absent.
int64_t search(const Grid& g, int64_t key) {
    auto it = std::lower_bound(g.keys.begin(), g.keys.end(), key);
    if (it != g.keys.end() && *it == key) return it - g.keys.begin();
    return g.n();
}

// ---------------------------------------------------------------- neighbours
int nnn(const Grid& g, int kind) {
    if (kind == NN_STAR) return 1 << g.dim;              // NNStar::nNN = 2^dim
    return g.dim == 3 ? 27 : 9;                           // NNFull::nNN = 3^dim
}

// findNeighbours (SparseGridGpu_kernels.cuh:1014-1035) with
// NNStar::getNNpos (SparseGridGpu_ker_util.hpp:91-112) and
// NNFull::getNNpos (SparseGridGpu.hpp:266-287).
std::vector<int64_t> find_neighbours(const Grid& g, int kind) {
    const int k = nnn(g, kind);
    std::vector<int64_t> out((size_t)g.n() * k);
    for (int64_t i = 0; i < g.n(); ++i) {
        for (int o = 0; o < k; ++o) {
            int64_t bc[3];
            block_coord(g, g.keys[i], bc);
            int64_t pos;
            if (kind == NN_STAR) {
                pos = -1;
                if (o < 2 * g.dim) {
                    int d = o / 2;
                    int64_t dpos = bc[d] + (o % 2) * 2 - 1;
                    bc[d] = dpos;
                    int bl = (int)block_lin_ref(g, bc);
                    bl = dpos < 0 ? -1 : bl;
                    pos = search(g, bl);
                }
            } else {
                pos = g.n();
                if (o != k / 2) {
                    int cnt = o;
                    for (int d = 0; d < g.dim; ++d) {
                        bc[d] += cnt % 3 - 1;
                        cnt /= 3;
                    }
                    pos = search(g, block_lin_ref(g, bc));
                }
            }
            out[(size_t)i * k + o] = pos;
        }
    }
    return out;
}

// Position in the neighbour table of the chunk holding an enlarged-tile cell
// whose per-dimension offsets (-1, 0, +1) are in dd.  NNStar only has faces.
int nn_slot(const Grid& g, int kind, const int* dd) {
    if (kind == NN_FULL) {
        int s = 0, m = 1;
        for (int d = 0; d < g.dim; ++d) { s += (dd[d] + 1) * m; m *= 3; }
        return s;
    }
    // NNStar::getNNskin (SparseGridGpu_ker_util.hpp:114-139): faces map to
    // 2d / 2d+1; edges and corners to neighbour 0.
    int slot = -1, ctr = 0;
    for (int d = 0; d < g.dim; ++d) {
        if (dd[d] < 0) { slot = 2 * d; ++ctr; }
        else if (dd[d] > 0) { slot = 2 * d + 1; ++ctr; }
    }
    return ctr > 1 ? 0 : slot;
}

// loadGhostBlock_impl<1>::load (SparseGridGpu_ker_util.hpp:487-564): fill the
// (edge+2)^dim tile of chunk i with property p (or the mask when p < 0).
// A cell whose source mask byte is 0 takes the background value (not for the
// mask itself).  The centre chunk comes from its own position.
template <typename T>
void load_tile(const Grid& g, const std::vector<int64_t>& nn, int kind, int64_t i, int p,
               std::vector<T>& tile) {
    const int e = g.edge, E = e + 2, k = nnn(g, kind);
    int tsz = 1;
    for (int d = 0; d < g.dim; ++d) tsz *= E;
    tile.assign(tsz, T(0));
    for (int t = 0; t < tsz; ++t) {
        int tc[3] = {0, 0, 0}, dd[3] = {0, 0, 0}, lc[3] = {0, 0, 0};
        int rem = t;
        bool halo = false;
        for (int d = 0; d < g.dim; ++d) {
            tc[d] = rem % E;
            rem /= E;
            int v = tc[d] - 1;
            dd[d] = v < 0 ? -1 : (v >= e ? 1 : 0);
            lc[d] = v < 0 ? v + e : (v >= e ? v - e : v);
            halo |= dd[d] != 0;
        }
        int off = 0, m = 1;
        for (int d = 0; d < g.dim; ++d) { off += lc[d] * m; m *= e; }
        int64_t src = i;
        if (halo) {
            int slot = nn_slot(g, kind, dd);
            src = nn[(size_t)i * k + slot];
        }
        uint8_t mk = g.mask[(size_t)src * g.bs + off];
        if (p < 0) {
            tile[t] = (T)mk;
        } else {
            T v;
            if (mk == 0) std::memcpy(&v, g.bck[p].data(), sizeof(T));
            else std::memcpy(&v, &g.data[p][((size_t)src * g.bs + off) * sizeof(T)], sizeof(T));
            tile[t] = v;
        }
    }
}

int tile_index(const Grid& g, const int* tc) {
    const int E = g.edge + 2;
    int s = 0, m = 1;
    for (int d = 0; d < g.dim; ++d) { s += tc[d] * m; m *= E; }
    return s;
}

void local_coord(const Grid& g, int off, int* lc) {
    for (int d = 0; d < g.dim; ++d) { lc[d] = off % g.edge; off /= g.edge; }
}

// applyStencilInPlace (SparseGridGpu_kernels.cuh:1045-1094): the mask is
// cleared for points outside the inclusive box [lo, hi].
uint8_t cur_mask(const Grid& g, int64_t i, int off, const int64_t* box) {
    uint8_t m = g.mask[(size_t)i * g.bs + off];
    if (box) {
        int64_t c[3];
        inv_lin(g, g.keys[i] * g.bs + off, c);
        for (int d = 0; d < g.dim; ++d)
            if (c[d] < box[d] || c[d] > box[3 + d]) m = 0;
    }
    return m;
}

bool active(uint8_t m) { return (m & 1) && !(m & 2); }

// ---------------------------------------------------------------- flush
template <typename T>
T apply_op_t(int op, T a, T b) {
    switch (op) {
        case OP_RIGHT: return b;                 // rightOperand_t (map_vector_sparse_cuda_kernels.cuh:43-48)
        case OP_LEFT: return a;                  // leftOperand_t (:74-79)
        case OP_ADD: return a + b;               // sadd_ -> plus_t
        case OP_MAX: return a > b ? a : b;       // smax_ -> maximum_t
        case OP_MIN: return a < b ? a : b;       // smin_ -> minimum_t
        default: return b;
    }
}

// BlockMapGpuKernels::applyOp (BlockMapGpu_kernels.cuh:151-167).
void apply_op(int type, int op, uint8_t* a, const uint8_t* b, bool ae, bool be) {
    if (ae && be) {
        if (type == T_F32) { float x, y; std::memcpy(&x, a, 4); std::memcpy(&y, b, 4); x = apply_op_t(op, x, y); std::memcpy(a, &x, 4); }
        else if (type == T_F64) { double x, y; std::memcpy(&x, a, 8); std::memcpy(&y, b, 8); x = apply_op_t(op, x, y); std::memcpy(a, &x, 8); }
        else if (type == T_I32) {
            int32_t x, y; std::memcpy(&x, a, 4); std::memcpy(&y, b, 4);
            x = op == OP_OR ? (x | y) : apply_op_t(op, x, y);
            std::memcpy(a, &x, 4);
        } else {
            uint8_t x = *a, y = *b;
            *a = op == OP_OR ? (uint8_t)(x | y) : apply_op_t(op, x, y);
        }
    } else if (be) {
        std::memcpy(a, b, elem_size(type));
    }
}

// Merge the sorted unique new chunk keys into the map; returns for every old
// chunk its new position and for every new key its position.  This is the
// layout that merge_indexes + solve_conflicts produce (map_vector_sparse.hpp:
// 1004-1190, BlockMapGpu_kernels.cuh:701-807): a sorted union of keys, data
// position == key position, background chunk last.
void merged_layout(const Grid& g, const std::vector<int64_t>& ukeys, std::vector<int64_t>& merged,
                   std::vector<int64_t>& old_pos, std::vector<int64_t>& new_pos, std::vector<int64_t>& new_old) {
    merged.clear();
    std::set_union(g.keys.begin(), g.keys.end(), ukeys.begin(), ukeys.end(), std::back_inserter(merged));
    old_pos.resize(g.keys.size());
    for (size_t j = 0; j < g.keys.size(); ++j)
        old_pos[j] = std::lower_bound(merged.begin(), merged.end(), g.keys[j]) - merged.begin();
    new_pos.resize(ukeys.size());
    new_old.resize(ukeys.size());
    for (size_t j = 0; j < ukeys.size(); ++j) {
        new_pos[j] = std::lower_bound(merged.begin(), merged.end(), ukeys[j]) - merged.begin();
        auto it = std::lower_bound(g.keys.begin(), g.keys.end(), ukeys[j]);
        new_old[j] = (it != g.keys.end() && *it == ukeys[j]) ? (it - g.keys.begin()) : -1;
    }
}

// Rebuild the data arrays for the merged layout: old chunks keep their
// content at their new position, chunks that are new start as background with
// an empty mask.
void relayout(Grid& g, const std::vector<int64_t>& merged, const std::vector<int64_t>& old_pos) {
    const int64_t nn_ = (int64_t)merged.size();
    std::vector<std::vector<uint8_t>> nd(g.nprop);
    std::vector<uint8_t> nm((size_t)(nn_ + 1) * g.bs, 0);
    for (int p = 0; p < g.nprop; ++p) {
        int es = g.es(p);
        nd[p].resize((size_t)(nn_ + 1) * g.bs * es);
        for (int64_t c = 0; c <= nn_; ++c)
            for (int o = 0; o < g.bs; ++o) std::memcpy(&nd[p][((size_t)c * g.bs + o) * es], g.bck[p].data(), es);
        for (size_t j = 0; j < old_pos.size(); ++j)
            std::memcpy(&nd[p][(size_t)old_pos[j] * g.bs * es], &g.data[p][j * g.bs * es], (size_t)g.bs * es);
    }
    for (size_t j = 0; j < old_pos.size(); ++j)
        std::memcpy(&nm[(size_t)old_pos[j] * g.bs], &g.mask[j * g.bs], g.bs);
    g.keys = merged;
    g.data.swap(nd);
    g.mask.swap(nm);
}

// One chunk of a HeatStencil step into `out` (the destination array's bytes).
void heat7_chunk(const Grid& g, const std::vector<int64_t>& nn, int64_t i, int src, float dt, const int64_t* box,
                 std::vector<float>& tile, std::vector<uint8_t>& out) {
    load_tile(g, nn, NN_STAR, i, src, tile);
    for (int o = 0; o < g.bs; ++o) {
        int lc[3] = {0, 0, 0}, tc[3] = {0, 0, 0};
        local_coord(g, o, lc);
        for (int d = 0; d < g.dim; ++d) tc[d] = lc[d] + 1;
        float cur = tile[tile_index(g, tc)];
        float res = cur;
        if (active(cur_mask(g, i, o, box))) {
            // laplacian = -2.0*dim*cur (exact in double, narrowed to float), then per dimension
            // += neighbourMinus + neighbourPlus: nvcc fuses the narrowed product with the first sum
            // (x) into one fma; res = cur + dt*laplacian is an fma too
            float lap = 0.0f;
            for (int d = 0; d < g.dim; ++d) {
                int a[3] = {tc[0], tc[1], tc[2]}, b[3] = {tc[0], tc[1], tc[2]};
                a[d] -= 1;
                b[d] += 1;
                const float pair = tile[tile_index(g, a)] + tile[tile_index(g, b)];
                lap = d == 0 ? std::fmaf((float)(-2.0 * g.dim), cur, pair) : lap + pair;
            }
            res = std::fmaf(dt, lap, cur);
        }
        std::memcpy(&out[((size_t)i * g.bs + o) * 4], &res, 4);
    }
}

// One chunk of a Gray-Scott step into `ou` / `ov` (the destination arrays' bytes).
void gs7_chunk(const Grid& g, const std::vector<int64_t>& nn, int64_t i, int pu, int pv, float Du, float Dv, float F,
               float nfk, float dt, const int64_t* box, std::vector<float>& tu, std::vector<float>& tv,
               std::vector<uint8_t>& ou, std::vector<uint8_t>& ov) {
    load_tile(g, nn, NN_STAR, i, pu, tu);
    load_tile(g, nn, NN_STAR, i, pv, tv);
    for (int o = 0; o < g.bs; ++o) {
        if (!active(cur_mask(g, i, o, box))) continue;
        int lc[3] = {0, 0, 0}, tc[3] = {0, 0, 0};
        local_coord(g, o, lc);
        for (int d = 0; d < g.dim; ++d) tc[d] = lc[d] + 1;
        int ci = tile_index(g, tc);
        float u = tu[ci], v = tv[ci];
        float lu = (float)(-2.0 * g.dim * (double)u), lv = (float)(-2.0 * g.dim * (double)v);
        for (int d = 0; d < g.dim; ++d) {
            int a[3] = {tc[0], tc[1], tc[2]}, b[3] = {tc[0], tc[1], tc[2]};
            a[d] -= 1;
            b[d] += 1;
            int ia = tile_index(g, a), ib = tile_index(g, b);
            lu = lu + (tu[ia] + tu[ib]);
            lv = lv + (tv[ia] + tv[ib]);
        }
        float uvv = (u * v) * v;
        float du = std::fmaf(F, 1.0f - u, std::fmaf(Du, lu, -uvv));
        float dv = std::fmaf(nfk, v, std::fmaf(Dv, lv, uvv));
        float un = std::fmaf(dt, du, u), vn = std::fmaf(dt, dv, v);
        std::memcpy(&ou[((size_t)i * g.bs + o) * 4], &un, 4);
        std::memcpy(&ov[((size_t)i * g.bs + o) * 4], &vn, 4);
    }
}

// Runs body(lo, hi) over [0, n) split into `threads` ranges (the floating-point mode as it is).
template <typename F>
void for_chunks_plain(int64_t n, int threads, F body) {
    threads = std::max(1, std::min<int>(threads, 256));
    if (threads == 1 || n < 2) {
        body(0, n);
        return;
    }
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t) {
        const int64_t lo = n * t / threads, hi = n * (t + 1) / threads;
        pool.emplace_back([&body, lo, hi] { body(lo, hi); });
    }
    for (auto& th : pool) th.join();
}

// Runs body(lo, hi) over [0, n) split into `threads` ranges, each thread with FTZ|DAZ set.
template <typename F>
void for_chunks(int64_t n, int threads, F body) {
    threads = std::max(1, std::min<int>(threads, 256));
    if (threads == 1 || n < 2) {
        FtzScope ftz;
        body(0, n);
        return;
    }
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t) {
        const int64_t lo = n * t / threads, hi = n * (t + 1) / threads;
        pool.emplace_back([&body, lo, hi] {
            FtzScope ftz;
            body(lo, hi);
        });
    }
    for (auto& th : pool) th.join();
}

}  // namespace

// =================================================================== C API
extern "C" {

void sgo_set_zorder(void* h, int z) { ((Grid*)h)->zorder = z != 0; }

void* sgo_create(int dim, int edge, const int64_t* size, int nprop, const int* ptypes) {
    Grid* g = new Grid();
    g->dim = dim;
    g->edge = edge;
    g->bs = 1;
    for (int d = 0; d < dim; ++d) {
        g->bs *= edge;
        g->sz[d] = size[d];
        g->bsz[d] = size[d] / edge + ((size[d] % edge) != 0);  // grid_smb ctor (grid_smb.hpp:48-57)
    }
    g->nprop = nprop;
    g->ptype.assign(ptypes, ptypes + nprop);
    g->data.resize(nprop);
    g->bck.assign(nprop, std::array<uint8_t, 8>{});
    g->reset_background();
    return g;
}

void sgo_destroy(void* h) { delete (Grid*)h; }

// setBackgroundValue (SparseGridGpu.hpp:2878-2884, BlockMapGpu.hpp:320-340).
void sgo_set_background(void* h, int p, const void* v) {
    Grid* g = (Grid*)h;
    std::memcpy(g->bck[p].data(), v, g->es(p));
    g->reset_background();
}

int64_t sgo_nchunks(void* h) { return ((Grid*)h)->n(); }

void sgo_lin_ids(void* h, int64_t n, const int64_t* coords, int64_t* out) {
    Grid* g = (Grid*)h;
    for (int64_t i = 0; i < n; ++i) out[i] = lin_id(*g, coords + i * g->dim);
}

void sgo_inv_lin(void* h, int64_t n, const int64_t* lin, int64_t* coords) {
    Grid* g = (Grid*)h;
    for (int64_t i = 0; i < n; ++i) inv_lin(*g, lin[i], coords + i * g->dim);
}

// Replace the whole block map (keys sorted, data without background chunk).
void sgo_load_map(void* h, int64_t n, const int64_t* keys, const void* const* data, const uint8_t* mask) {
    Grid* g = (Grid*)h;
    g->keys.assign(keys, keys + n);
    for (int p = 0; p < g->nprop; ++p) {
        g->data[p].assign((const uint8_t*)data[p], (const uint8_t*)data[p] + (size_t)n * g->bs * g->es(p));
    }
    g->mask.assign(mask, mask + (size_t)n * g->bs);
    g->reset_background();
}

// Copy out keys, data (n+1 chunks including the background) and mask.
void sgo_export_map(void* h, int64_t* keys, void* const* data, uint8_t* mask) {
    Grid* g = (Grid*)h;
    if (keys) std::memcpy(keys, g->keys.data(), g->keys.size() * 8);
    for (int p = 0; p < g->nprop; ++p)
        if (data && data[p]) std::memcpy(data[p], g->data[p].data(), g->data[p].size());
    if (mask) std::memcpy(mask, g->mask.data(), g->mask.size());
}

// Flush at the reference's own granularity: every insert owns a whole chunk
// slot (vector_sparse_gpu_ker::insert, map_vector_sparse_cuda_ker.cuh:309-318).
// Slots are reduced in a stable order by key (CUB radix sort is stable,
// sort_ofp.cuh:335-376): A = first slot; A = op(A, next) under the applyOp
// mask rule; then A = op(A, old); masks are OR-ed (segreduce_total[_with_mask],
// BlockMapGpu_kernels.cuh:181-477).  Properties with OP_NONE are not written
// for chunks that received inserts (solve_conflicts only launches the
// reduction for listed properties, :786-794): the oracle leaves the old value
// (background for new chunks) there; the reference leaves them undefined.
void sgo_flush_chunks(void* h, int64_t nslots, const int64_t* slot_keys, const void* const* slot_data,
                      const uint8_t* slot_mask, const int* ops) {
    Grid* g = (Grid*)h;
    if (nslots == 0) return;
    std::vector<int64_t> order(nslots);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return slot_keys[a] < slot_keys[b]; });
    std::vector<int64_t> ukeys, seg;
    for (int64_t i = 0; i < nslots; ++i) {
        if (i == 0 || slot_keys[order[i]] != slot_keys[order[i - 1]]) { ukeys.push_back(slot_keys[order[i]]); seg.push_back(i); }
    }
    seg.push_back(nslots);
    std::vector<int64_t> merged, old_pos, new_pos, new_old;
    merged_layout(*g, ukeys, merged, old_pos, new_pos, new_old);
    Grid old = *g;
    relayout(*g, merged, old_pos);
    const int bs = g->bs;
    bool any_listed = false;
    for (int p = 0; p < g->nprop; ++p) any_listed |= ops[p] != OP_NONE;
    for (size_t s = 0; s + 1 < seg.size(); ++s) {
        int64_t P = new_pos[s], O = new_old[s];
        for (int o = 0; o < bs; ++o) {
            for (int p = 0; p < g->nprop; ++p) {
                if (ops[p] == OP_NONE) continue;
                int es = g->es(p);
                uint8_t A[8];
                int64_t first = order[seg[s]];
                std::memcpy(A, (const uint8_t*)slot_data[p] + ((size_t)first * bs + o) * es, es);
                uint8_t am = slot_mask[(size_t)first * bs + o];
                for (int64_t r = seg[s] + 1; r < seg[s + 1]; ++r) {
                    int64_t q = order[r];
                    uint8_t bm = slot_mask[(size_t)q * bs + o];
                    apply_op(g->ptype[p], ops[p], A, (const uint8_t*)slot_data[p] + ((size_t)q * bs + o) * es, am & 1, bm & 1);
                    am |= bm;
                }
                if (O >= 0) {
                    uint8_t bm = old.mask[(size_t)O * bs + o];
                    apply_op(g->ptype[p], ops[p], A, &old.data[p][((size_t)O * bs + o) * es], am & 1, bm & 1);
                    am |= bm;
                }
                std::memcpy(g->at(p, P, o), A, es);
            }
            if (any_listed) {
                uint8_t am = 0;
                for (int64_t r = seg[s]; r < seg[s + 1]; ++r) am |= slot_mask[(size_t)order[r] * bs + o];
                if (O >= 0) am |= old.mask[(size_t)O * bs + o];
                g->mask[(size_t)P * bs + o] = am;
            }
        }
    }
}

// Flush of single-point inserts (the common insert<p>(coord) path).  Each
// point is one chunk slot whose mask is set at one offset only, so the chunk
// reduction above collapses to a per-point fold: the inserts of one point in
// insertion order, A = first, A = op(A, next), then A = op(A, old) when the
// point already exists; mask = OR.  Equivalence with sgo_flush_chunks is
// checked by the test suite.
void sgo_flush_points(void* h, int64_t n, const int64_t* lin, const void* const* vals, const uint8_t* pmask,
                      const int* ops) {
    Grid* g = (Grid*)h;
    if (n == 0) return;
    const int bs = g->bs;
    std::vector<int64_t> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return lin[a] < lin[b]; });
    std::vector<int64_t> ukeys;
    for (int64_t i = 0; i < n; ++i) {
        int64_t b = lin[order[i]] / bs;
        if (ukeys.empty() || ukeys.back() != b) ukeys.push_back(b);
    }
    std::vector<int64_t> merged, old_pos, new_pos, new_old;
    merged_layout(*g, ukeys, merged, old_pos, new_pos, new_old);
    relayout(*g, merged, old_pos);
    bool any_listed = false;
    for (int p = 0; p < g->nprop; ++p) any_listed |= ops[p] != OP_NONE;
    for (int64_t i = 0; i < n;) {
        int64_t j = i;
        while (j < n && lin[order[j]] == lin[order[i]]) ++j;
        int64_t key = lin[order[i]];
        int64_t P = std::lower_bound(g->keys.begin(), g->keys.end(), key / bs) - g->keys.begin();
        int o = (int)(key % bs);
        uint8_t oldm = g->mask[(size_t)P * bs + o];
        for (int p = 0; p < g->nprop; ++p) {
            if (ops[p] == OP_NONE) continue;
            int es = g->es(p);
            uint8_t A[8];
            std::memcpy(A, (const uint8_t*)vals[p] + (size_t)order[i] * es, es);
            uint8_t am = pmask ? pmask[order[i]] : 1;
            for (int64_t r = i + 1; r < j; ++r) {
                uint8_t bm = pmask ? pmask[order[r]] : 1;
                apply_op(g->ptype[p], ops[p], A, (const uint8_t*)vals[p] + (size_t)order[r] * es, am & 1, bm & 1);
                am |= bm;
            }
            apply_op(g->ptype[p], ops[p], A, g->at(p, P, o), am & 1, oldm & 1);
            std::memcpy(g->at(p, P, o), A, es);
        }
        if (any_listed) {
            uint8_t am = 0;
            for (int64_t r = i; r < j; ++r) am |= pmask ? pmask[order[r]] : 1;
            g->mask[(size_t)P * bs + o] = am | oldm;
        }
        i = j;
    }
}

// Neighbour table in the reference's nn_blocks format: data position of the
// neighbour chunk, the background position n when absent, -1 for the unused
// NNStar slots.
int sgo_find_neighbours(void* h, int kind, int64_t* out) {
    Grid* g = (Grid*)h;
    auto nn = find_neighbours(*g, kind);
    std::memcpy(out, nn.data(), nn.size() * 8);
    return nnn(*g, kind);
}

// tagBoundaries (SparseGridGpu_kernels.cuh:676-737): for every existing point
// set PADDING if one of its neighbours (NNStar faces, SparseGridGpu_ker_util.hpp:
// 141-157; NNFull 3^dim box, SparseGridGpu.hpp:200-228) does not exist, clear
// it otherwise.  Non-existing points are left alone.
void sgo_tag_boundaries(void* h, int kind) {
    Grid* g = (Grid*)h;
    auto nn = find_neighbours(*g, kind);
    std::vector<uint8_t> newmask = g->mask;
    std::vector<uint8_t> tile;
    for (int64_t i = 0; i < g->n(); ++i) {
        load_tile(*g, nn, kind, i, -1, tile);
        for (int o = 0; o < g->bs; ++o) {
            int lc[3] = {0, 0, 0};
            local_coord(*g, o, lc);
            int tc[3];
            for (int d = 0; d < g->dim; ++d) tc[d] = lc[d] + 1;
            uint8_t cur = tile[tile_index(*g, tc)];
            if (!(cur & 1)) continue;
            bool pad = false;
            if (kind == NN_STAR) {
                for (int d = 0; d < g->dim && !pad; ++d) {
                    for (int s = -1; s <= 1; s += 2) {
                        int nc[3] = {tc[0], tc[1], tc[2]};
                        nc[d] += s;
                        pad |= !(tile[tile_index(*g, nc)] & 1);
                    }
                }
            } else {
                int nb = g->dim == 3 ? 27 : 9;
                for (int q = 0; q < nb && !pad; ++q) {
                    int nc[3] = {tc[0], tc[1], tc[2]}, r = q;
                    for (int d = 0; d < g->dim; ++d) { nc[d] += r % 3 - 1; r /= 3; }
                    pad |= !(tile[tile_index(*g, nc)] & 1);
                }
            }
            newmask[(size_t)i * g->bs + o] = pad ? (uint8_t)(cur | 2) : (uint8_t)(cur & ~2);
        }
    }
    g->mask.swap(newmask);
}

// HeatStencil::stencil (src/SparseGridGpu/tests/utils/SparseGridGpu_util_test.cuh:
// 224-290) driven by applyStencilInPlace: active points get
//   lap = (float)(-2.0*dim*cur); lap += xm + xp; ... ; res = cur + dt*lap
// with the roundings nvcc gives that source: the double product -6*cur is
// exact, so its narrowing to float is a float multiply, which the default FMA
// contraction fuses with the first sum, lap = fma(-6, cur, xm + xp), and
// res = fma(dt, lap, cur) (the drop-in test compiles the reference's functor
// and checks this point by point).  Every other point of the destination
// chunk receives the tile value (its own value, or the background when its
// mask is 0): storeBlock writes the whole chunk (SparseGridGpu_ker.cuh:877-896).
void sgo_heat7(void* h, int src, int dst, float dt, const int64_t* box) {
    FtzScope ftz;
    Grid* g = (Grid*)h;
    auto nn = find_neighbours(*g, NN_STAR);
    std::vector<float> tile;
    std::vector<uint8_t> out(g->data[dst]);
    for (int64_t i = 0; i < g->n(); ++i) heat7_chunk(*g, nn, i, src, dt, box, tile, out);
    g->data[dst].swap(out);
}

// Gray-Scott written as a conv2_b user function (stencil_func_conv2_b,
// SparseGridGpu_kernels.cuh:383-451): only active points are written.  The
// Laplacian is assembled in HeatStencil's association order.  Update:
//   du = Du*lu - u*v*v + F*(1-u);  dv = Dv*lv + u*v*v - (F+k)*v
//   u' = u + dt*du;                v' = v + dt*dv
// evaluated as   uvv = (u*v)*v
//                du = fma(F, 1-u, fma(Du, lu, -uvv))
//                dv = fma(-(F+k), v, fma(Dv, lv, uvv))
//                u' = fma(dt, du, u);  v' = fma(dt, dv, v)
// with -(F+k) rounded to float once.
void sgo_gs7(void* h, int pu, int pv, int pu2, int pv2, float Du, float Dv, float F, float k, float dt,
             const int64_t* box) {
    FtzScope ftz;
    Grid* g = (Grid*)h;
    auto nn = find_neighbours(*g, NN_STAR);
    std::vector<float> tu, tv;
    std::vector<uint8_t> ou(g->data[pu2]), ov(g->data[pv2]);
    const float nfk = -(F + k);
    for (int64_t i = 0; i < g->n(); ++i) gs7_chunk(*g, nn, i, pu, pv, Du, Dv, F, nfk, dt, box, tu, tv, ou, ov);
    g->data[pu2].swap(ou);
    g->data[pv2].swap(ov);
}

// `steps` Gray-Scott / heat steps ping-ponging (pu, pv) -> (pu2, pv2) -> (pu, pv) ...,
// with the chunks of each step shared out over `threads` host threads.  Every
// chunk of a step reads only the step's source arrays and writes only its own
// part of the destination arrays, so the result is the same bits as the serial
// sgo_gs7 / sgo_heat7 calls, for any thread count.  Every thread sets FTZ|DAZ.
void sgo_gs7_steps(void* h, int pu, int pv, int pu2, int pv2, float Du, float Dv, float F, float k, float dt,
                   int steps, int threads) {
    Grid* g = (Grid*)h;
    auto nn = find_neighbours(*g, NN_STAR);
    const float nfk = -(F + k);
    int a0 = pu, a1 = pv, b0 = pu2, b1 = pv2;
    for (int s = 0; s < steps; ++s) {
        std::vector<uint8_t> ou(g->data[b0]), ov(g->data[b1]);
        for_chunks(g->n(), threads, [&](int64_t lo, int64_t hi) {
            std::vector<float> tu, tv;
            for (int64_t i = lo; i < hi; ++i) gs7_chunk(*g, nn, i, a0, a1, Du, Dv, F, nfk, dt, nullptr, tu, tv, ou, ov);
        });
        g->data[b0].swap(ou);
        g->data[b1].swap(ov);
        std::swap(a0, b0);
        std::swap(a1, b1);
    }
}

void sgo_heat7_steps(void* h, int src, int dst, float dt, int steps, int threads) {
    Grid* g = (Grid*)h;
    auto nn = find_neighbours(*g, NN_STAR);
    int a = src, b = dst;
    for (int s = 0; s < steps; ++s) {
        std::vector<uint8_t> out(g->data[b]);
        for_chunks(g->n(), threads, [&](int64_t lo, int64_t hi) {
            std::vector<float> tile;
            for (int64_t i = lo; i < hi; ++i) heat7_chunk(*g, nn, i, a, dt, nullptr, tile, out);
        });
        g->data[b].swap(out);
        std::swap(a, b);
    }
}

// Conv3x3x3 (src/SparseGridGpu/tests/SparseGridGpu_tests.cu:887-952) with an
// NNFull halo: tot = 0; for i,j,k: tot += tile[x+i-1][y+j-1][z+k-1]*c[i][j][k]
// (an FMA chain in i-major order); only active points are written.
void sgo_box27(void* h, int src, int dst, const float* coeff, const int64_t* box) {
    FtzScope ftz;
    Grid* g = (Grid*)h;
    auto nn = find_neighbours(*g, NN_FULL);
    std::vector<float> tile;
    std::vector<uint8_t> out(g->data[dst]);
    for (int64_t i = 0; i < g->n(); ++i) {
        load_tile(*g, nn, NN_FULL, i, src, tile);
        for (int o = 0; o < g->bs; ++o) {
            if (!active(cur_mask(*g, i, o, box))) continue;
            int lc[3] = {0, 0, 0}, tc[3] = {0, 0, 0};
            local_coord(*g, o, lc);
            for (int d = 0; d < 3; ++d) tc[d] = lc[d] + 1;
            float tot = 0.0f;
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b)
                    for (int c = 0; c < 3; ++c) {
                        int nc[3] = {tc[0] + a - 1, tc[1] + b - 1, tc[2] + c - 1};
                        tot = std::fmaf(tile[tile_index(*g, nc)], coeff[a * 9 + b * 3 + c], tot);
                    }
            std::memcpy(&out[((size_t)i * g->bs + o) * 4], &tot, 4);
        }
    }
    g->data[dst].swap(out);
}

// Conv3x3x3_noshared (src/SparseGridGpu/tests/SparseGridGpu_tests.cu:955-1010)
// applied by applyStencilInPlaceNoShared (SparseGridGpu_kernels.cuh:1096-1150)
// over the existing points: for an active point, tot += get(getNNPoint(key)) *
// coeff[i][j][k] with key = (k-1, j-1, i-1), i outermost (so i runs along z
// and k along x, the transpose of Conv3x3x3), contracted to an FMA.  The
// neighbour value is read from the chunk data as it is (no background
// substitution for non-existing points; an absent chunk is the background
// chunk, SparseGridGpu.hpp:269-291, getNNPoint SparseGridGpu_ker.cuh:297-327).
void sgo_box27_ns(void* h, int src, int dst, const float* coeff, const int64_t* box) {
    FtzScope ftz;
    Grid* g = (Grid*)h;
    auto nn = find_neighbours(*g, NN_FULL);
    const int e = g->edge, bs = g->bs;
    const float* in = (const float*)g->data[src].data();
    std::vector<uint8_t> out(g->data[dst]);
    for (int64_t c = 0; c < g->n(); ++c) {
        for (int o = 0; o < bs; ++o) {
            if (!active(cur_mask(*g, c, o, box))) continue;
            int lc[3] = {0, 0, 0};
            local_coord(*g, o, lc);
            float tot = 0.0f;
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j)
                    for (int k = 0; k < 3; ++k) {
                        const int q[3] = {lc[0] + k - 1, lc[1] + j - 1, lc[2] + i - 1};
                        int nidx = 0, off = 0;
                        for (int d = 2; d >= 0; --d) {
                            const int p = q[d] < 0 ? 0 : (q[d] >= e ? 2 : 1);
                            nidx = nidx * 3 + p;
                            off = off * e + (q[d] + (1 - p) * e);
                        }
                        const int64_t pos = nidx == 13 ? c : nn[(size_t)c * 27 + nidx];
                        tot = std::fmaf(in[(size_t)pos * bs + off], coeff[i * 9 + j * 3 + k], tot);
                    }
            std::memcpy(&out[((size_t)c * bs + o) * 4], &tot, 4);
        }
    }
    g->data[dst].swap(out);
}

// FP64 references for error statements: the same updates in double precision
// on caller-owned double fields laid out like the chunk data ((n+1)*bs, the
// background chunk last).  Active set and neighbourhoods come from the grid.
void sgo_heat7_f64(void* h, double* f_src, double* f_dst, double dt, double bck, int steps) {
    Grid* g = (Grid*)h;
    auto nn = find_neighbours(*g, NN_STAR);
    const int bs = g->bs, e = g->edge;
    double* a = f_src;
    double* b = f_dst;
    for (int s = 0; s < steps; ++s) {
        for (int64_t i = 0; i < g->n(); ++i) {
            for (int o = 0; o < bs; ++o) {
                uint8_t m = g->mask[(size_t)i * bs + o];
                double cur = m ? a[(size_t)i * bs + o] : bck;
                if (!active(m)) { b[(size_t)i * bs + o] = cur; continue; }
                int lc[3] = {0, 0, 0};
                local_coord(*g, o, lc);
                double lap = -2.0 * g->dim * cur;
                for (int d = 0; d < g->dim; ++d) {
                    for (int sgn = -1; sgn <= 1; sgn += 2) {
                        int nc[3] = {lc[0], lc[1], lc[2]};
                        nc[d] += sgn;
                        int64_t src = i;
                        if (nc[d] < 0 || nc[d] >= e) {
                            src = nn[(size_t)i * nnn(*g, NN_STAR) + 2 * d + (sgn > 0)];
                            nc[d] = (nc[d] + e) % e;
                        }
                        int off = 0, mm = 1;
                        for (int q = 0; q < g->dim; ++q) { off += nc[q] * mm; mm *= e; }
                        uint8_t nm = g->mask[(size_t)src * bs + off];
                        lap += nm ? a[(size_t)src * bs + off] : bck;
                    }
                }
                b[(size_t)i * bs + o] = cur + dt * lap;
            }
        }
        std::swap(a, b);
    }
    if (steps % 2 == 1) std::memcpy(f_src, f_dst, sizeof(double) * (size_t)(g->n() + 1) * bs);
    else if (a != f_src) std::memcpy(f_src, a, sizeof(double) * (size_t)(g->n() + 1) * bs);
}

void sgo_gs7_f64_mt(void* h, double* u, double* v, double* u2, double* v2, double Du, double Dv, double F,
                    double k, double dt, double bcku, double bckv, int steps, int threads);

void sgo_gs7_f64(void* h, double* u, double* v, double* u2, double* v2, double Du, double Dv, double F,
                 double k, double dt, double bcku, double bckv, int steps) {
    sgo_gs7_f64_mt(h, u, v, u2, v2, Du, Dv, F, k, dt, bcku, bckv, steps, 1);
}

// The same with the chunks of each step shared out over host threads (no FTZ: a double-precision
// reference keeps its subnormals).
void sgo_gs7_f64_mt(void* h, double* u, double* v, double* u2, double* v2, double Du, double Dv, double F,
                    double k, double dt, double bcku, double bckv, int steps, int threads) {
    Grid* g = (Grid*)h;
    auto nn = find_neighbours(*g, NN_STAR);
    const int bs = g->bs, e = g->edge, K = nnn(*g, NN_STAR);
    double *ua = u, *va = v, *ub = u2, *vb = v2;
    for (int s = 0; s < steps; ++s) {
      for_chunks_plain(g->n(), threads, [&](int64_t c0, int64_t c1) {
        for (int64_t i = c0; i < c1; ++i) {
            for (int o = 0; o < bs; ++o) {
                uint8_t m = g->mask[(size_t)i * bs + o];
                size_t idx = (size_t)i * bs + o;
                if (!active(m)) { ub[idx] = ua[idx]; vb[idx] = va[idx]; continue; }
                int lc[3] = {0, 0, 0};
                local_coord(*g, o, lc);
                double cu = ua[idx], cv = va[idx];
                double lu = -2.0 * g->dim * cu, lv = -2.0 * g->dim * cv;
                for (int d = 0; d < g->dim; ++d) {
                    for (int sgn = -1; sgn <= 1; sgn += 2) {
                        int nc[3] = {lc[0], lc[1], lc[2]};
                        nc[d] += sgn;
                        int64_t src = i;
                        if (nc[d] < 0 || nc[d] >= e) {
                            src = nn[(size_t)i * K + 2 * d + (sgn > 0)];
                            nc[d] = (nc[d] + e) % e;
                        }
                        int off = 0, mm = 1;
                        for (int q = 0; q < g->dim; ++q) { off += nc[q] * mm; mm *= e; }
                        uint8_t nm = g->mask[(size_t)src * bs + off];
                        lu += nm ? ua[(size_t)src * bs + off] : bcku;
                        lv += nm ? va[(size_t)src * bs + off] : bckv;
                    }
                }
                double uvv = cu * cv * cv;
                ub[idx] = cu + dt * (Du * lu - uvv + F * (1.0 - cu));
                vb[idx] = cv + dt * (Dv * lv + uvv - (F + k) * cv);
            }
        }
      });
        std::swap(ua, ub);
        std::swap(va, vb);
    }
    size_t tot = sizeof(double) * (size_t)(g->n() + 1) * bs;
    if (ua != u) { std::memcpy(u, ua, tot); std::memcpy(v, va, tot); }
}

// remove(box) + removePoints (src/SparseGridGpu/SparseGridGpu.hpp:3417-3489, 3528-3531;
// SparseGridGpu_kernels.cuh:1235-1340): every existing point inside any of the
// boxes gets mask byte 0; chunks stay.  The boxes are converted to unsigned int
// as the reference's Box<dim, unsigned int> kernels do, so a negative lower
// corner matches nothing and a negative upper corner matches everything above
// the lower one.  boxes: nb x {lo[3], hi[3]}, inclusive.
void sgo_remove_boxes(void* h, int64_t nb, const int64_t* boxes) {
    Grid* g = (Grid*)h;
    for (int64_t i = 0; i < g->n(); ++i) {
        for (int o = 0; o < g->bs; ++o) {
            uint8_t& m = g->mask[(size_t)i * g->bs + o];
            if (!(m & 1)) continue;
            int64_t c[3] = {0, 0, 0};
            inv_lin(*g, g->keys[i] * g->bs + o, c);
            for (int64_t k = 0; k < nb; ++k) {
                bool in = true;
                for (int d = 0; d < g->dim; ++d) {
                    const uint32_t lo = (uint32_t)boxes[k * 6 + d], hi = (uint32_t)boxes[k * 6 + 3 + d];
                    const uint32_t p = (uint32_t)c[d];
                    in = in && p >= lo && p <= hi;
                }
                if (in) m = 0;
            }
        }
    }
}

}  // extern "C"
