// CPU baseline: a restatement of openfpm_data's CPU sparse grid (sgrid_cpu)
// stencil path, used only as the timed CPU comparison and as a second
// cross-check of the oracle.  TEST / BENCHMARK INFRASTRUCTURE ONLY.
//
// Structure followed (the reference itself needs Boost and Vc, absent here):
//   * 16^3 chunks (default_chunking<3>, src/SparseGrid/SparseGridUtil.hpp:124-140)
//   * chunks found through a hash map from chunk coordinate to chunk index
//     (find_active_chunk / pre_insert, src/SparseGrid/SparseGrid.hpp:686-827;
//     the reference uses a tsl hopscotch map, this uses std::unordered_map)
//   * per chunk: the six face-neighbour chunks are resolved once, then rows
//     along x are swept, rows whose mask is all zero are skipped and the
//     store is masked (conv_impl<3>::conv_cross, src/SparseGrid/
//     SparseGrid_conv_opt.hpp:349-512).  Vc is unavailable, so the row loop
//     is scalar code left to the compiler's vectoriser.
//   * new chunks are filled with the background value, so a missing
//     neighbour reads the background.
// The reference path is single threaded; the OpenMP variant over chunks is an
// extension of this baseline and is reported separately.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <unordered_map>
#include <vector>

namespace {

constexpr int CE = 16;            // chunk edge
constexpr int CS = CE * CE * CE;  // points per chunk

struct CpuGrid {
    int64_t sz[3];
    int64_t nc[3];
    int nprop;
    std::vector<float> bck;
    std::unordered_map<int64_t, int32_t> map;
    std::vector<int64_t> ckey;
    std::vector<std::vector<float>> prop;  // (nchunks + 1) * CS, background chunk last
    std::vector<uint8_t> mask;
    std::vector<int32_t> nbr;               // 6 per chunk, background index when absent

    int32_t nchunks() const { return (int32_t)ckey.size(); }

    int32_t chunk_of(int64_t cx, int64_t cy, int64_t cz) const {
        if (cx < 0 || cy < 0 || cz < 0 || cx >= nc[0] || cy >= nc[1] || cz >= nc[2]) return nchunks();
        auto it = map.find((cz * nc[1] + cy) * nc[0] + cx);
        return it == map.end() ? nchunks() : it->second;
    }
};

void finalize(CpuGrid& g) {
    // background chunk at the end, then the per-chunk neighbour list
    const int32_t n = g.nchunks();
    for (int p = 0; p < g.nprop; ++p) {
        g.prop[p].resize((size_t)(n + 1) * CS);
        std::fill(g.prop[p].begin() + (size_t)n * CS, g.prop[p].end(), g.bck[p]);
    }
    g.mask.resize((size_t)(n + 1) * CS);
    std::fill(g.mask.begin() + (size_t)n * CS, g.mask.end(), 0);
    g.nbr.assign((size_t)n * 6, n);
    for (int32_t c = 0; c < n; ++c) {
        int64_t k = g.ckey[c];
        int64_t cx = k % g.nc[0], cy = (k / g.nc[0]) % g.nc[1], cz = k / (g.nc[0] * g.nc[1]);
        g.nbr[c * 6 + 0] = g.chunk_of(cx - 1, cy, cz);
        g.nbr[c * 6 + 1] = g.chunk_of(cx + 1, cy, cz);
        g.nbr[c * 6 + 2] = g.chunk_of(cx, cy - 1, cz);
        g.nbr[c * 6 + 3] = g.chunk_of(cx, cy + 1, cz);
        g.nbr[c * 6 + 4] = g.chunk_of(cx, cy, cz - 1);
        g.nbr[c * 6 + 5] = g.chunk_of(cx, cy, cz + 1);
    }
}

// Neighbour value along one axis, taken from the adjacent chunk across a
// chunk face (the offset_jump logic of conv_cross).
template <int AX, int DIR>
inline float nb(const float* base, const float* const* nbase, int x, int y, int z) {
    int c[3] = {x, y, z};
    c[AX] += DIR;
    if (c[AX] < 0 || c[AX] >= CE) {
        c[AX] = (c[AX] + CE) % CE;
        return nbase[2 * AX + (DIR > 0)][c[0] + CE * c[1] + CE * CE * c[2]];
    }
    return base[c[0] + CE * c[1] + CE * CE * c[2]];
}

}  // namespace

extern "C" {

void* cpub_create(const int64_t* size, int nprop, const float* bck) {
    CpuGrid* g = new CpuGrid();
    for (int d = 0; d < 3; ++d) {
        g->sz[d] = size[d];
        g->nc[d] = (size[d] + CE - 1) / CE;
    }
    g->nprop = nprop;
    g->bck.assign(bck, bck + nprop);
    g->prop.resize(nprop);
    finalize(*g);
    return g;
}

void cpub_destroy(void* h) { delete (CpuGrid*)h; }

int32_t cpub_nchunks(void* h) { return ((CpuGrid*)h)->nchunks(); }

// Insert points (x,y,z int64 triples) with one float value per property.
void cpub_insert(void* h, int64_t n, const int64_t* coords, const float* const* vals) {
    CpuGrid* g = (CpuGrid*)h;
    const int32_t n0 = g->nchunks();
    // drop the background chunk while inserting
    for (int p = 0; p < g->nprop; ++p) g->prop[p].resize((size_t)n0 * CS);
    g->mask.resize((size_t)n0 * CS);
    for (int64_t i = 0; i < n; ++i) {
        int64_t x = coords[3 * i], y = coords[3 * i + 1], z = coords[3 * i + 2];
        int64_t key = ((z / CE) * g->nc[1] + (y / CE)) * g->nc[0] + (x / CE);
        auto it = g->map.find(key);
        int32_t c;
        if (it == g->map.end()) {
            c = g->nchunks();
            g->map.emplace(key, c);
            g->ckey.push_back(key);
            for (int p = 0; p < g->nprop; ++p) g->prop[p].resize((size_t)(c + 1) * CS, g->bck[p]);
            g->mask.resize((size_t)(c + 1) * CS, 0);
        } else {
            c = it->second;
        }
        size_t off = (size_t)c * CS + (x % CE) + CE * (y % CE) + CE * CE * (z % CE);
        for (int p = 0; p < g->nprop; ++p) g->prop[p][off] = vals[p][i];
        g->mask[off] = 1;
    }
    finalize(*g);
}

// Read values back (background where the point does not exist).
void cpub_get(void* h, int64_t n, const int64_t* coords, int p, float* out) {
    CpuGrid* g = (CpuGrid*)h;
    for (int64_t i = 0; i < n; ++i) {
        int64_t x = coords[3 * i], y = coords[3 * i + 1], z = coords[3 * i + 2];
        int32_t c = g->chunk_of(x / CE, y / CE, z / CE);
        size_t off = (size_t)c * CS + (x % CE) + CE * (y % CE) + CE * CE * (z % CE);
        out[i] = g->mask[off] ? g->prop[p][off] : g->bck[p];
    }
}

// `steps` heat updates u <- u + dt*lap(u), ping-ponging between properties
// src and dst.  Returns the property holding the result.
int cpub_heat(void* h, int src, int dst, float dt, int steps, int nthreads) {
    CpuGrid* g = (CpuGrid*)h;
    const int32_t n = g->nchunks();
    for (int s = 0; s < steps; ++s) {
        const float* in = g->prop[src].data();
        float* out = g->prop[dst].data();
        const uint8_t* mk = g->mask.data();
#pragma omp parallel for schedule(static) num_threads(nthreads)
        for (int32_t c = 0; c < n; ++c) {
            const float* base = in + (size_t)c * CS;
            const float* nbase[6];
            for (int q = 0; q < 6; ++q) nbase[q] = in + (size_t)g->nbr[c * 6 + q] * CS;
            const uint8_t* m = mk + (size_t)c * CS;
            float* o = out + (size_t)c * CS;
            for (int z = 0; z < CE; ++z)
                for (int y = 0; y < CE; ++y) {
                    const int r = CE * y + CE * CE * z;
                    uint64_t w0, w1;
                    std::memcpy(&w0, m + r, 8);
                    std::memcpy(&w1, m + r + 8, 8);
                    if ((w0 | w1) == 0) continue;
                    for (int x = 0; x < CE; ++x) {
                        if (!m[r + x]) continue;
                        float cur = base[r + x];
                        float lap = -6.0f * cur;
                        lap += nb<0, -1>(base, nbase, x, y, z) + nb<0, 1>(base, nbase, x, y, z);
                        lap += nb<1, -1>(base, nbase, x, y, z) + nb<1, 1>(base, nbase, x, y, z);
                        lap += nb<2, -1>(base, nbase, x, y, z) + nb<2, 1>(base, nbase, x, y, z);
                        o[r + x] = cur + dt * lap;
                    }
                }
        }
        std::swap(src, dst);
    }
    return src;
}

// `steps` Gray-Scott updates (same formula as the GPU path); properties
// (u, v) -> (u2, v2) and back.  Returns 0 when the result is in (u, v), 1 when
// it is in (u2, v2).
int cpub_gs(void* h, int pu, int pv, int pu2, int pv2, float Du, float Dv, float F, float k, float dt, int steps,
            int nthreads) {
    CpuGrid* g = (CpuGrid*)h;
    const int32_t n = g->nchunks();
    const float nfk = -(F + k);
    for (int s = 0; s < steps; ++s) {
        const float* iu = g->prop[pu].data();
        const float* iv = g->prop[pv].data();
        float* ou = g->prop[pu2].data();
        float* ov = g->prop[pv2].data();
        const uint8_t* mk = g->mask.data();
#pragma omp parallel for schedule(static) num_threads(nthreads)
        for (int32_t c = 0; c < n; ++c) {
            const float* bu = iu + (size_t)c * CS;
            const float* bv = iv + (size_t)c * CS;
            const float *nu[6], *nv[6];
            for (int q = 0; q < 6; ++q) {
                nu[q] = iu + (size_t)g->nbr[c * 6 + q] * CS;
                nv[q] = iv + (size_t)g->nbr[c * 6 + q] * CS;
            }
            const uint8_t* m = mk + (size_t)c * CS;
            float* pu_o = ou + (size_t)c * CS;
            float* pv_o = ov + (size_t)c * CS;
            for (int z = 0; z < CE; ++z)
                for (int y = 0; y < CE; ++y) {
                    const int r = CE * y + CE * CE * z;
                    uint64_t w0, w1;
                    std::memcpy(&w0, m + r, 8);
                    std::memcpy(&w1, m + r + 8, 8);
                    if ((w0 | w1) == 0) continue;
                    for (int x = 0; x < CE; ++x) {
                        if (!m[r + x]) continue;
                        float u = bu[r + x], v = bv[r + x];
                        float lu = -6.0f * u, lv = -6.0f * v;
                        lu += nb<0, -1>(bu, nu, x, y, z) + nb<0, 1>(bu, nu, x, y, z);
                        lu += nb<1, -1>(bu, nu, x, y, z) + nb<1, 1>(bu, nu, x, y, z);
                        lu += nb<2, -1>(bu, nu, x, y, z) + nb<2, 1>(bu, nu, x, y, z);
                        lv += nb<0, -1>(bv, nv, x, y, z) + nb<0, 1>(bv, nv, x, y, z);
                        lv += nb<1, -1>(bv, nv, x, y, z) + nb<1, 1>(bv, nv, x, y, z);
                        lv += nb<2, -1>(bv, nv, x, y, z) + nb<2, 1>(bv, nv, x, y, z);
                        float uvv = (u * v) * v;
                        float du = std::fmaf(F, 1.0f - u, std::fmaf(Du, lu, -uvv));
                        float dv = std::fmaf(nfk, v, std::fmaf(Dv, lv, uvv));
                        pu_o[r + x] = std::fmaf(dt, du, u);
                        pv_o[r + x] = std::fmaf(dt, dv, v);
                    }
                }
        }
        std::swap(pu, pu2);
        std::swap(pv, pv2);
    }
    return steps % 2;
}

}  // extern "C"
