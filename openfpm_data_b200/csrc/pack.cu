// Packing of sub-boxes of a grid for ghost exchange, and unpacking.
//
// Format of one packed box, the reference's (SparseGridGpu.hpp:2984-3040
// packCalculate, 3244-3300 pack, SparseGridGpu_kernels.cuh:1658-1697
// pack_data), with indexT = int64:
//   uint64 n_cnk;  int32 start[3];  int32 size[3];
//   int64  chunk_id[n_cnk]                 (the chunks holding packed points, index order)
//   uint32 scan[n_cnk + 1]                 (first packed point of each chunk; scan[n_cnk] = n_pnt)
//   data: for each packed property, n_pnt elements of its type, back to back
//   int16  offset[n_pnt]                   (the point's offset inside its chunk)
//   uint8  mask[n_pnt]
// where the scan, the data block, the offsets and the masks are each padded
// to a multiple of 8 bytes.  Packed points are the existing points inside the
// inclusive box.  Inside a chunk the reference orders them by a shared-memory
// atomic counter (any order); here they are in offset order.
//
// Unpacking stages the points of every box of a buffer as inserts at their
// coordinates plus a shift (the caller then flushes with the reduction it
// wants, e.g. sRight_ to overwrite): the unpack-then-merge step of the
// reference's ghost exchange (unpack 3665-3750 + removeAddUnpackFinalize).
#include <cstring>
#include <vector>

#include "common.cuh"
#include "internal.h"

namespace sgb {

__host__ __device__ inline int64_t pad8(int64_t b) { return (b + 7) & ~(int64_t)7; }

struct PackLayout {
    int64_t n_cnk, n_pnt;
    int64_t off_ids, off_scan, off_data, off_offs, off_mask, bytes, data_bytes;
    int64_t prop_off[kMaxProps];
};

__host__ __device__ inline PackLayout layout_of(int64_t n_cnk, int64_t n_pnt, int np, const int* es) {
    PackLayout L{};
    L.n_cnk = n_cnk;
    L.n_pnt = n_pnt;
    int64_t o = 8 + 2 * 3 * 4;
    L.off_ids = o;
    o += 8 * n_cnk;
    L.off_scan = o;
    o += pad8(4 * (n_cnk + 1));
    L.off_data = o;
    int64_t d = 0;
    for (int p = 0; p < np; ++p) {
        L.prop_off[p] = d;
        d += n_pnt * es[p];
    }
    L.data_bytes = d;
    o += pad8(d);
    L.off_offs = o;
    o += pad8(2 * n_pnt);
    L.off_mask = o;
    o += pad8(n_pnt);
    L.bytes = o;
    return L;
}

__device__ __forceinline__ void origin_of(const Geometry& geo, int64_t key, int64_t* o) { chunk_origin(geo, key, o); }

struct Box6 {
    int64_t b[6];
};

__device__ __forceinline__ bool inside6(const Box6& bx, int64_t x, int64_t y, int64_t z) {
    return x >= bx.b[0] && x <= bx.b[3] && y >= bx.b[1] && y <= bx.b[4] && z >= bx.b[2] && z <= bx.b[5];
}

// Does the chunk at origin o (edge e) meet the box?
__device__ __forceinline__ bool chunk_meets(const Box6& bx, const int64_t* o, int e) {
    return o[0] <= bx.b[3] && o[0] + e - 1 >= bx.b[0] && o[1] <= bx.b[4] && o[1] + e - 1 >= bx.b[1] &&
           o[2] <= bx.b[5] && o[2] + e - 1 >= bx.b[2];
}

// Chunk-coordinate bounds of a box: the chunk at block coordinate c (origin c * e) meets the box
// exactly when lo <= c <= hi in every dimension, lo = floor(low / e), hi = floor(high / e) --
// the same test as chunk_meets, without the origin.  Each CTA stages the bounds of the first
// kStageBoxes boxes in shared memory.
constexpr int kStageBoxes = 64;
struct CBounds {
    int64_t lo[3], hi[3];
};
__device__ __forceinline__ int64_t floor_div(int64_t a, int64_t b) {  // b > 0
    const int64_t q = a / b;
    return (a % b != 0 && a < 0) ? q - 1 : q;
}
__device__ __forceinline__ CBounds cbounds_of(const Box6& bx, int e) {
    CBounds cb;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        cb.lo[d] = floor_div(bx.b[d], e);
        cb.hi[d] = floor_div(bx.b[d + 3], e);
    }
    return cb;
}
__device__ __forceinline__ bool meets_cb(const CBounds& cb, const int64_t* bc) {
    return bc[0] >= cb.lo[0] && bc[0] <= cb.hi[0] && bc[1] >= cb.lo[1] && bc[1] <= cb.hi[1] && bc[2] >= cb.lo[2] &&
           bc[2] <= cb.hi[2];
}

// Counts for all boxes in one pass: cnt[k * (n + 1) + c] = existing points of
// chunk c inside box k, flg[...] = (cnt != 0).  Both arrays are zeroed by the
// caller (row entries c = n stay 0 so that one scan over all rows gives every
// box's offsets).  One warp per chunk; boxes the chunk does not meet cost no
// mask read.
__global__ void k_pack_count(const int64_t* __restrict__ keys, int64_t n, Geometry geo, const uint8_t* __restrict__ mask,
                             const Box6* __restrict__ boxes, int nb, uint32_t* cnt, uint32_t* flg) {
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int bs = geo.bs, e = geo.edge;
    __shared__ CBounds sb[kStageBoxes];
    for (int k = threadIdx.x; k < nb && k < kStageBoxes; k += blockDim.x) sb[k] = cbounds_of(boxes[k], e);
    __syncthreads();
    for (int64_t c = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; c < n; c += nw) {
        int64_t bc[3], o[3];
        block_coords(geo, keys[c], bc);
        for (int d = 0; d < 3; ++d) o[d] = bc[d] * e;
        for (int k = 0; k < nb; ++k) {
            if (k < kStageBoxes ? !meets_cb(sb[k], bc) : !chunk_meets(boxes[k], o, e)) continue;  // uniform
            const Box6 bx = boxes[k];
            uint8_t mv[16];  // the lane's mask bytes, all loads in flight at once (bs <= 512)
#pragma unroll
            for (int i = 0; i < 16; ++i) mv[i] = lane + 32 * i < bs ? mask[c * bs + lane + 32 * i] : 0;
            uint32_t t = 0;
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                if (32 * i >= bs) break;
                const int pt = lane + 32 * i;
                const bool in = (mv[i] & 1) && inside6(bx, o[0] + pt % e, o[1] + (pt / e) % e, o[2] + pt / (e * e));
                t += __popc(__ballot_sync(0xffffffffu, in));
            }
            if (lane == 0 && t) {
                cnt[(int64_t)k * (n + 1) + c] = t;
                flg[(int64_t)k * (n + 1) + c] = 1;
            }
        }
    }
}

// Row starts of the two scans (box k's first point / chunk) for k = 0..nb.
__global__ void k_pack_rows(const uint32_t* __restrict__ scnt, const uint32_t* __restrict__ sflg, int64_t n, int nb,
                            uint32_t* out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k > nb) return;
    out[2 * k] = scnt[(int64_t)k * (n + 1)];
    out[2 * k + 1] = sflg[(int64_t)k * (n + 1)];
}

struct PackProps {
    const unsigned char* src[kMaxProps];
    int es[kMaxProps];
    int wide[kMaxProps];  // 1: the property's packed block is aligned to its element size
    int np;
};

// One packed box: its place in the output, its layout, its box.
struct PackBox {
    Box6 box;
    int64_t base;  // byte offset of the box in the output
    PackLayout L;
    uint32_t pnt0, cnk0;  // the box's row starts in the scans
};

template <typename T>
__device__ __forceinline__ void copy_elem(unsigned char* d, const unsigned char* s) {
    *reinterpret_cast<T*>(d) = *reinterpret_cast<const T*>(s);
}

__global__ void k_pack_emit(const int64_t* __restrict__ keys, int64_t n, Geometry geo, const uint8_t* __restrict__ mask,
                            const PackBox* __restrict__ pbs, int nb, const uint32_t* __restrict__ scnt,
                            const uint32_t* __restrict__ sflg, PackProps pp, unsigned char* out) {
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int bs = geo.bs, e = geo.edge;
    __shared__ CBounds sb[kStageBoxes];
    for (int k = threadIdx.x; k < nb && k < kStageBoxes; k += blockDim.x) sb[k] = cbounds_of(pbs[k].box, e);
    __syncthreads();
    for (int64_t c = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; c < n; c += nw) {
        const int64_t key = keys[c];
        int64_t bc[3], o[3];
        block_coords(geo, key, bc);
        for (int d = 0; d < 3; ++d) o[d] = bc[d] * e;
        for (int k = 0; k < nb; ++k) {
            // uniform over the warp; no scan read for a box the chunk misses
            if (k < kStageBoxes ? !meets_cb(sb[k], bc) : !chunk_meets(pbs[k].box, o, e)) continue;
            const PackBox& P = pbs[k];
            const Box6 bx = P.box;
            const int64_t r = (int64_t)k * (n + 1) + c;
            uint32_t base = scnt[r];
            if (scnt[r + 1] == base) continue;  // no packed point of box k here (uniform)
            unsigned char* b = out + P.base;
            base -= P.pnt0;
            const uint32_t slot = sflg[r] - P.cnk0;
            if (lane == 0) {
                reinterpret_cast<int64_t*>(b + P.L.off_ids)[slot] = key;
                reinterpret_cast<uint32_t*>(b + P.L.off_scan)[slot] = base;
            }
            int16_t* offs = reinterpret_cast<int16_t*>(b + P.L.off_offs);
            uint8_t* msk = b + P.L.off_mask;
            uint8_t mv[16];  // the lane's mask bytes, all loads in flight at once (bs <= 512)
#pragma unroll
            for (int i = 0; i < 16; ++i) mv[i] = lane + 32 * i < bs ? mask[c * bs + lane + 32 * i] : 0;
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                if (32 * i >= bs) break;
                const int pt = lane + 32 * i;
                const uint8_t m = mv[i];
                const bool in = (m & 1) && inside6(bx, o[0] + pt % e, o[1] + (pt / e) % e, o[2] + pt / (e * e));
                const unsigned bal = __ballot_sync(0xffffffffu, in);
                if (in) {
                    const int64_t j = base + __popc(bal & lanemask_lt());
                    const int64_t idx = c * bs + pt;
                    for (int p = 0; p < pp.np; ++p) {
                        const int es = pp.es[p];
                        unsigned char* d = b + P.L.off_data + P.L.prop_off[p] + j * es;
                        const unsigned char* sp = pp.src[p] + idx * es;
                        if (pp.wide[p] && es == 4) copy_elem<uint32_t>(d, sp);
                        else if (pp.wide[p] && es == 8) copy_elem<uint64_t>(d, sp);
                        else
                            for (int q = 0; q < es; ++q) d[q] = sp[q];
                    }
                    offs[j] = (int16_t)pt;
                    msk[j] = m;
                }
                base += __popc(bal);
            }
        }
    }
}

// Per box: the header, scan[n_cnk] = n_pnt, and zeros in the padding tails.
__global__ void k_pack_finish(const PackBox* __restrict__ pbs, int nb, int32_t sx, int32_t sy, int32_t sz,
                              unsigned char* out) {
    const int k = blockIdx.x;
    if (k >= nb) return;
    const PackBox& P = pbs[k];
    unsigned char* b = out + P.base;
    const PackLayout& L = P.L;
    const int t = threadIdx.x;
    if (t == 0) {
        *reinterpret_cast<uint64_t*>(b) = (uint64_t)L.n_cnk;
        int32_t* h = reinterpret_cast<int32_t*>(b + 8);
        h[0] = (int32_t)P.box.b[0];
        h[1] = (int32_t)P.box.b[1];
        h[2] = (int32_t)P.box.b[2];
        h[3] = sx;
        h[4] = sy;
        h[5] = sz;
        reinterpret_cast<uint32_t*>(b + L.off_scan)[L.n_cnk] = (uint32_t)L.n_pnt;
    }
    // tails: [end of section, next section) for scan, data, offsets, masks
    const int64_t ends[4] = {L.off_scan + 4 * (L.n_cnk + 1), L.off_data + L.data_bytes, L.off_offs + 2 * L.n_pnt,
                             L.off_mask + L.n_pnt};
    const int64_t next[4] = {L.off_data, L.off_offs, L.off_mask, L.bytes};
    if (t < 32) {
        const int s = t >> 3, q = t & 7;
        if (ends[s] + q < next[s]) b[ends[s] + q] = 0;
    }
}

struct UnpackDst {
    unsigned char* p[kMaxProps];  // staged values of the k-th packed property
};

// Staged inserts of the packed points of one box at their coordinates + shift.
__global__ void k_unpack_stage(const unsigned char* __restrict__ buf, PackLayout L, Geometry src_geo, Geometry dst_geo,
                               int64_t sx, int64_t sy, int64_t sz, int64_t* out_lin, PackProps pp, UnpackDst dst,
                               unsigned* err) {
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= L.n_pnt) return;
    const int64_t* ids = reinterpret_cast<const int64_t*>(buf + L.off_ids);
    const uint32_t* scan = reinterpret_cast<const uint32_t*>(buf + L.off_scan);
    const int16_t* offs = reinterpret_cast<const int16_t*>(buf + L.off_offs);
    // the chunk of point j: the last c with scan[c] <= j
    int64_t lo = 0, hi = L.n_cnk;
    while (hi - lo > 1) {
        const int64_t mid = (lo + hi) >> 1;
        if (scan[mid] <= (uint32_t)j) lo = mid;
        else hi = mid;
    }
    int64_t o[3];
    origin_of(src_geo, ids[lo], o);
    const int e = src_geo.edge, pt = offs[j];
    const int64_t c[3] = {o[0] + pt % e + sx, o[1] + (pt / e) % e + sy, o[2] + pt / (e * e) + sz};
    bool ok = pt >= 0 && pt < src_geo.bs;
    for (int d = 0; d < 3; ++d) ok = ok && c[d] >= 0 && c[d] < dst_geo.size[d];
    int64_t lin = -1;
    if (ok) {
        int64_t b, l;
        point_key(dst_geo, c, &b, &l);
        lin = b * dst_geo.bs + l;
    } else {
        atomicOr(err, kErrOutOfDomain);
    }
    out_lin[j] = lin;
    for (int p = 0; p < pp.np; ++p) {
        const int es = pp.es[p];
        const unsigned char* s = buf + L.off_data + L.prop_off[p] + j * es;
        for (int b = 0; b < es; ++b) dst.p[p][j * es + b] = s[b];
    }
}

// One packed box of a buffer, as found by k_unpack_walk.
struct UnpackBox {
    int64_t pos;       // byte offset of the box in the buffer
    int64_t n_cnk, n_pnt;
    int64_t start[3];  // packed box lower corner
    int64_t size[3];   // packing grid size
    int64_t pnt0;      // points of the boxes before this one
    int64_t shift[3];  // destination - packed coordinates
    int32_t bad;       // 1: the header does not fit the buffer
};

struct ElemSizes {
    int es[kMaxProps];
    int np;
};

// Walk the headers of nb packed boxes (one thread: each box's place follows
// from the sizes of the boxes before it).
__global__ void k_unpack_walk(const unsigned char* __restrict__ buf, int64_t nbytes, int nb, ElemSizes es,
                              UnpackBox* out) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    int64_t pos = 0, pts = 0;
    for (int k = 0; k < nb; ++k) {
        UnpackBox B{};
        B.pos = pos;
        B.pnt0 = pts;
        B.bad = 1;
        if (nbytes - pos >= 40) {
            const uint64_t nc = *reinterpret_cast<const uint64_t*>(buf + pos);
            if (nc <= (uint64_t)(nbytes - pos - 36) / 12) {
                const int32_t* h = reinterpret_cast<const int32_t*>(buf + pos + 8);
                const uint32_t np_ = *reinterpret_cast<const uint32_t*>(buf + pos + 32 + 12 * (int64_t)nc);
                const PackLayout L = layout_of((int64_t)nc, np_, es.np, es.es);
                bool ok = L.bytes <= nbytes - pos && !(nc == 0 && np_ != 0);
                for (int d = 0; d < 3; ++d) ok = ok && h[3 + d] >= 1;
                if (ok) {
                    B.n_cnk = (int64_t)nc;
                    B.n_pnt = np_;
                    for (int d = 0; d < 3; ++d) {
                        B.start[d] = h[d];
                        B.size[d] = h[3 + d];
                    }
                    B.bad = 0;
                    pos += L.bytes;
                    pts += np_;
                }
            }
        }
        out[k] = B;
        if (B.bad) {
            for (int j = k + 1; j < nb; ++j) out[j].bad = 1;
            return;
        }
    }
}

// Staged inserts of every packed point of the boxes: thread j finds its box
// by the point offsets, then proceeds as k_unpack_stage.
__global__ void k_unpack_stage_all(const unsigned char* __restrict__ buf, const UnpackBox* __restrict__ boxes, int nb,
                                   int64_t total, ElemSizes es, Geometry dst_geo, int64_t* out_lin, UnpackDst dst,
                                   unsigned* err) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= total) return;
    int lo = 0, hi = nb;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (boxes[mid].pnt0 <= t) lo = mid;
        else hi = mid;
    }
    const UnpackBox& B = boxes[lo];
    const PackLayout L = layout_of(B.n_cnk, B.n_pnt, es.np, es.es);
    const int64_t j = t - B.pnt0;
    const unsigned char* b = buf + B.pos;
    const int64_t* ids = reinterpret_cast<const int64_t*>(b + L.off_ids);
    const uint32_t* scan = reinterpret_cast<const uint32_t*>(b + L.off_scan);
    const int16_t* offs = reinterpret_cast<const int16_t*>(b + L.off_offs);
    int64_t clo = 0, chi = L.n_cnk;
    while (chi - clo > 1) {
        const int64_t mid = (clo + chi) >> 1;
        if (scan[mid] <= (uint32_t)j) clo = mid;
        else chi = mid;
    }
    Geometry src = dst_geo;
    for (int d = 0; d < 3; ++d) {
        src.size[d] = B.size[d];
        src.bsz[d] = (B.size[d] + src.edge - 1) / src.edge;
    }
    int64_t o[3];
    origin_of(src, ids[clo], o);
    const int e = src.edge, pt = offs[j];
    const int64_t c[3] = {o[0] + pt % e + B.shift[0], o[1] + (pt / e) % e + B.shift[1],
                          o[2] + pt / (e * e) + B.shift[2]};
    bool ok = pt >= 0 && pt < src.bs;
    for (int d = 0; d < 3; ++d) ok = ok && c[d] >= 0 && c[d] < dst_geo.size[d];
    int64_t lin = -1;
    if (ok) {
        int64_t kb, kl;
        point_key(dst_geo, c, &kb, &kl);
        lin = kb * dst_geo.bs + kl;
    } else {
        atomicOr(err, kErrOutOfDomain);
    }
    out_lin[t] = lin;
    for (int p = 0; p < es.np; ++p) {
        const int sz = es.es[p];
        const unsigned char* sp = b + L.off_data + L.prop_off[p] + j * sz;
        for (int q = 0; q < sz; ++q) dst.p[p][t * sz + q] = sp[q];
    }
}

static unsigned wgrid(const sgb_grid* g, int64_t n) {
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>((int64_t)g->num_sms * 8, (n + 7) / 8));
}

// The counting pass over all boxes: row starts of the point and chunk scans
// to rows[2 * (nb + 1)] (host), scans in scratch[2] / scratch[4].
static int pack_counts(sgb_grid* g, int64_t nboxes, const int64_t* boxes_host, std::vector<uint32_t>& rows,
                       cudaStream_t s) {
    const int64_t n = g->n;
    const int64_t len = nboxes * (n + 1);  // rows of n + 1 entries; the scans' totals land at [len]
    rows.assign(2 * (nboxes + 1), 0);
    if (nboxes == 0 || n == 0) return SGB_OK;
    if (len >= (int64_t(1) << 31)) {
        set_error("too many boxes x chunks in one pack call");
        return SGB_ERANGE;
    }
    SGB_TRY(g->scratch[0].ensure((size_t)nboxes * sizeof(Box6)));
    for (int k = 1; k <= 4; ++k) SGB_TRY(g->scratch[k].ensure((size_t)(len + 1) * 4 + 16));
    const size_t hb = std::max<size_t>((size_t)nboxes * sizeof(Box6), rows.size() * 4);
    SGB_TRY(g->hscratch.ensure(hb));
    std::memcpy(g->hscratch.p, boxes_host, (size_t)nboxes * sizeof(Box6));
    SGB_CUDA(cudaMemcpyAsync(g->scratch[0].p, g->hscratch.p, (size_t)nboxes * sizeof(Box6), cudaMemcpyHostToDevice, s));
    uint32_t *cnt = g->scratch[1].as<uint32_t>(), *scnt = g->scratch[2].as<uint32_t>(),
             *flg = g->scratch[3].as<uint32_t>(), *sflg = g->scratch[4].as<uint32_t>();
    SGB_CUDA(cudaMemsetAsync(cnt, 0, (size_t)len * 4, s));
    SGB_CUDA(cudaMemsetAsync(flg, 0, (size_t)len * 4, s));
    k_pack_count<<<wgrid(g, n), 256, 0, s>>>(g->keys.as<int64_t>(), n, g->geo, g->mask.as<uint8_t>(),
                                             g->scratch[0].as<Box6>(), (int)nboxes, cnt, flg);
    SGB_CUDA(cudaGetLastError());
    SGB_TRY(scan_exclusive_u32(cnt, scnt, len, scnt + len, &g->scratch[6], s));
    SGB_TRY(scan_exclusive_u32(flg, sflg, len, sflg + len, &g->scratch[6], s));
    // the row starts go through scratch[1], which the scans no longer need
    k_pack_rows<<<(unsigned)((nboxes + 1 + 127) / 128), 128, 0, s>>>(scnt, sflg, n, (int)nboxes, cnt);
    SGB_CUDA(cudaGetLastError());
    SGB_CUDA(cudaMemcpyAsync(g->hscratch.p, cnt, rows.size() * 4, cudaMemcpyDeviceToHost, s));
    SGB_CUDA(cudaStreamSynchronize(s));
    std::memcpy(rows.data(), g->hscratch.p, rows.size() * 4);
    return SGB_OK;
}

static int check_props(const sgb_grid* g, int nprops, const int* props, int* es) {
    if (nprops < 0 || nprops > kMaxProps || (nprops > 0 && !props)) return SGB_EINVAL;
    for (int k = 0; k < nprops; ++k) {
        if (props[k] < 0 || props[k] >= g->nprop) return SGB_EINVAL;
        es[k] = elem_size(g->ptype[props[k]]);
    }
    return SGB_OK;
}

}  // namespace sgb

using namespace sgb;

extern "C" int sgb_pack_request(sgb_grid* g, int64_t nboxes, const int64_t* boxes_host, int nprops, const int* props,
                                int64_t* bytes_host, sgb_stream stream) {
    if (!g || nboxes < 0 || (nboxes > 0 && (!boxes_host || !bytes_host))) return SGB_EINVAL;
    if (g->geo.dim != 3) return SGB_ENOTSUP;
    int es[kMaxProps];
    SGB_TRY(check_props(g, nprops, props, es));
    std::vector<uint32_t> rows;
    SGB_TRY(pack_counts(g, nboxes, boxes_host, rows, (cudaStream_t)stream));
    for (int64_t k = 0; k < nboxes; ++k)
        bytes_host[k] = layout_of(rows[2 * k + 3] - rows[2 * k + 1], rows[2 * k + 2] - rows[2 * k], nprops, es).bytes;
    return SGB_OK;
}

extern "C" int sgb_pack(sgb_grid* g, int64_t nboxes, const int64_t* boxes_host, int nprops, const int* props,
                        void* out_dev, int64_t capacity, int64_t* bytes_written, sgb_stream stream) {
    if (!g || nboxes < 0 || (nboxes > 0 && (!boxes_host || !out_dev)) || !bytes_written) return SGB_EINVAL;
    if (g->geo.dim != 3) return SGB_ENOTSUP;
    if ((uintptr_t)out_dev % 8 != 0) {
        set_error("the pack buffer must be 8-byte aligned");
        return SGB_EINVAL;
    }
    int es[kMaxProps];
    SGB_TRY(check_props(g, nprops, props, es));
    *bytes_written = 0;
    if (nboxes == 0) return SGB_OK;
    cudaStream_t s = (cudaStream_t)stream;
    std::vector<uint32_t> rows;
    SGB_TRY(pack_counts(g, nboxes, boxes_host, rows, s));
    std::vector<PackBox> pb((size_t)nboxes);
    int64_t pos = 0;
    bool any_points = false;
    for (int64_t k = 0; k < nboxes; ++k) {
        PackBox& P = pb[k];
        std::memcpy(P.box.b, boxes_host + 6 * k, sizeof(P.box.b));
        P.pnt0 = rows[2 * k];
        P.cnk0 = rows[2 * k + 1];
        P.L = layout_of(rows[2 * k + 3] - rows[2 * k + 1], rows[2 * k + 2] - rows[2 * k], nprops, es);
        P.base = pos;
        pos += P.L.bytes;
        any_points |= P.L.n_pnt > 0;
    }
    if (pos > capacity) {
        set_error("the pack buffer is smaller than sgb_pack_request reported");
        return SGB_ERANGE;
    }
    SGB_TRY(g->scratch[5].ensure(pb.size() * sizeof(PackBox)));
    SGB_TRY(g->hscratch.ensure(pb.size() * sizeof(PackBox)));
    std::memcpy(g->hscratch.p, pb.data(), pb.size() * sizeof(PackBox));
    SGB_CUDA(cudaMemcpyAsync(g->scratch[5].p, g->hscratch.p, pb.size() * sizeof(PackBox), cudaMemcpyHostToDevice, s));
    unsigned char* out = (unsigned char*)out_dev;
    if (any_points) {
        PackProps pp{};
        pp.np = nprops;
        for (int p = 0; p < nprops; ++p) {
            pp.src[p] = g->data[props[p]].as<unsigned char>();
            pp.es[p] = es[p];
            // every box's block of property p starts at a multiple of es when the blocks before it do
            bool wide = true;
            for (const PackBox& P : pb) wide = wide && (P.base + P.L.off_data + P.L.prop_off[p]) % es[p] == 0;
            pp.wide[p] = wide;
        }
        k_pack_emit<<<wgrid(g, g->n), 256, 0, s>>>(g->keys.as<int64_t>(), g->n, g->geo, g->mask.as<uint8_t>(),
                                                  g->scratch[5].as<PackBox>(), (int)nboxes, g->scratch[2].as<uint32_t>(),
                                                  g->scratch[4].as<uint32_t>(), pp, out);
        SGB_CUDA(cudaGetLastError());
    }
    k_pack_finish<<<(unsigned)nboxes, 32, 0, s>>>(g->scratch[5].as<PackBox>(), (int)nboxes, (int32_t)g->geo.size[0],
                                                 (int32_t)g->geo.size[1], (int32_t)g->geo.size[2], out);
    SGB_CUDA(cudaGetLastError());
    SGB_CUDA(cudaStreamSynchronize(s));  // the host staging of the box table is reused by the next call
    *bytes_written = pos;
    return SGB_OK;
}

extern "C" int sgb_unpack(sgb_grid* g, const void* buf_dev, int64_t nbytes, int nprops, const int* props,
                          const int64_t* start_host, int64_t* consumed, sgb_stream stream) {
    if (!g || !consumed || nbytes < 0 || (nbytes > 0 && !buf_dev)) return SGB_EINVAL;
    *consumed = 0;
    if (g->geo.dim != 3) return SGB_ENOTSUP;
    if ((uintptr_t)buf_dev % 8 != 0) {
        set_error("the pack buffer must be 8-byte aligned");
        return SGB_EINVAL;
    }
    int es[kMaxProps];
    SGB_TRY(check_props(g, nprops, props, es));
    for (int k = 0; k < nprops; ++k)
        for (int j = 0; j < k; ++j)
            if (props[j] == props[k]) return SGB_EINVAL;
    if (nbytes < 40) {  // the smallest packed box: header + one scan entry
        set_error("truncated pack buffer");
        return SGB_EINVAL;
    }
    cudaStream_t s = (cudaStream_t)stream;
    const unsigned char* buf = (const unsigned char*)buf_dev;
    SGB_TRY(g->hscratch.ensure(64));
    unsigned char* h = (unsigned char*)g->hscratch.p;
    SGB_CUDA(cudaMemcpyAsync(h, buf, 32, cudaMemcpyDeviceToHost, s));
    SGB_CUDA(cudaStreamSynchronize(s));
    uint64_t ncu;
    int32_t pst[3], psz[3];
    std::memcpy(&ncu, h, 8);
    std::memcpy(pst, h + 8, 12);
    std::memcpy(psz, h + 20, 12);
    if (ncu > (uint64_t)(nbytes - 36) / 12) {  // ids, scan and scan[n_cnk] must fit
        set_error("corrupt pack buffer (chunk count)");
        return SGB_EINVAL;
    }
    const int64_t nc_ = (int64_t)ncu;
    SGB_CUDA(cudaMemcpyAsync(h + 48, buf + 32 + 12 * nc_, 4, cudaMemcpyDeviceToHost, s));
    SGB_CUDA(cudaStreamSynchronize(s));
    uint32_t npu;
    std::memcpy(&npu, h + 48, 4);
    const PackLayout L = layout_of(nc_, npu, nprops, es);
    if (L.bytes > nbytes || (nc_ == 0 && npu != 0)) {
        set_error("corrupt pack buffer, or one packed with other properties");
        return SGB_EINVAL;
    }
    for (int d = 0; d < 3; ++d)
        if (psz[d] < 1) {
            set_error("corrupt pack buffer (grid size)");
            return SGB_EINVAL;
        }
    // the packing grid's chunk indexing: its size from the header, the same chunk edge
    Geometry src = g->geo;
    for (int d = 0; d < 3; ++d) {
        src.size[d] = psz[d];
        src.bsz[d] = (psz[d] + src.edge - 1) / src.edge;
    }
    int64_t sh[3] = {0, 0, 0};
    if (start_host)
        for (int d = 0; d < 3; ++d) sh[d] = start_host[d] - pst[d];
    const int64_t np_ = npu;
    if (np_ > 0) {
        SGB_TRY(g->pend_lin.reserve((size_t)(g->npend + np_) * 8));
        for (int p = 0; p < g->nprop; ++p)
            SGB_TRY(g->pend_val[p].reserve((size_t)(g->npend + np_) * elem_size(g->ptype[p])));
        // the properties that are not unpacked are staged with their background
        bool packed[kMaxProps] = {};
        for (int k = 0; k < nprops; ++k) packed[props[k]] = true;
        for (int p = 0; p < g->nprop; ++p) {
            const int pe = elem_size(g->ptype[p]);
            if (packed[p]) g->pend_has[p] = true;
            else SGB_TRY(fill(g->pend_val[p].as<unsigned char>() + (size_t)g->npend * pe, np_, pe, bck_pattern(g, p), s));
        }
        PackProps pp{};
        UnpackDst dst{};
        pp.np = nprops;
        for (int k = 0; k < nprops; ++k) {
            pp.es[k] = es[k];
            dst.p[k] = g->pend_val[props[k]].as<unsigned char>() + (size_t)g->npend * es[k];
        }
        k_unpack_stage<<<(unsigned)((np_ + 255) / 256), 256, 0, s>>>(buf, L, src, g->geo, sh[0], sh[1], sh[2],
                                                                     g->pend_lin.as<int64_t>() + g->npend, pp, dst,
                                                                     g->err.as<unsigned>());
        SGB_CUDA(cudaGetLastError());
        g->npend += np_;
    }
    *consumed = L.bytes;
    return SGB_OK;
}

extern "C" int sgb_unpack_boxes(sgb_grid* g, const void* buf_dev, int64_t nbytes, int nprops, const int* props,
                                int64_t nboxes, const int64_t* starts_host, int64_t* consumed, sgb_stream stream) {
    if (!g || !consumed || nbytes < 0 || nboxes < 0 || (nbytes > 0 && !buf_dev)) return SGB_EINVAL;
    *consumed = 0;
    if (g->geo.dim != 3) return SGB_ENOTSUP;
    if ((uintptr_t)buf_dev % 8 != 0) {
        set_error("the pack buffer must be 8-byte aligned");
        return SGB_EINVAL;
    }
    ElemSizes es{};
    SGB_TRY(check_props(g, nprops, props, es.es));
    es.np = nprops;
    for (int k = 0; k < nprops; ++k)
        for (int j = 0; j < k; ++j)
            if (props[j] == props[k]) return SGB_EINVAL;
    if (nboxes == 0) return SGB_OK;
    if (nboxes > (int64_t(1) << 20)) return SGB_EINVAL;
    cudaStream_t s = (cudaStream_t)stream;
    const size_t tb = (size_t)nboxes * sizeof(UnpackBox);
    SGB_TRY(g->scratch[0].ensure(tb));
    SGB_TRY(g->hscratch.ensure(tb));
    UnpackBox* dboxes = g->scratch[0].as<UnpackBox>();
    k_unpack_walk<<<1, 1, 0, s>>>((const unsigned char*)buf_dev, nbytes, (int)nboxes, es, dboxes);
    SGB_CUDA(cudaGetLastError());
    SGB_CUDA(cudaMemcpyAsync(g->hscratch.p, dboxes, tb, cudaMemcpyDeviceToHost, s));
    SGB_CUDA(cudaStreamSynchronize(s));
    std::vector<UnpackBox> hb((size_t)nboxes);
    std::memcpy(hb.data(), g->hscratch.p, tb);
    for (const UnpackBox& B : hb)
        if (B.bad) {
            set_error("corrupt or truncated pack buffer, or one packed with other properties");
            return SGB_EINVAL;
        }
    const int64_t total = hb.back().pnt0 + hb.back().n_pnt;
    for (int64_t k = 0; k < nboxes; ++k)
        for (int d = 0; d < 3; ++d) hb[k].shift[d] = starts_host ? starts_host[3 * k + d] - hb[k].start[d] : 0;
    if (total > 0) {
        std::memcpy(g->hscratch.p, hb.data(), tb);
        SGB_CUDA(cudaMemcpyAsync(dboxes, g->hscratch.p, tb, cudaMemcpyHostToDevice, s));
        SGB_TRY(g->pend_lin.reserve((size_t)(g->npend + total) * 8));
        for (int p = 0; p < g->nprop; ++p)
            SGB_TRY(g->pend_val[p].reserve((size_t)(g->npend + total) * elem_size(g->ptype[p])));
        bool packed[kMaxProps] = {};
        for (int k = 0; k < nprops; ++k) packed[props[k]] = true;
        for (int p = 0; p < g->nprop; ++p) {
            const int pe = elem_size(g->ptype[p]);
            if (packed[p]) g->pend_has[p] = true;
            else SGB_TRY(fill(g->pend_val[p].as<unsigned char>() + (size_t)g->npend * pe, total, pe, bck_pattern(g, p), s));
        }
        UnpackDst dst{};
        for (int k = 0; k < nprops; ++k) dst.p[k] = g->pend_val[props[k]].as<unsigned char>() + (size_t)g->npend * es.es[k];
        k_unpack_stage_all<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(
            (const unsigned char*)buf_dev, dboxes, (int)nboxes, total, es, g->geo, g->pend_lin.as<int64_t>() + g->npend,
            dst, g->err.as<unsigned>());
        SGB_CUDA(cudaGetLastError());
        SGB_CUDA(cudaStreamSynchronize(s));  // the host staging of the box table is reused by the next call
        g->npend += total;
    }
    const PackLayout Ll = layout_of(hb.back().n_cnk, hb.back().n_pnt, nprops, es.es);
    *consumed = hb.back().pos + Ll.bytes;
    return SGB_OK;
}
