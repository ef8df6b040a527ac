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

static inline int64_t pad8(int64_t b) { return (b + 7) & ~(int64_t)7; }

struct PackLayout {
    int64_t n_cnk, n_pnt;
    int64_t off_ids, off_scan, off_data, off_offs, off_mask, bytes;
    int64_t prop_off[kMaxProps];
};

static PackLayout layout_of(int64_t n_cnk, int64_t n_pnt, int np, const int* es) {
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
    o += pad8(d);
    L.off_offs = o;
    o += pad8(2 * n_pnt);
    L.off_mask = o;
    o += pad8(n_pnt);
    L.bytes = o;
    return L;
}

__device__ __forceinline__ void origin_of(const Geometry& geo, int64_t key, int64_t* o) {
    o[0] = (key % geo.bsz[0]) * geo.edge;
    o[1] = ((key / geo.bsz[0]) % geo.bsz[1]) * geo.edge;
    o[2] = (key / (geo.bsz[0] * geo.bsz[1])) * geo.edge;
}

struct Box6 {
    int64_t b[6];
};

__device__ __forceinline__ bool inside6(const Box6& bx, int64_t x, int64_t y, int64_t z) {
    return x >= bx.b[0] && x <= bx.b[3] && y >= bx.b[1] && y <= bx.b[4] && z >= bx.b[2] && z <= bx.b[5];
}

// Existing points of each chunk inside the box, and whether the chunk has any.
__global__ void k_pack_count(const int64_t* __restrict__ keys, int64_t n, Geometry geo, const uint8_t* __restrict__ mask,
                             Box6 box, uint32_t* counts, uint32_t* flags) {
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int bs = geo.bs, e = geo.edge;
    for (int64_t c = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; c < n; c += nw) {
        int64_t o[3];
        origin_of(geo, keys[c], o);
        uint32_t cnt = 0;
        for (int pt = lane; pt < bs; pt += 32) {
            const bool in = (mask[c * bs + pt] & 1) && inside6(box, o[0] + pt % e, o[1] + (pt / e) % e, o[2] + pt / (e * e));
            cnt += __popc(__ballot_sync(0xffffffffu, in));
        }
        if (lane == 0) {
            counts[c] = cnt;
            flags[c] = cnt != 0;
        }
    }
}

struct PackProps {
    const unsigned char* src[kMaxProps];
    int es[kMaxProps];
    int64_t off[kMaxProps];  // byte offset of the property's block inside the data block
    int np;
};

__global__ void k_pack_emit(const int64_t* __restrict__ keys, int64_t n, Geometry geo, const uint8_t* __restrict__ mask,
                            Box6 box, const uint32_t* __restrict__ counts, const uint32_t* __restrict__ pt_off,
                            const uint32_t* __restrict__ c_off, PackProps pp, unsigned char* out, PackLayout L) {
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int bs = geo.bs, e = geo.edge;
    int64_t* ids = reinterpret_cast<int64_t*>(out + L.off_ids);
    uint32_t* scan = reinterpret_cast<uint32_t*>(out + L.off_scan);
    int16_t* offs = reinterpret_cast<int16_t*>(out + L.off_offs);
    uint8_t* msk = out + L.off_mask;
    for (int64_t c = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; c < n; c += nw) {
        if (counts[c] == 0) continue;  // uniform over the warp
        const int64_t key = keys[c];
        if (lane == 0) {
            ids[c_off[c]] = key;
            scan[c_off[c]] = pt_off[c];
        }
        int64_t o[3];
        origin_of(geo, key, o);
        uint32_t base = pt_off[c];
        for (int pt = lane; pt < bs; pt += 32) {
            const uint8_t m = mask[c * bs + pt];
            const bool in = (m & 1) && inside6(box, o[0] + pt % e, o[1] + (pt / e) % e, o[2] + pt / (e * e));
            const unsigned bal = __ballot_sync(0xffffffffu, in);
            if (in) {
                const int64_t j = base + __popc(bal & lanemask_lt());
                const int64_t idx = c * bs + pt;
                for (int p = 0; p < pp.np; ++p) {
                    const int es = pp.es[p];
                    unsigned char* d = out + L.off_data + pp.off[p] + j * es;
                    const unsigned char* sp = pp.src[p] + idx * es;
                    for (int b = 0; b < es; ++b) d[b] = sp[b];
                }
                offs[j] = (int16_t)pt;
                msk[j] = m;
            }
            base += __popc(bal);
        }
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
        const int de = dst_geo.edge;
        int64_t b = c[2] / de, l = c[2] % de;
        b = b * dst_geo.bsz[1] + c[1] / de;
        l = l * de + c[1] % de;
        b = b * dst_geo.bsz[0] + c[0] / de;
        l = l * de + c[0] % de;
        lin = b * dst_geo.bs + l;
    } else {
        atomicOr(err, kErrOutOfDomain);
    }
    out_lin[j] = lin;
    for (int p = 0; p < pp.np; ++p) {
        const int es = pp.es[p];
        const unsigned char* s = buf + L.off_data + pp.off[p] + j * es;
        for (int b = 0; b < es; ++b) dst.p[p][j * es + b] = s[b];
    }
}

static unsigned wgrid(const sgb_grid* g, int64_t n) {
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>((int64_t)g->num_sms * 8, (n + 7) / 8));
}

// Counts of one box: fills scratch[1] (counts), [2] (point offsets), [3] (flags), [4] (chunk offsets);
// returns n_pnt and n_cnk.
static int box_counts(sgb_grid* g, const Box6& box, int64_t* n_pnt, int64_t* n_cnk, cudaStream_t s) {
    const int64_t n = g->n;
    *n_pnt = *n_cnk = 0;
    if (n == 0) return SGB_OK;
    for (int k = 1; k <= 4; ++k) SGB_TRY(g->scratch[k].ensure((size_t)(n + 1) * 4 + 16));
    uint32_t *cnt = g->scratch[1].as<uint32_t>(), *poff = g->scratch[2].as<uint32_t>(),
             *flg = g->scratch[3].as<uint32_t>(), *coff = g->scratch[4].as<uint32_t>();
    k_pack_count<<<wgrid(g, n), 256, 0, s>>>(g->keys.as<int64_t>(), n, g->geo, g->mask.as<uint8_t>(), box, cnt, flg);
    SGB_CUDA(cudaGetLastError());
    SGB_TRY(scan_exclusive_u32(cnt, poff, n, poff + n, &g->scratch[6], s));
    SGB_TRY(scan_exclusive_u32(flg, coff, n, coff + n, &g->scratch[6], s));
    SGB_TRY(g->hscratch.ensure(64));
    uint32_t* h = (uint32_t*)g->hscratch.p;
    SGB_CUDA(cudaMemcpyAsync(h, poff + n, 4, cudaMemcpyDeviceToHost, s));
    SGB_CUDA(cudaMemcpyAsync(h + 1, coff + n, 4, cudaMemcpyDeviceToHost, s));
    SGB_CUDA(cudaStreamSynchronize(s));
    *n_pnt = h[0];
    *n_cnk = h[1];
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
    cudaStream_t s = (cudaStream_t)stream;
    for (int64_t k = 0; k < nboxes; ++k) {
        Box6 box;
        std::memcpy(box.b, boxes_host + k * 6, sizeof(box.b));
        int64_t np_, nc_;
        SGB_TRY(box_counts(g, box, &np_, &nc_, s));
        bytes_host[k] = layout_of(nc_, np_, nprops, es).bytes;
    }
    return SGB_OK;
}

extern "C" int sgb_pack(sgb_grid* g, int64_t nboxes, const int64_t* boxes_host, int nprops, const int* props,
                        void* out_dev, int64_t capacity, int64_t* bytes_written, sgb_stream stream) {
    if (!g || nboxes < 0 || (nboxes > 0 && (!boxes_host || !out_dev)) || !bytes_written) return SGB_EINVAL;
    if (g->geo.dim != 3) return SGB_ENOTSUP;
    int es[kMaxProps];
    SGB_TRY(check_props(g, nprops, props, es));
    if ((uintptr_t)out_dev % 8 != 0) {
        set_error("the pack buffer must be 8-byte aligned");
        return SGB_EINVAL;
    }
    cudaStream_t s = (cudaStream_t)stream;
    unsigned char* out = (unsigned char*)out_dev;
    int64_t pos = 0;
    *bytes_written = 0;
    SGB_TRY(g->hscratch.ensure(64));
    for (int64_t k = 0; k < nboxes; ++k) {
        Box6 box;
        std::memcpy(box.b, boxes_host + k * 6, sizeof(box.b));
        int64_t np_, nc_;
        SGB_TRY(box_counts(g, box, &np_, &nc_, s));
        const PackLayout L = layout_of(nc_, np_, nprops, es);
        if (pos + L.bytes > capacity) {
            set_error("the pack buffer is smaller than sgb_pack_request reported");
            return SGB_ERANGE;
        }
        unsigned char* b = out + pos;
        // header: n_cnk, start = the box's lower corner, size = the grid's size
        unsigned char hdr[32];
        const uint64_t ncu = (uint64_t)nc_;
        std::memcpy(hdr, &ncu, 8);
        for (int d = 0; d < 3; ++d) {
            const int32_t st = (int32_t)box.b[d], sz = (int32_t)g->geo.size[d];
            std::memcpy(hdr + 8 + 4 * d, &st, 4);
            std::memcpy(hdr + 20 + 4 * d, &sz, 4);
        }
        std::memcpy(g->hscratch.p, hdr, 32);
        SGB_CUDA(cudaMemcpyAsync(b, g->hscratch.p, 32, cudaMemcpyHostToDevice, s));
        // zero the padding so packed buffers compare bytewise
        SGB_CUDA(cudaMemsetAsync(b + 32, 0, L.bytes - 32, s));
        if (np_ > 0) {
            PackProps pp{};
            pp.np = nprops;
            for (int p = 0; p < nprops; ++p) {
                pp.src[p] = g->data[props[p]].as<unsigned char>();
                pp.es[p] = es[p];
                pp.off[p] = L.prop_off[p];
            }
            k_pack_emit<<<wgrid(g, g->n), 256, 0, s>>>(g->keys.as<int64_t>(), g->n, g->geo, g->mask.as<uint8_t>(), box,
                                                      g->scratch[1].as<uint32_t>(), g->scratch[2].as<uint32_t>(),
                                                      g->scratch[4].as<uint32_t>(), pp, b, L);
            SGB_CUDA(cudaGetLastError());
        }
        // scan[n_cnk] = n_pnt
        const uint32_t npu = (uint32_t)np_;
        std::memcpy((unsigned char*)g->hscratch.p + 32, &npu, 4);
        SGB_CUDA(cudaMemcpyAsync(b + L.off_scan + 4 * nc_, (unsigned char*)g->hscratch.p + 32, 4, cudaMemcpyHostToDevice, s));
        SGB_CUDA(cudaStreamSynchronize(s));  // the host staging is reused by the next box
        pos += L.bytes;
    }
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
            pp.off[k] = L.prop_off[k];
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
