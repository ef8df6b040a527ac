// Links between the levels of a multi-resolution hierarchy of grids.
//
// construct_link_dw / construct_link_up (src/SparseGridGpu/SparseGridGpu.hpp:
// 2113-2262; kernels count_paddings, collect_paddings, link_construct_*_count,
// link_construct_insert_*, SparseGridGpu_kernels.cuh:775-1000): the padding
// points (mask bit 1) of this grid inside an inclusive box are listed; a
// padding point at p links
//   down: to the existing points of the finer grid at 2p + p_dw + (j & 1,
//         (j >> 1) & 1, (j >> 2) & 1) for j = 0 .. 2*dim - 1 (the reference's
//         loop bound; in 3-D the children (0,1,1) and (1,1,1) are not
//         visited), in j order;
//   up:   to the existing point of the coarser grid at (p - p_up) / 2 (C
//         division, truncating toward zero).
// The other grid is read as the reference's SparseGridGpu_ker::get does:
// grid_smb::LinId without bounds checks, the id cast to unsigned int, chunk
// looked up, existence from the mask.  Results: per padding point the offset
// of its first link (exclusive scan) and the links (chunk position, offset)
// of the other grid; padding points are listed in (chunk position, offset)
// order (the reference collects them through a shared-memory atomic
// counter, any order inside a chunk).
#include <algorithm>

#include "common.cuh"
#include "internal.h"

namespace sgb {

struct Box6i {
    int64_t b[6];  // lo[3], hi[3], inclusive (Box<dim,int>::isInsideKey)
    __device__ __forceinline__ bool inside(const int64_t* p) const {
        return p[0] >= b[0] && p[0] <= b[3] && p[1] >= b[1] && p[1] <= b[4] && p[2] >= b[2] && p[2] <= b[5];
    }
};

struct OtherGrid {
    const int64_t* keys;
    const uint8_t* mask;
    int64_t n;
    Geometry geo;
};

__device__ __forceinline__ void coords_of(const Geometry& geo, int64_t key, int off, int64_t* p) {
    const int e = geo.edge;
    chunk_origin(geo, key, p);
    p[0] += off % e;
    p[1] += (off / e) % e;
    p[2] += off / (e * e);
}

// grid_smb::LinId (src/Grid/Geometry/grid_smb.hpp:176-190) then
// BlockMapGpu_ker::get_sparse(unsigned int linId) (BlockMapGpu_ker.cuh:234-249).
__device__ __forceinline__ bool other_exists(const OtherGrid& o, const int64_t* c, int32_t* pos, int16_t* off) {
    int64_t blk, loc;
    if (o.geo.zorder && (c[0] < 0 || c[1] < 0 || c[2] < 0)) {
        *pos = (int32_t)o.n;  // absent: see sgb_construct_link_dw
        *off = 0;
        return false;
    }
    point_key(o.geo, c, &blk, &loc);
    const uint32_t lin = (uint32_t)(blk * o.geo.bs + loc);
    const uint32_t b = lin / (uint32_t)o.geo.bs, ofs = lin % (uint32_t)o.geo.bs;
    int64_t p = find_key(o.keys, o.n, (int64_t)b);
    if (p < 0) p = o.n;  // the background chunk
    *pos = (int32_t)p;
    *off = (int16_t)ofs;
    return (o.mask[p * o.geo.bs + ofs] & 1) != 0;
}

__global__ void k_pad_count(const int64_t* __restrict__ keys, int64_t n, Geometry geo, const uint8_t* __restrict__ mask,
                            Box6i box, uint32_t* counts) {
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int bs = geo.bs;
    for (int64_t c = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; c < n; c += nw) {
        const int64_t key = keys[c];
        uint32_t t = 0;
        for (int pt = lane; pt < bs; pt += 32) {
            int64_t p[3];
            coords_of(geo, key, pt, p);
            const bool pad = (mask[c * bs + pt] & 2) && box.inside(p);
            t += __popc(__ballot_sync(0xffffffffu, pad));
        }
        if (lane == 0) counts[c] = t;
    }
}

__global__ void k_pad_emit(const int64_t* __restrict__ keys, int64_t n, Geometry geo, const uint8_t* __restrict__ mask,
                           Box6i box, const uint32_t* __restrict__ offs, int32_t* pad_pos, int16_t* pad_off) {
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int bs = geo.bs;
    for (int64_t c = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; c < n; c += nw) {
        const int64_t key = keys[c];
        uint32_t base = offs[c];
        for (int pt = lane; pt < bs; pt += 32) {
            int64_t p[3];
            coords_of(geo, key, pt, p);
            const bool pad = (mask[c * bs + pt] & 2) && box.inside(p);
            const unsigned bal = __ballot_sync(0xffffffffu, pad);
            if (pad) {
                const uint32_t j = base + __popc(bal & lanemask_lt());
                pad_pos[j] = (int32_t)c;
                pad_off[j] = (int16_t)pt;
            }
            base += __popc(bal);
        }
    }
}

// One thread per padding point: count (out_pos == NULL) or write its links.
template <bool DOWN>
__global__ void k_links(const int64_t* __restrict__ keys, Geometry geo, const int32_t* __restrict__ pad_pos,
                        const int16_t* __restrict__ pad_off, int64_t npad, OtherGrid o, int64_t sx, int64_t sy, int64_t sz,
                        uint32_t* counts, const uint32_t* __restrict__ scan, int32_t* out_pos, int16_t* out_off) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= npad) return;
    int64_t p[3];
    coords_of(geo, keys[pad_pos[t]], pad_off[t], p);
    const int64_t sh[3] = {sx, sy, sz};
    uint32_t k = 0, at = out_pos ? scan[t] : 0;
    if (DOWN) {
        for (int j = 0; j < 2 * 3; ++j) {
            int64_t c[3];
            for (int d = 0; d < 3; ++d) c[d] = p[d] * 2 + sh[d] + ((j >> d) & 1);
            int32_t lp;
            int16_t lo;
            if (other_exists(o, c, &lp, &lo)) {
                if (out_pos) {
                    out_pos[at + k] = lp;
                    out_off[at + k] = lo;
                }
                ++k;
            }
        }
    } else {
        int64_t c[3];
        for (int d = 0; d < 3; ++d) c[d] = (p[d] - sh[d]) / 2;
        int32_t lp;
        int16_t lo;
        if (other_exists(o, c, &lp, &lo)) {
            if (out_pos) {
                out_pos[at] = lp;
                out_off[at] = lo;
            }
            k = 1;
        }
    }
    if (!out_pos) counts[t] = k;
}

static unsigned warp_grid(const sgb_grid* g, int64_t n) {
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>((int64_t)g->num_sms * 8, (n + 7) / 8));
}

static int construct_links(sgb_grid* g, const sgb_grid* other, const int64_t* box_host, const int64_t* shift_host,
                           int up, cudaStream_t s) {
    if (!g || !other || !box_host || !shift_host) return SGB_EINVAL;
    if (g->geo.dim != 3 || other->geo.dim != 3) return SGB_ENOTSUP;
    if (other->geo.edge != g->geo.edge) {
        set_error("linked grids share the chunk edge");
        return SGB_EINVAL;
    }
    if (other->device != g->device) {
        set_error("linked grids live on the same device");
        return SGB_EINVAL;
    }
    Box6i box;
    for (int k = 0; k < 6; ++k) box.b[k] = box_host[k];
    LinkSet& L = g->links[up];
    L.npad = L.nlinks = 0;
    const int64_t n = g->n;
    SGB_TRY(g->hscratch.ensure(64));
    if (n > 0) {
        SGB_TRY(g->scratch[1].ensure((size_t)n * 4 + 16));
        SGB_TRY(g->scratch[2].ensure((size_t)(n + 1) * 4 + 16));
        uint32_t* counts = g->scratch[1].as<uint32_t>();
        uint32_t* offs = g->scratch[2].as<uint32_t>();
        k_pad_count<<<warp_grid(g, n), 256, 0, s>>>(g->keys.as<int64_t>(), n, g->geo, g->mask.as<uint8_t>(), box, counts);
        SGB_CUDA(cudaGetLastError());
        SGB_TRY(scan_exclusive_u32(counts, offs, n, offs + n, &g->scratch[6], s));
        SGB_CUDA(cudaMemcpyAsync(g->hscratch.p, offs + n, 4, cudaMemcpyDeviceToHost, s));
        SGB_CUDA(cudaStreamSynchronize(s));
        L.npad = *(uint32_t*)g->hscratch.p;
        SGB_TRY(L.pad_pos.ensure((size_t)L.npad * 4 + 16));
        SGB_TRY(L.pad_off.ensure((size_t)L.npad * 2 + 16));
        k_pad_emit<<<warp_grid(g, n), 256, 0, s>>>(g->keys.as<int64_t>(), n, g->geo, g->mask.as<uint8_t>(), box, offs,
                                                  L.pad_pos.as<int32_t>(), L.pad_off.as<int16_t>());
        SGB_CUDA(cudaGetLastError());
    }
    SGB_TRY(L.scan.ensure((size_t)(L.npad + 1) * 4 + 16));
    if (L.npad > 0) {
        OtherGrid o{other->keys.as<int64_t>(), other->mask.as<uint8_t>(), other->n, other->geo};
        SGB_TRY(g->scratch[1].ensure((size_t)L.npad * 4 + 16));
        uint32_t* counts = g->scratch[1].as<uint32_t>();
        uint32_t* scan = L.scan.as<uint32_t>();
        const unsigned blocks = (unsigned)((L.npad + 255) / 256);
        if (up)
            k_links<false><<<blocks, 256, 0, s>>>(g->keys.as<int64_t>(), g->geo, L.pad_pos.as<int32_t>(),
                                                 L.pad_off.as<int16_t>(), L.npad, o, shift_host[0], shift_host[1],
                                                 shift_host[2], counts, nullptr, nullptr, nullptr);
        else
            k_links<true><<<blocks, 256, 0, s>>>(g->keys.as<int64_t>(), g->geo, L.pad_pos.as<int32_t>(),
                                                L.pad_off.as<int16_t>(), L.npad, o, shift_host[0], shift_host[1],
                                                shift_host[2], counts, nullptr, nullptr, nullptr);
        SGB_CUDA(cudaGetLastError());
        SGB_TRY(scan_exclusive_u32(counts, scan, L.npad, scan + L.npad, &g->scratch[6], s));
        SGB_CUDA(cudaMemcpyAsync(g->hscratch.p, scan + L.npad, 4, cudaMemcpyDeviceToHost, s));
        SGB_CUDA(cudaStreamSynchronize(s));
        L.nlinks = *(uint32_t*)g->hscratch.p;
        SGB_TRY(L.pos.ensure((size_t)L.nlinks * 4 + 16));
        SGB_TRY(L.off.ensure((size_t)L.nlinks * 2 + 16));
        if (up)
            k_links<false><<<blocks, 256, 0, s>>>(g->keys.as<int64_t>(), g->geo, L.pad_pos.as<int32_t>(),
                                                 L.pad_off.as<int16_t>(), L.npad, o, shift_host[0], shift_host[1],
                                                 shift_host[2], nullptr, scan, L.pos.as<int32_t>(), L.off.as<int16_t>());
        else
            k_links<true><<<blocks, 256, 0, s>>>(g->keys.as<int64_t>(), g->geo, L.pad_pos.as<int32_t>(),
                                                L.pad_off.as<int16_t>(), L.npad, o, shift_host[0], shift_host[1],
                                                shift_host[2], nullptr, scan, L.pos.as<int32_t>(), L.off.as<int16_t>());
        SGB_CUDA(cudaGetLastError());
    } else {
        SGB_CUDA(cudaMemsetAsync(L.scan.p, 0, 4, s));
    }
    SGB_CUDA(cudaStreamSynchronize(s));
    return SGB_OK;
}

}  // namespace sgb

using namespace sgb;

extern "C" int sgb_construct_link_dw(sgb_grid* g, const sgb_grid* grid_dw, const int64_t* box_host,
                                     const int64_t* p_dw_host, sgb_stream s) {
    return construct_links(g, grid_dw, box_host, p_dw_host, 0, (cudaStream_t)s);
}

extern "C" int sgb_construct_link_up(sgb_grid* g, const sgb_grid* grid_up, const int64_t* box_host,
                                     const int64_t* p_up_host, sgb_stream s) {
    return construct_links(g, grid_up, box_host, p_up_host, 1, (cudaStream_t)s);
}

extern "C" int sgb_get_links(sgb_grid* g, int up, sgb_links* out) {
    if (!g || !out || (up != 0 && up != 1)) return SGB_EINVAL;
    const LinkSet& L = g->links[up];
    out->npad = L.npad;
    out->pad_pos = L.pad_pos.as<int32_t>();
    out->pad_off = L.pad_off.as<int16_t>();
    out->offsets = L.scan.as<uint32_t>();
    out->nlinks = L.nlinks;
    out->link_pos = L.pos.as<int32_t>();
    out->link_off = L.off.as<int16_t>();
    return SGB_OK;
}
