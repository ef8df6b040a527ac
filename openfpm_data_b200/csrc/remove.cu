// Point removal by boxes and enumeration of the existing points.
//
// remove(box) + removePoints (src/SparseGridGpu/SparseGridGpu.hpp:3417-3489,
// 3528-3531; SparseGridGpu_kernels.cuh:1235-1340): every existing point
// inside one of the queued boxes loses its mask byte; the chunks stay.  The
// reference tests points against Box<dim, unsigned int>, so the int boxes are
// converted to unsigned int here too.  The removed points also get their
// properties' backgrounds, which keeps the grid's background invariant.
//
// The enumeration lists the existing points in (chunk position, offset in the
// chunk) order, the order in which the reference's iterators
// (src/SparseGridGpu/Iterators/SparseGridGpu_iterator.hpp:17-304) visit them.
#include <cstring>
#include <vector>

#include "common.cuh"
#include "internal.h"

namespace sgb {

struct UBox {
    uint32_t lo[3], hi[3];
};

struct BckSet {
    unsigned char* p[kMaxProps];
    uint64_t pat[kMaxProps];
    int es[kMaxProps];
    int nprop;
};

// One CTA per chunk (grid-stride): skip chunks that no box touches, then test
// every existing point.
__global__ void k_remove_boxes(const int64_t* __restrict__ keys, int64_t n, Geometry geo, uint8_t* mask,
                               const UBox* __restrict__ boxes, int nb, BckSet bck) {
    const int bs = geo.bs, e = geo.edge;
    for (int64_t c = blockIdx.x; c < n; c += gridDim.x) {
        int64_t o[3];
        chunk_origin(geo, keys[c], o);
        bool touch = false;
        for (int k = 0; k < nb && !touch; ++k) {
            bool t = true;
            for (int d = 0; d < 3; ++d) {
                const uint32_t clo = (uint32_t)o[d], chi = (uint32_t)(o[d] + e - 1);
                t = t && !(chi < boxes[k].lo[d] || clo > boxes[k].hi[d]);
            }
            touch = t;
        }
        if (!touch) continue;  // uniform over the CTA
        for (int pt = threadIdx.x; pt < bs; pt += blockDim.x) {
            const int64_t idx = c * bs + pt;
            if (!(mask[idx] & 1)) continue;
            const uint32_t pc[3] = {(uint32_t)(o[0] + pt % e), (uint32_t)(o[1] + (pt / e) % e),
                                    (uint32_t)(o[2] + pt / (e * e))};
            bool in = false;
            for (int k = 0; k < nb && !in; ++k)
                in = pc[0] >= boxes[k].lo[0] && pc[0] <= boxes[k].hi[0] && pc[1] >= boxes[k].lo[1] &&
                     pc[1] <= boxes[k].hi[1] && pc[2] >= boxes[k].lo[2] && pc[2] <= boxes[k].hi[2];
            if (!in) continue;
            mask[idx] = 0;
            for (int p = 0; p < bck.nprop; ++p) {
                unsigned char* q = bck.p[p] + (size_t)idx * bck.es[p];
                for (int b = 0; b < bck.es[p]; ++b) q[b] = (unsigned char)(bck.pat[p] >> (8 * b));
            }
        }
    }
}

__device__ __forceinline__ bool in_ibox(const int64_t* box, int64_t x, int64_t y, int64_t z) {
    return x >= box[0] && x <= box[3] && y >= box[1] && y <= box[4] && z >= box[2] && z <= box[5];
}

struct IBox {
    int64_t b[6];
    int has;
};

// Existing points per chunk (inside the box when there is one): one warp per chunk.
__global__ void k_count_points(const int64_t* __restrict__ keys, int64_t n, Geometry geo, const uint8_t* __restrict__ mask,
                               IBox box, uint32_t* counts) {
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int bs = geo.bs, e = geo.edge;
    for (int64_t c = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; c < n; c += nw) {
        int64_t o[3];
        chunk_origin(geo, keys[c], o);
        uint32_t cnt = 0;
        for (int pt = lane; pt < bs; pt += 32) {
            bool ex = mask[c * bs + pt] & 1;
            if (box.has) ex = ex && in_ibox(box.b, o[0] + pt % e, o[1] + (pt / e) % e, o[2] + pt / (e * e));
            cnt += __popc(__ballot_sync(0xffffffffu, ex));
        }
        if (lane == 0) counts[c] = cnt;
    }
}

// Coordinates of those points at their scanned offsets, in offset order inside each chunk.
__global__ void k_emit_points(const int64_t* __restrict__ keys, int64_t n, Geometry geo, const uint8_t* __restrict__ mask,
                              IBox box, const uint32_t* __restrict__ offs, int32_t* out) {
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int bs = geo.bs, e = geo.edge;
    for (int64_t c = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; c < n; c += nw) {
        int64_t o[3];
        chunk_origin(geo, keys[c], o);
        uint32_t base = offs[c];
        for (int pt = lane; pt < bs; pt += 32) {
            const int64_t x = o[0] + pt % e, y = o[1] + (pt / e) % e, z = o[2] + pt / (e * e);
            bool ex = mask[c * bs + pt] & 1;
            if (box.has) ex = ex && in_ibox(box.b, x, y, z);
            const unsigned bal = __ballot_sync(0xffffffffu, ex);
            if (ex) {
                const uint32_t k = base + __popc(bal & lanemask_lt());
                out[(size_t)k * 3 + 0] = (int32_t)x;
                out[(size_t)k * 3 + 1] = (int32_t)y;
                out[(size_t)k * 3 + 2] = (int32_t)z;
            }
            base += __popc(bal);
        }
    }
}

static unsigned warp_blocks(const sgb_grid* g, int64_t n) {
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>((int64_t)g->num_sms * 8, (n + 7) / 8));
}

}  // namespace sgb

using namespace sgb;

extern "C" int sgb_remove_boxes(sgb_grid* g, int64_t nboxes, const int64_t* boxes_host, sgb_stream stream) {
    if (!g || nboxes < 0 || (nboxes > 0 && !boxes_host)) return SGB_EINVAL;
    if (g->geo.dim != 3) {
        set_error("removal by boxes is implemented for 3-D grids");
        return SGB_ENOTSUP;
    }
    if (nboxes == 0 || g->n == 0) return SGB_OK;
    cudaStream_t s = (cudaStream_t)stream;
    std::vector<UBox> hb((size_t)nboxes);
    for (int64_t k = 0; k < nboxes; ++k)
        for (int d = 0; d < 3; ++d) {
            hb[k].lo[d] = (uint32_t)(int32_t)boxes_host[k * 6 + d];  // Box<dim,int> -> Box<dim,unsigned int>
            hb[k].hi[d] = (uint32_t)(int32_t)boxes_host[k * 6 + 3 + d];
        }
    SGB_TRY(g->scratch[0].ensure(hb.size() * sizeof(UBox)));
    SGB_TRY(g->hscratch.ensure(hb.size() * sizeof(UBox)));
    std::memcpy(g->hscratch.p, hb.data(), hb.size() * sizeof(UBox));
    SGB_CUDA(cudaMemcpyAsync(g->scratch[0].p, g->hscratch.p, hb.size() * sizeof(UBox), cudaMemcpyHostToDevice, s));
    BckSet bk{};
    bk.nprop = g->nprop;
    for (int p = 0; p < g->nprop; ++p) {
        bk.p[p] = g->data[p].as<unsigned char>();
        bk.pat[p] = bck_pattern(g, p);
        bk.es[p] = elem_size(g->ptype[p]);
    }
    const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>(g->n, (int64_t)g->num_sms * 8));
    k_remove_boxes<<<blocks, 256, 0, s>>>(g->keys.as<int64_t>(), g->n, g->geo, g->mask.as<uint8_t>(),
                                          g->scratch[0].as<UBox>(), (int)nboxes, bk);
    SGB_CUDA(cudaGetLastError());
    // the host copy of the boxes must outlive the asynchronous upload
    SGB_CUDA(cudaStreamSynchronize(s));
    // existence changed; chunks, neighbours and backgrounds did not
    g->bits_valid = false;
    g->epts_valid = false;
    return SGB_OK;
}

extern "C" int sgb_existing_points(sgb_grid* g, const int64_t* box_host, int32_t* coords_dev, int64_t capacity,
                                   int64_t* count, sgb_stream stream) {
    if (!g || !count || capacity < 0 || (capacity > 0 && !coords_dev)) return SGB_EINVAL;
    if (g->geo.dim != 3) {
        set_error("point enumeration is implemented for 3-D grids");
        return SGB_ENOTSUP;
    }
    *count = 0;
    if (g->n == 0) return SGB_OK;
    cudaStream_t s = (cudaStream_t)stream;
    IBox box{};
    if (box_host) {
        std::memcpy(box.b, box_host, sizeof(box.b));
        box.has = 1;
    }
    const int64_t n = g->n;
    SGB_TRY(g->scratch[1].ensure((size_t)n * 4 + 16));
    SGB_TRY(g->scratch[2].ensure((size_t)(n + 1) * 4 + 16));
    uint32_t* counts = g->scratch[1].as<uint32_t>();
    uint32_t* offs = g->scratch[2].as<uint32_t>();
    k_count_points<<<warp_blocks(g, n), 256, 0, s>>>(g->keys.as<int64_t>(), n, g->geo, g->mask.as<uint8_t>(), box,
                                                     counts);
    SGB_CUDA(cudaGetLastError());
    SGB_TRY(scan_exclusive_u32(counts, offs, n, offs + n, &g->scratch[6], s));
    SGB_TRY(g->hscratch.ensure(64));
    SGB_CUDA(cudaMemcpyAsync(g->hscratch.p, offs + n, 4, cudaMemcpyDeviceToHost, s));
    SGB_CUDA(cudaStreamSynchronize(s));
    const int64_t total = *(uint32_t*)g->hscratch.p;
    *count = total;
    if (total == 0 || capacity < total) return SGB_OK;  // the caller sizes the buffer from *count
    k_emit_points<<<warp_blocks(g, n), 256, 0, s>>>(g->keys.as<int64_t>(), n, g->geo, g->mask.as<uint8_t>(), box,
                                                    offs, coords_dev);
    SGB_CUDA(cudaGetLastError());
    return SGB_OK;
}
