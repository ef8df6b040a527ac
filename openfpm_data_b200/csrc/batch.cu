// Batched form: many independent grids advanced by one persistent launch per
// step over their concatenated block maps.  No reference counterpart (the
// reference launches one applyStencils per grid,
// src/SparseGridGpu/SparseGridGpu.hpp:2704-2734).
//
// Layout: the member grids' chunks are concatenated; per chunk the batch
// keeps the mask, an 8-entry NNStar neighbour list in batch positions (-1
// absent: a grid never sees another grid's chunks), the owning slot id and
// two ping-pong buffers per source property.  A slot added at global step T0
// with nsteps steps reads buffer (t - T0) & 1 at step t and idles afterwards,
// so every launch of a captured graph is valid without device-side state.
#include <algorithm>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "internal.h"
#include "stencil.cuh"

struct sgb_batch {
    int device = 0;
    int kind = -1, edge = 0, np = 0;
    int64_t n = 0, cap = 0;
    sgb::DevBuf keys, mask, nn, gid, grids;
    sgb::DevBuf field[2][2];
    // compaction targets
    sgb::DevBuf keys2, mask2, nn2, gid2;
    sgb::DevBuf field2[2][2];
    struct Slot {
        bool live = false;
        int64_t off = 0, n = 0;
        sgb::GridInfo gi{};
        int src[2] = {0, 0}, dst[2] = {0, 0};  // grid properties behind buffers 0 / 1
    };
    std::vector<Slot> slots;
    int64_t T = 0;
    bool dirty = true;     // grids table must be uploaded
    bool holes = false;    // removed slots to compact
    int num_sms = 148, ctas_per_sm = 0, stages = 0;  // 0: automatic
    sgb::DevBuf err;
    // the instantiated graph of the last sgb_batch_step call with use_graph, updated in place for the
    // next call of the same step count (kernel arguments change, the graph's shape does not)
    cudaGraphExec_t exec = nullptr;
    int exec_nsteps = -1;
    // pinned staging of the grids table: two buffers used in turn, each free once its copy event fired
    void* grids_host[2] = {nullptr, nullptr};
    size_t grids_host_bytes[2] = {0, 0};
    cudaEvent_t grids_done[2] = {nullptr, nullptr};
    int grids_turn = 0;
};

namespace sgb {

__global__ void k_offset_nn(const int32_t* in, int32_t* out, int64_t count, int64_t delta) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < count) {
        const int32_t v = in[i];
        out[i] = v >= 0 ? (int32_t)(v + delta) : -1;
    }
}

__global__ void k_fill_i32(int32_t* out, int64_t count, int32_t v) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < count) out[i] = v;
}

static int batch_reserve(sgb_batch* b, int64_t chunks) {
    if (chunks <= b->cap) return SGB_OK;
    int64_t nc = std::max<int64_t>(chunks, b->cap + b->cap / 2);
    nc = std::max<int64_t>(nc, 64);
    const int bs = b->edge * b->edge * b->edge;
    SGB_TRY(b->keys.reserve((size_t)nc * 8));
    SGB_TRY(b->mask.reserve((size_t)nc * bs));
    SGB_TRY(b->nn.reserve((size_t)nc * 8 * 4));
    SGB_TRY(b->gid.reserve((size_t)nc * 4));
    for (int k = 0; k < 2; ++k)
        for (int p = 0; p < b->np; ++p) SGB_TRY(b->field[k][p].reserve((size_t)nc * bs * 4));
    b->cap = nc;
    return SGB_OK;
}

// Remove dead slots: copy live chunk ranges to the front (second buffer set).
static int batch_compact(sgb_batch* b, cudaStream_t s) {
    if (!b->holes) return SGB_OK;
    const int bs = b->edge * b->edge * b->edge;
    int64_t live = 0;
    for (auto& sl : b->slots)
        if (sl.live) live += sl.n;
    const int64_t c = std::max<int64_t>(live, 64);
    SGB_TRY(b->keys2.ensure((size_t)c * 8));
    SGB_TRY(b->mask2.ensure((size_t)c * bs));
    SGB_TRY(b->nn2.ensure((size_t)c * 32));
    SGB_TRY(b->gid2.ensure((size_t)c * 4));
    for (int k = 0; k < 2; ++k)
        for (int p = 0; p < b->np; ++p) SGB_TRY(b->field2[k][p].ensure((size_t)c * bs * 4));
    int64_t off = 0;
    for (size_t si = 0; si < b->slots.size(); ++si) {
        auto& sl = b->slots[si];
        if (!sl.live || sl.n == 0) {
            if (!sl.live) sl.n = 0;
            continue;
        }
        SGB_CUDA(cudaMemcpyAsync(b->keys2.as<int64_t>() + off, b->keys.as<int64_t>() + sl.off, sl.n * 8,
                                 cudaMemcpyDeviceToDevice, s));
        SGB_CUDA(cudaMemcpyAsync(b->mask2.as<uint8_t>() + off * bs, b->mask.as<uint8_t>() + sl.off * bs, sl.n * bs,
                                 cudaMemcpyDeviceToDevice, s));
        for (int k = 0; k < 2; ++k)
            for (int p = 0; p < b->np; ++p)
                SGB_CUDA(cudaMemcpyAsync(b->field2[k][p].as<float>() + off * bs, b->field[k][p].as<float>() + sl.off * bs,
                                         sl.n * bs * 4, cudaMemcpyDeviceToDevice, s));
        k_offset_nn<<<(unsigned)((sl.n * 8 + 255) / 256), 256, 0, s>>>(b->nn.as<int32_t>() + sl.off * 8,
                                                                        b->nn2.as<int32_t>() + off * 8, sl.n * 8,
                                                                        off - sl.off);
        k_fill_i32<<<(unsigned)((sl.n + 255) / 256), 256, 0, s>>>(b->gid2.as<int32_t>() + off, sl.n, (int32_t)si);
        SGB_CUDA(cudaGetLastError());
        sl.off = off;
        off += sl.n;
    }
    std::swap(b->keys, b->keys2);
    std::swap(b->mask, b->mask2);
    std::swap(b->nn, b->nn2);
    std::swap(b->gid, b->gid2);
    for (int k = 0; k < 2; ++k)
        for (int p = 0; p < b->np; ++p) std::swap(b->field[k][p], b->field2[k][p]);
    // the capacity every array holds (their allocations round differently)
    int64_t cap = std::min<int64_t>((int64_t)(b->keys.bytes / 8), (int64_t)(b->mask.bytes / bs));
    cap = std::min<int64_t>(cap, (int64_t)(b->nn.bytes / 32));
    cap = std::min<int64_t>(cap, (int64_t)(b->gid.bytes / 4));
    for (int k = 0; k < 2; ++k)
        for (int p = 0; p < b->np; ++p) cap = std::min<int64_t>(cap, (int64_t)(b->field[k][p].bytes / ((size_t)bs * 4)));
    b->cap = cap;
    b->n = off;
    b->holes = false;
    return SGB_OK;
}

// Upload the grids table without a host wait: it is staged in one of two pinned buffers, taken in
// turn; a buffer is rewritten only after the event recorded behind its previous copy has fired.
static int batch_upload_grids(sgb_batch* b, cudaStream_t s) {
    if (!b->dirty) return SGB_OK;
    const size_t bytes = std::max<size_t>(1, b->slots.size()) * sizeof(GridInfo);
    SGB_TRY(b->grids.ensure(bytes));
    const int k = b->grids_turn;
    b->grids_turn ^= 1;
    if (b->grids_done[k]) SGB_CUDA(cudaEventSynchronize(b->grids_done[k]));
    else SGB_CUDA(cudaEventCreateWithFlags(&b->grids_done[k], cudaEventDisableTiming));
    if (b->grids_host_bytes[k] < bytes) {
        if (b->grids_host[k]) cudaFreeHost(b->grids_host[k]);
        b->grids_host[k] = nullptr;
        b->grids_host_bytes[k] = 0;
        SGB_CUDA(cudaMallocHost(&b->grids_host[k], bytes * 2));
        b->grids_host_bytes[k] = bytes * 2;
    }
    GridInfo* h = static_cast<GridInfo*>(b->grids_host[k]);
    for (size_t i = 0; i < b->slots.size(); ++i) h[i] = b->slots[i].gi;
    if (!b->slots.empty())
        SGB_CUDA(cudaMemcpyAsync(b->grids.p, h, b->slots.size() * sizeof(GridInfo), cudaMemcpyHostToDevice, s));
    SGB_CUDA(cudaEventRecord(b->grids_done[k], s));
    b->dirty = false;
    return SGB_OK;
}

static int batch_launch(sgb_batch* b, int64_t t, cudaStream_t s) {
    LaunchDesc L;
    std::memset(&L, 0, sizeof(L));
    L.kind = b->kind;
    L.edge = b->edge;
    L.use_tile = 0;
    L.stages = b->stages;
    L.num_sms = b->num_sms;
    const int cps = b->ctas_per_sm > 0 ? b->ctas_per_sm : auto_ctas_per_sm(b->kind);
    L.ctas = (unsigned)std::max<int64_t>(1, std::min<int64_t>(b->n, (int64_t)b->num_sms * cps));
    for (int k = 0; k < 2; ++k)
        for (int j = 0; j < 2; ++j) {
            const int p = j < b->np ? j : 0;
            L.fs.in[k][j] = b->field[k][p].as<float>();
            L.fs.out[k][j] = b->field[1 - k][p].as<float>();
        }
    L.mask = b->mask.as<uint8_t>();
    L.nn = b->nn.as<int32_t>();
    L.keys = b->keys.as<int64_t>();
    L.gid = b->gid.as<int32_t>();
    L.grids = b->grids.as<GridInfo>();
    L.n = b->n;
    L.arr_chunks = b->n;
    L.geo.edge = b->edge;
    L.geo.bs = b->edge * b->edge * b->edge;
    L.t = t;
    L.err = b->err.as<unsigned>();
    return launch_fields(L, s);
}

}  // namespace sgb

using namespace sgb;

extern "C" {

int sgb_batch_create(sgb_batch** out, int device) {
    if (!out) return SGB_EINVAL;
    DeviceGuard dg(device);
    SGB_CUDA(dg.status);
    sgb_batch* b = new sgb_batch();
    b->device = device;
    cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, device);
    if (b->err.ensure(16) != SGB_OK || cudaMemset(b->err.p, 0, 16) != cudaSuccess) {
        delete b;
        return SGB_ENOMEM;
    }
    *out = b;
    return SGB_OK;
}

int sgb_batch_destroy(sgb_batch* b) {
    if (!b) return SGB_EINVAL;
    DeviceGuard dg(b->device);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    for (int k = 0; k < 2; ++k) {
        if (b->grids_done[k]) {
            cudaEventSynchronize(b->grids_done[k]);
            cudaEventDestroy(b->grids_done[k]);
        }
        if (b->grids_host[k]) cudaFreeHost(b->grids_host[k]);
    }
    for (DevBuf* d : {&b->keys, &b->mask, &b->nn, &b->gid, &b->grids, &b->keys2, &b->mask2, &b->nn2, &b->gid2, &b->err})
        d->release();
    for (int k = 0; k < 2; ++k)
        for (int p = 0; p < 2; ++p) {
            b->field[k][p].release();
            b->field2[k][p].release();
        }
    delete b;
    return SGB_OK;
}

int sgb_batch_set_launch_config(sgb_batch* b, int ctas_per_sm, int stages) {
    if (!b || ctas_per_sm < -1 || ctas_per_sm > 16 || stages < -1 || (stages > 0 && (stages < 3 || stages > 16)))
        return SGB_EINVAL;
    if (ctas_per_sm) b->ctas_per_sm = ctas_per_sm < 0 ? 0 : ctas_per_sm;  // -1: automatic
    if (stages) b->stages = stages < 0 ? 0 : stages;  // -1: automatic depth
    return SGB_OK;
}

int sgb_batch_add(sgb_batch* b, sgb_grid* g, int kind, const int* src, const int* dst, const float* params,
                  int nparams, int64_t nsteps, int* slot, sgb_stream stream) {
    if (!b || !g || !slot || nsteps < 0) return SGB_EINVAL;
    if (kind != SGB_HEAT7 && kind != SGB_GS7) {
        set_error("batches run HEAT7 or GS7");
        return SGB_ENOTSUP;
    }
    if (g->geo.zorder) {
        set_error("batches hold grids with x-fastest chunk ids");
        return SGB_ENOTSUP;
    }
    if (b->kind >= 0 && (b->kind != kind || b->edge != g->geo.edge)) {
        set_error("all grids of a batch share the stencil kind and the chunk edge");
        return SGB_EINVAL;
    }
    cudaStream_t s = (cudaStream_t)stream;
    StencilParams prm;
    SGB_TRY(make_params(g, kind, src, dst, params, nparams, nullptr, prm));
    if (b->kind < 0) {
        b->kind = kind;
        b->edge = g->geo.edge;
        b->np = kind == SGB_GS7 ? 2 : 1;
    }
    SGB_TRY(batch_compact(b, s));
    SGB_TRY(ensure_neighbours(g, SGB_NN_STAR, s));
    for (int p = 0; p < b->np; ++p) {  // batched kernels rely on background-filled empty points
        SGB_TRY(ensure_clean(g, src[p], s));
        SGB_TRY(ensure_clean(g, dst[p], s));
    }
    const int bs = g->geo.bs;
    SGB_TRY(batch_reserve(b, b->n + g->n));
    const int64_t off = b->n;
    if (g->n > 0) {
        SGB_CUDA(cudaMemcpyAsync(b->keys.as<int64_t>() + off, g->keys.p, g->n * 8, cudaMemcpyDeviceToDevice, s));
        SGB_CUDA(cudaMemcpyAsync(b->mask.as<uint8_t>() + off * bs, g->mask.p, g->n * bs, cudaMemcpyDeviceToDevice, s));
        for (int p = 0; p < b->np; ++p) {
            SGB_CUDA(cudaMemcpyAsync(b->field[0][p].as<float>() + off * bs, g->data[src[p]].p, g->n * bs * 4,
                                     cudaMemcpyDeviceToDevice, s));
            SGB_CUDA(cudaMemcpyAsync(b->field[1][p].as<float>() + off * bs, g->data[dst[p]].p, g->n * bs * 4,
                                     cudaMemcpyDeviceToDevice, s));
        }
        k_offset_nn<<<(unsigned)((g->n * 8 + 255) / 256), 256, 0, s>>>(g->nn[0].as<int32_t>(),
                                                                        b->nn.as<int32_t>() + off * 8, g->n * 8, off);
        SGB_CUDA(cudaGetLastError());
    }
    sgb_batch::Slot sl;
    sl.live = true;
    sl.off = off;
    sl.n = g->n;
    sl.gi = grid_info_of(prm);
    sl.gi.start = b->T;
    sl.gi.nsteps = nsteps;
    for (int p = 0; p < b->np; ++p) {
        sl.src[p] = src[p];
        sl.dst[p] = dst[p];
    }
    // reuse a dead slot id when one is free
    int id = -1;
    for (size_t i = 0; i < b->slots.size(); ++i)
        if (!b->slots[i].live && b->slots[i].n == 0) {
            id = (int)i;
            break;
        }
    if (id < 0) {
        id = (int)b->slots.size();
        b->slots.push_back(sl);
    } else {
        b->slots[id] = sl;
    }
    if (g->n > 0) {
        k_fill_i32<<<(unsigned)((g->n + 255) / 256), 256, 0, s>>>(b->gid.as<int32_t>() + off, g->n, id);
        SGB_CUDA(cudaGetLastError());
    }
    b->n += g->n;
    b->dirty = true;
    *slot = id;
    return SGB_OK;
}

int sgb_batch_remove(sgb_batch* b, int slot, sgb_stream) {
    if (!b || slot < 0 || slot >= (int)b->slots.size() || !b->slots[slot].live) return SGB_EINVAL;
    b->slots[slot].live = false;
    b->slots[slot].gi.nsteps = 0;  // idle until compacted away
    b->holes = true;
    b->dirty = true;
    return SGB_OK;
}

int sgb_batch_step(sgb_batch* b, int nsteps, int use_graph, sgb_stream stream) {
    if (!b || nsteps < 0) return SGB_EINVAL;
    cudaStream_t s = (cudaStream_t)stream;
    SGB_TRY(batch_compact(b, s));
    SGB_TRY(batch_upload_grids(b, s));
    if (nsteps == 0) return SGB_OK;
    if (b->n == 0) {
        b->T += nsteps;
        return SGB_OK;
    }
    int st;
    if (use_graph) {
        // capture the nsteps launches, then update the cached executable graph in place (same shape:
        // only kernel arguments differ) or instantiate a new one; the launch does not wait for the GPU
        const int64_t T0 = b->T;
        cudaStream_t cap;
        SGB_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
        cudaGraph_t graph = nullptr;
        st = SGB_OK;
        cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            for (int k = 0; k < nsteps && st == SGB_OK; ++k) st = batch_launch(b, T0 + k, cap);
            const cudaError_t e2 = cudaStreamEndCapture(cap, &graph);
            if (st == SGB_OK && e2 != cudaSuccess) st = cuda_status(e2, "cudaStreamEndCapture");
        } else {
            st = cuda_status(e, "cudaStreamBeginCapture");
        }
        if (st == SGB_OK) {
            bool updated = false;
            if (b->exec && b->exec_nsteps == nsteps) {
                cudaGraphExecUpdateResultInfo info;
                updated = cudaGraphExecUpdate(b->exec, graph, &info) == cudaSuccess;
                if (!updated) cudaGetLastError();  // clear the update failure; instantiate instead
            }
            if (!updated) {
                if (b->exec) cudaGraphExecDestroy(b->exec);
                b->exec = nullptr;
                b->exec_nsteps = -1;
                e = cudaGraphInstantiate(&b->exec, graph, 0);
                if (e != cudaSuccess) {
                    b->exec = nullptr;
                    st = cuda_status(e, "cudaGraphInstantiate");
                } else {
                    b->exec_nsteps = nsteps;
                }
            }
            if (st == SGB_OK) {
                e = cudaGraphLaunch(b->exec, s);
                if (e != cudaSuccess) st = cuda_status(e, "cudaGraphLaunch");
            }
        }
        if (graph) cudaGraphDestroy(graph);
        cudaStreamDestroy(cap);
    } else {
        st = SGB_OK;
        for (int k = 0; k < nsteps && st == SGB_OK; ++k) st = batch_launch(b, b->T + k, s);
    }
    if (st == SGB_OK) b->T += nsteps;
    return st;
}

int sgb_batch_slot_steps(const sgb_batch* b, int slot, int64_t* done) {
    if (!b || !done || slot < 0 || slot >= (int)b->slots.size()) return SGB_EINVAL;
    const auto& sl = b->slots[slot];
    *done = std::max<int64_t>(0, std::min<int64_t>(b->T - sl.gi.start, sl.gi.nsteps));
    return SGB_OK;
}

int sgb_batch_extract(sgb_batch* b, int slot, sgb_grid* g, int* final_is_dst, sgb_stream stream) {
    if (!b || !g || slot < 0 || slot >= (int)b->slots.size() || !b->slots[slot].live) return SGB_EINVAL;
    const auto& sl = b->slots[slot];
    if (g->n != sl.n || g->geo.edge != b->edge) return SGB_EINVAL;
    cudaStream_t s = (cudaStream_t)stream;
    const int bs = g->geo.bs;
    int64_t done = 0;
    sgb_batch_slot_steps(b, slot, &done);
    if (final_is_dst) *final_is_dst = (int)(done & 1);
    // buffer 0 mirrors the src properties, buffer 1 the dst properties
    for (int p = 0; p < b->np; ++p) {
        if (sl.src[p] >= g->nprop || sl.dst[p] >= g->nprop) return SGB_EINVAL;
        SGB_CUDA(cudaMemcpyAsync(g->data[sl.src[p]].p, b->field[0][p].as<float>() + sl.off * bs, sl.n * bs * 4,
                                 cudaMemcpyDeviceToDevice, s));
        SGB_CUDA(cudaMemcpyAsync(g->data[sl.dst[p]].p, b->field[1][p].as<float>() + sl.off * bs, sl.n * bs * 4,
                                 cudaMemcpyDeviceToDevice, s));
    }
    return SGB_OK;
}

int sgb_batch_info(const sgb_batch* b, int* ngrids, int64_t* nchunks, int64_t* bytes) {
    if (!b) return SGB_EINVAL;
    int live = 0;
    for (auto& sl : b->slots) live += sl.live;
    if (ngrids) *ngrids = live;
    if (nchunks) *nchunks = b->n;
    if (bytes) {
        size_t t = b->keys.bytes + b->mask.bytes + b->nn.bytes + b->gid.bytes + b->grids.bytes + b->keys2.bytes +
                   b->mask2.bytes + b->nn2.bytes + b->gid2.bytes;
        for (int k = 0; k < 2; ++k)
            for (int p = 0; p < 2; ++p) t += b->field[k][p].bytes + b->field2[k][p].bytes;
        *bytes = (int64_t)t;
    }
    return SGB_OK;
}

}  // extern "C"

static int batch_read(sgb_batch* b, int slot, int64_t* keys, uint8_t* mask, float* const* fields, int64_t* nchunks,
                      sgb_stream stream, bool wait) {
    if (!b || slot < 0 || slot >= (int)b->slots.size() || !b->slots[slot].live) return SGB_EINVAL;
    const auto& sl = b->slots[slot];
    cudaStream_t s = (cudaStream_t)stream;
    const int bs = b->edge * b->edge * b->edge;
    if (nchunks) *nchunks = sl.n;
    int64_t done = 0;
    sgb_batch_slot_steps(b, slot, &done);
    const int cur = (int)(done & 1);  // buffer holding the latest state
    if (sl.n > 0) {
        if (keys) SGB_CUDA(cudaMemcpyAsync(keys, b->keys.as<int64_t>() + sl.off, sl.n * 8, cudaMemcpyDeviceToHost, s));
        if (mask) SGB_CUDA(cudaMemcpyAsync(mask, b->mask.as<uint8_t>() + sl.off * bs, sl.n * bs, cudaMemcpyDeviceToHost, s));
        if (fields)
            for (int p = 0; p < b->np; ++p)
                if (fields[p])
                    SGB_CUDA(cudaMemcpyAsync(fields[p], b->field[cur][p].as<float>() + sl.off * bs, sl.n * bs * 4,
                                             cudaMemcpyDeviceToHost, s));
    }
    if (wait) SGB_CUDA(cudaStreamSynchronize(s));
    return SGB_OK;
}

extern "C" int sgb_batch_read(sgb_batch* b, int slot, int64_t* keys, uint8_t* mask, float* const* fields,
                              int64_t* nchunks, sgb_stream stream) {
    return batch_read(b, slot, keys, mask, fields, nchunks, stream, true);
}

extern "C" int sgb_batch_read_async(sgb_batch* b, int slot, int64_t* keys, uint8_t* mask, float* const* fields,
                                    int64_t* nchunks, sgb_stream stream) {
    return batch_read(b, slot, keys, mask, fields, nchunks, stream, false);
}
