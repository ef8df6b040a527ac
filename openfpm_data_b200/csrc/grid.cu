// Grid handles, buffers, map upload/download, staged inserts and point reads.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>

#include <cuda.h>

#include "common.cuh"
#include "internal.h"

namespace sgb {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

int cuda_status(cudaError_t e, const char* what) {
    set_error(std::string(what) + ": " + cudaGetErrorString(e));
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        return SGB_ENOMEM;
    }
    return SGB_ECUDA;
}

// Driver calls for growth in place (virtual memory management), looked up through the runtime so that
// the library does not link the driver library itself.
namespace {
struct VmmApi {
    CUresult (*reserve)(CUdeviceptr*, size_t, size_t, CUdeviceptr, unsigned long long) = nullptr;
    CUresult (*free_va)(CUdeviceptr, size_t) = nullptr;
    CUresult (*create)(CUmemGenericAllocationHandle*, size_t, const CUmemAllocationProp*, unsigned long long) =
        nullptr;
    CUresult (*release)(CUmemGenericAllocationHandle) = nullptr;
    CUresult (*map)(CUdeviceptr, size_t, size_t, CUmemGenericAllocationHandle, unsigned long long) = nullptr;
    CUresult (*unmap)(CUdeviceptr, size_t) = nullptr;
    CUresult (*access)(CUdeviceptr, size_t, const CUmemAccessDesc*, size_t) = nullptr;
    CUresult (*granularity)(size_t*, const CUmemAllocationProp*, CUmemAllocationGranularity_flags) = nullptr;
    bool ok = false;
};
const VmmApi& vmm() {
    static VmmApi api = [] {
        VmmApi a;
        auto get = [](const char* name, void** fn) {
            cudaDriverEntryPointQueryResult q;
            return cudaGetDriverEntryPointByVersion(name, fn, 12000, cudaEnableDefault, &q) == cudaSuccess &&
                   q == cudaDriverEntryPointSuccess && *fn != nullptr;
        };
        a.ok = get("cuMemAddressReserve", (void**)&a.reserve) && get("cuMemAddressFree", (void**)&a.free_va) &&
               get("cuMemCreate", (void**)&a.create) && get("cuMemRelease", (void**)&a.release) &&
               get("cuMemMap", (void**)&a.map) && get("cuMemUnmap", (void**)&a.unmap) &&
               get("cuMemSetAccess", (void**)&a.access) &&
               get("cuMemGetAllocationGranularity", (void**)&a.granularity);
        return a;
    }();
    return api;
}
CUmemAllocationProp device_prop(int dev) {
    CUmemAllocationProp prop = {};
    prop.type = CU_MEM_ALLOCATION_TYPE_PINNED;
    prop.location.type = CU_MEM_LOCATION_TYPE_DEVICE;
    prop.location.id = dev;
    return prop;
}
// map `size` bytes of new physical memory of device `dev` at `at`; the handle goes to `maps`
int map_more(const VmmApi& api, int dev, unsigned long long at, size_t size,
             std::vector<std::pair<unsigned long long, size_t>>& maps) {
    const CUmemAllocationProp prop = device_prop(dev);
    CUmemGenericAllocationHandle h = 0;
    if (api.create(&h, size, &prop, 0) != CUDA_SUCCESS) {
        set_error("cuMemCreate: out of device memory");
        return SGB_ENOMEM;
    }
    if (api.map((CUdeviceptr)at, size, 0, h, 0) != CUDA_SUCCESS) {
        api.release(h);
        set_error("cuMemMap failed");
        return SGB_ECUDA;
    }
    CUmemAccessDesc acc = {};
    acc.location = prop.location;
    acc.flags = CU_MEM_ACCESS_FLAGS_PROT_READWRITE;
    if (api.access((CUdeviceptr)at, size, &acc, 1) != CUDA_SUCCESS) {
        api.unmap((CUdeviceptr)at, size);
        api.release(h);
        set_error("cuMemSetAccess failed");
        return SGB_ECUDA;
    }
    maps.emplace_back((unsigned long long)h, size);
    return SGB_OK;
}
// unmap and release every mapping of a reserved range, then the range
void unmap_all(const VmmApi& api, unsigned long long va, size_t va_bytes,
               std::vector<std::pair<unsigned long long, size_t>>& maps) {
    size_t off = 0;
    for (auto& m : maps) {
        api.unmap((CUdeviceptr)(va + off), m.second);
        api.release((CUmemGenericAllocationHandle)m.first);
        off += m.second;
    }
    maps.clear();
    if (va) api.free_va((CUdeviceptr)va, va_bytes);
}
}  // namespace

// a buffer from cudaMalloc grown by allocating a larger one and copying the contents over
static int realloc_copy(DevBuf& b, size_t need) {
    size_t nb = need + need / 2 + 256;
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, nb);
    if (e != cudaSuccess) return cuda_status(e, "cudaMalloc");
    if (b.p && b.bytes) {
        // work queued on any stream may still write the old buffer
        e = cudaDeviceSynchronize();
        if (e == cudaSuccess) e = cudaMemcpy(q, b.p, b.bytes, cudaMemcpyDeviceToDevice);
        if (e != cudaSuccess) {
            cudaFree(q);
            return cuda_status(e, "cudaMemcpy(grow)");
        }
    }
    if (b.p) cudaFree(b.p);
    b.p = q;
    b.bytes = nb;
    return SGB_OK;
}

int DevBuf::grow_in_place(size_t need) {
    if (need <= bytes) return SGB_OK;
    if (!va && need < kInPlaceMinBytes) return realloc_copy(*this, need);
    const VmmApi& api = vmm();
    if (!api.ok) {
        if (va) return SGB_ECUDA;      // cannot happen: the range was made through the same calls
        return realloc_copy(*this, need);  // no driver support: reallocate and copy
    }
    int dev = 0;
    SGB_CUDA(cudaGetDevice(&dev));
    const CUmemAllocationProp prop = device_prop(dev);
    size_t gran = 0;
    if (api.granularity(&gran, &prop, CU_MEM_ALLOC_GRANULARITY_RECOMMENDED) != CUDA_SUCCESS || gran == 0) {
        if (va) {
            set_error("cuMemGetAllocationGranularity failed");
            return SGB_ECUDA;
        }
        return realloc_copy(*this, need);
    }
    auto round_up = [gran](size_t x) { return (x + gran - 1) / gran * gran; };
    const size_t target = round_up(std::max(need, bytes + bytes / 2));
    if (va && target <= va_bytes) {  // map the difference behind the current end
        SGB_TRY(map_more(api, dev, va + bytes, target - bytes, maps));
        bytes = target;
        return SGB_OK;
    }
    // a new range with room for eight times the target (at least 4 GiB, at most the device's memory),
    // the contents copied over once
    size_t total = 0, free_b = 0;
    SGB_CUDA(cudaMemGetInfo(&free_b, &total));
    size_t want = std::max(target * 8, size_t(4) << 30);
    want = std::max(target, std::min(want, round_up(total)));
    want = round_up(want);
    CUdeviceptr nva = 0;
    if (api.reserve(&nva, want, 0, 0, 0) != CUDA_SUCCESS) {
        set_error("cuMemAddressReserve failed");
        return SGB_ENOMEM;
    }
    std::vector<std::pair<unsigned long long, size_t>> nmaps;
    int st = map_more(api, dev, (unsigned long long)nva, target, nmaps);
    if (st == SGB_OK && p && bytes) {
        // work queued on any stream may still write the old buffer
        cudaError_t e = cudaDeviceSynchronize();
        if (e == cudaSuccess) e = cudaMemcpy((void*)nva, p, bytes, cudaMemcpyDeviceToDevice);
        if (e != cudaSuccess) st = cuda_status(e, "cudaMemcpy(grow)");
    }
    if (st != SGB_OK) {
        unmap_all(api, (unsigned long long)nva, want, nmaps);
        return st;
    }
    release();
    va = (unsigned long long)nva;
    va_bytes = want;
    maps = std::move(nmaps);
    p = (void*)nva;
    bytes = target;
    return SGB_OK;
}

int DevBuf::reserve(size_t need) {
    if (need <= bytes) return SGB_OK;
    if (va || need >= kInPlaceMinBytes) return grow_in_place(need);
    return realloc_copy(*this, need);
}

// Tables that follow a growing map (neighbour tables, bitmaps, point lists) are small next to it, so
// they grow to four times the need: a growing map reallocates them, with the device sync of cudaFree,
// half as often as at twice the need.
int DevBuf::grow(size_t need) { return need <= bytes ? SGB_OK : ensure(4 * need); }

int DevBuf::ensure(size_t need) {
    if (need <= bytes) return SGB_OK;
    if (va) return grow_in_place(need);
    if (need >= kInPlaceMinBytes) {
        release();  // nothing to keep: the new range starts empty
        return grow_in_place(need);
    }
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    size_t nb = need + need / 4 + 256;
    cudaError_t e = cudaMalloc(&p, nb);
    if (e != cudaSuccess) {
        p = nullptr;
        return cuda_status(e, "cudaMalloc");
    }
    bytes = nb;
    return SGB_OK;
}

void DevBuf::release() {
    if (va) {
        // in-place buffers may still be read by queued work, as cudaFree would wait for
        cudaDeviceSynchronize();
        unmap_all(vmm(), va, va_bytes, maps);
        va = 0;
        va_bytes = 0;
    } else if (p) {
        cudaFree(p);
    }
    p = nullptr;
    bytes = 0;
}

int HostScratch::ensure(size_t need) {
    if (need <= bytes) return SGB_OK;
    if (p) cudaFreeHost(p);
    p = nullptr;
    bytes = 0;
    cudaError_t e = cudaMallocHost(&p, need);
    if (e != cudaSuccess) return cuda_status(e, "cudaMallocHost");
    bytes = need;
    return SGB_OK;
}

void HostScratch::release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    bytes = 0;
}

// Fill `count` elements of `esize` bytes with one pattern.
__global__ void k_fill(unsigned char* dst, int64_t count, int esize, uint64_t pattern) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; i < count; i += stride) {
        if (esize == 4) reinterpret_cast<uint32_t*>(dst)[i] = (uint32_t)pattern;
        else if (esize == 8) reinterpret_cast<uint64_t*>(dst)[i] = pattern;
        else dst[i] = (unsigned char)pattern;
    }
}

int fill(void* dst, int64_t count, int esize, uint64_t pattern, cudaStream_t s) {
    if (count <= 0) return SGB_OK;
    int64_t blocks = (count + 255) / 256;
    if (blocks > 4096) blocks = 4096;
    k_fill<<<(unsigned)blocks, 256, 0, s>>>((unsigned char*)dst, count, esize, pattern);
    SGB_CUDA(cudaGetLastError());
    return SGB_OK;
}

uint64_t bck_pattern(const sgb_grid* g, int p) {
    uint64_t v = 0;
    std::memcpy(&v, g->bck[p], elem_size(g->ptype[p]));
    return v;
}

int write_background(sgb_grid* g, int64_t pos, cudaStream_t s, DevBuf* data, DevBuf& mask) {
    const int bs = g->geo.bs;
    for (int p = 0; p < g->nprop; ++p) {
        int es = elem_size(g->ptype[p]);
        SGB_TRY(fill(data[p].as<unsigned char>() + (size_t)pos * bs * es, bs, es, bck_pattern(g, p), s));
    }
    SGB_CUDA(cudaMemsetAsync(mask.as<unsigned char>() + (size_t)pos * bs, 0, bs, s));
    return SGB_OK;
}

int grid_reserve(sgb_grid* g, int64_t chunks, bool keep) {
    if (chunks <= g->cap && g->keys.p) return SGB_OK;
    int64_t nc = chunks;
    if (nc < g->cap + g->cap / 2) nc = g->cap + g->cap / 2;
    if (nc < 16) nc = 16;
    const int bs = g->geo.bs;
    if (keep) {
        SGB_TRY(g->keys.reserve((size_t)nc * 8));
        for (int p = 0; p < g->nprop; ++p)
            SGB_TRY(g->data[p].reserve((size_t)(nc + 1) * bs * elem_size(g->ptype[p])));
        SGB_TRY(g->mask.reserve((size_t)(nc + 1) * bs));
    } else {
        SGB_TRY(g->keys.ensure((size_t)nc * 8));
        for (int p = 0; p < g->nprop; ++p)
            SGB_TRY(g->data[p].ensure((size_t)(nc + 1) * bs * elem_size(g->ptype[p])));
        SGB_TRY(g->mask.ensure((size_t)(nc + 1) * bs));
    }
    g->cap = nc;
    return SGB_OK;
}

static void invalidate_derived(sgb_grid* g) {
    g->nn_valid[0] = g->nn_valid[1] = false;
    g->nnhash_ok = false;
    g->bits_valid = false;
    g->epts_valid = false;
}

// Points whose mask byte is 0 take the background value: 16 mask bytes per
// thread step, element stores only where needed.
template <typename T>
__global__ void k_sanitize(const uint8_t* mask, T* data, int64_t total, T bck) {
    const int64_t words = total / 16;
    for (int64_t w = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; w < words; w += (int64_t)gridDim.x * blockDim.x) {
        const uint4 m = reinterpret_cast<const uint4*>(mask)[w];
        const unsigned mw[4] = {m.x, m.y, m.z, m.w};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            if (mw[q] == 0x01010101u) continue;
#pragma unroll
            for (int b = 0; b < 4; ++b)
                if (((mw[q] >> (8 * b)) & 0xffu) == 0) data[w * 16 + q * 4 + b] = bck;
        }
    }
}

int sanitize_prop(sgb_grid* g, int p, cudaStream_t s) {
    const int64_t total = g->n * (int64_t)g->geo.bs;  // bs is a multiple of 16
    if (total > 0) {
        const unsigned blocks = (unsigned)std::min<int64_t>(8192, (total / 16 + 255) / 256);
        const uint8_t* m = g->mask.as<uint8_t>();
        switch (elem_size(g->ptype[p])) {
            case 1: k_sanitize<uint8_t><<<blocks, 256, 0, s>>>(m, g->data[p].as<uint8_t>(), total, (uint8_t)bck_pattern(g, p)); break;
            case 4: k_sanitize<uint32_t><<<blocks, 256, 0, s>>>(m, g->data[p].as<uint32_t>(), total, (uint32_t)bck_pattern(g, p)); break;
            default: k_sanitize<uint64_t><<<blocks, 256, 0, s>>>(m, g->data[p].as<uint64_t>(), total, bck_pattern(g, p)); break;
        }
        SGB_CUDA(cudaGetLastError());
    }
    g->clean[p] = true;
    return SGB_OK;
}

int ensure_clean(sgb_grid* g, int p, cudaStream_t s) { return g->clean[p] ? SGB_OK : sanitize_prop(g, p, s); }

int fill_background_all(sgb_grid* g, int p, cudaStream_t s) {
    const int es = elem_size(g->ptype[p]);
    SGB_TRY(fill(g->data[p].p, (g->n + 1) * g->geo.bs, es, bck_pattern(g, p), s));
    g->clean[p] = true;
    return SGB_OK;
}

// grid_smb::LinId / grid_zmb::LinId on device (src/Grid/Geometry/
// grid_smb.hpp:176-190, grid_zmb.hpp:63-76), with a domain check that the
// reference does not do.
__global__ void k_lin_from_coords(const int32_t* coords, int64_t n, Geometry geo, int64_t* lin, unsigned* err) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    int64_t c[3];
    bool ok = true;
    for (int d = 0; d < geo.dim; ++d) {
        c[d] = coords[i * geo.dim + d];
        ok &= c[d] >= 0 && c[d] < geo.size[d];
    }
    if (!ok) {
        atomicOr(err, kErrOutOfDomain);
        lin[i] = -1;
        return;
    }
    int64_t b, l;
    point_key(geo, c, &b, &l);
    lin[i] = b * geo.bs + l;
}

__global__ void k_check_lin(const int64_t* lin_in, int64_t n, Geometry geo, int64_t* lin_out, unsigned* err) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    int64_t v = lin_in[i];
    if (v < 0 || !key_in_domain(geo, v / geo.bs)) {
        atomicOr(err, kErrOutOfDomain);
        v = -1;
    }
    lin_out[i] = v;
}

static int stage_values(sgb_grid* g, int64_t n, const void* const* values, cudaStream_t s) {
    for (int p = 0; p < g->nprop; ++p) {
        const int es = elem_size(g->ptype[p]);
        SGB_TRY(g->pend_val[p].reserve((size_t)(g->npend + n) * es));
        unsigned char* dst = g->pend_val[p].as<unsigned char>() + (size_t)g->npend * es;
        if (values && values[p]) {
            SGB_CUDA(cudaMemcpyAsync(dst, values[p], (size_t)n * es, cudaMemcpyDeviceToDevice, s));
            g->pend_has[p] = true;
        } else {
            SGB_TRY(fill(dst, n, es, bck_pattern(g, p), s));
        }
    }
    return SGB_OK;
}

template <typename T>
__global__ void k_get(const int32_t* coords, int64_t n, Geometry geo, const int64_t* keys, int64_t nchunks,
                      const T* data, const uint8_t* mask, T* out) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    int64_t c[3] = {0, 0, 0};
    bool inside = true;
    for (int d = 0; d < geo.dim; ++d) {
        c[d] = coords[i * geo.dim + d];
        inside &= c[d] >= 0 && c[d] < geo.size[d];
    }
    if (!inside) {  // outside the domain: the background
        out[i] = data[(size_t)nchunks * geo.bs];
        return;
    }
    int64_t b, l;
    point_key(geo, c, &b, &l);
    int64_t pos = find_key(keys, nchunks, b);
    if (pos < 0) pos = nchunks;
    // BlockMapGpu_ker::get (src/SparseGridGpu/BlockMapGpu_ker.cuh:117-135)
    const size_t idx = (size_t)pos * geo.bs + l;
    out[i] = (mask[idx] & 1) ? data[idx] : data[(size_t)nchunks * geo.bs + l];
}

// Pool counts clamped to the pool capacity (an overflowing pool raises the
// out-of-domain error word: its extra inserts had nowhere to go).
__global__ void k_clamp_counts(const int32_t* counts, int64_t npools, int32_t nslot, uint32_t* out, unsigned* err) {
    int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (b >= npools) return;
    int32_t c = counts[b];
    if (c < 0 || c > nslot) {
        atomicOr(err, kErrPoolOverflow);
        c = c < 0 ? 0 : nslot;
    }
    out[b] = (uint32_t)c;
}

struct PoolCopy {
    const unsigned char* src[kMaxProps];
    unsigned char* dst[kMaxProps];
    int es[kMaxProps];
    uint64_t bck[kMaxProps];
    int nprop;
};

// One CTA per pool: its first counts[b] slots, in slot order, after the
// pools before it.
__global__ void k_pool_copy(const uint32_t* counts, const uint32_t* off, int64_t nslot, const int64_t* lin,
                            Geometry geo, int64_t* out_lin, PoolCopy pc, unsigned* err) {
    const int64_t b = blockIdx.x;
    const uint32_t c = counts[b], o = off[b];
    for (uint32_t k = threadIdx.x; k < c; k += blockDim.x) {
        const int64_t src = b * nslot + k, dst = (int64_t)o + k;
        int64_t v = lin[src];
        if (v < 0 || !key_in_domain(geo, v / geo.bs)) {
            atomicOr(err, kErrOutOfDomain);
            v = -1;
        }
        out_lin[dst] = v;
        for (int p = 0; p < pc.nprop; ++p) {
            const int es = pc.es[p];
            unsigned char* d = pc.dst[p] + dst * es;
            if (pc.src[p]) {
                for (int q = 0; q < es; ++q) d[q] = pc.src[p][src * es + q];
            } else {
                for (int q = 0; q < es; ++q) d[q] = (unsigned char)(pc.bck[p] >> (8 * q));
            }
        }
    }
}

// EXIST points per chunk: one warp per chunk, one ballot per 32 mask bytes
// (calc_exist_points, SparseGridGpu_kernels.cuh:1194-1225).
__global__ void k_chunk_counts(const uint8_t* mask, int64_t n, int bs, uint32_t* counts) {
    const int64_t chunk = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (chunk >= n) return;
    const uint8_t* m = mask + (size_t)chunk * bs;
    uint32_t c = 0;
    for (int r = 0; r < bs / 32; ++r) c += __popc(__ballot_sync(0xffffffffu, m[r * 32 + lane] & 1));
    if (lane == 0) counts[chunk] = c;
}

__global__ void k_offsets_i64(const uint32_t* scanned, const uint32_t* total, int64_t n, int64_t* out) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) out[i] = scanned[i];
    else if (i == n) out[n] = *total;
}

__global__ void k_count(const uint8_t* mask, int64_t total, unsigned long long* out) {
    unsigned long long e = 0, p = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        uint8_t m = mask[i];
        e += m & 1;
        p += (m & 1) && (m & 2);
    }
    for (int o = 16; o > 0; o >>= 1) {
        e += __shfl_down_sync(0xffffffffu, e, o);
        p += __shfl_down_sync(0xffffffffu, p, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(out, e);
        atomicAdd(out + 1, p);
    }
}

// Points of the chunk slots written through insertBlock: per slot (pool b,
// slot k below the pool's clamped count) the number of mask bytes with EXIST
// set; one warp per slot, one ballot per 32 mask bytes.
__global__ void k_block_counts(const uint32_t* pool_counts, int64_t npools, int64_t nslot, const uint8_t* masks,
                               int bs, uint32_t* out) {
    const int64_t slot = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (slot >= npools * nslot) return;
    const int64_t b = slot / nslot, k = slot % nslot;
    uint32_t c = 0;
    if (k < (int64_t)pool_counts[b]) {
        const uint8_t* m = masks + slot * bs;
        for (int r = 0; r < bs; r += 32) {
            const bool e = r + lane < bs && (m[r + lane] & 1);
            c += __popc(__ballot_sync(0xffffffffu, e));
        }
    }
    if (lane == 0) out[slot] = c;
}

// Emit every EXIST point of every counted slot, in (pool, slot, offset) order,
// as a staged insert: linear id key * bs + offset and the slot's values.
__global__ void k_block_emit(const uint32_t* pool_counts, int64_t npools, int64_t nslot, const int64_t* keys,
                             const uint8_t* masks, const uint32_t* off, Geometry geo, int64_t* out_lin, PoolCopy pc,
                             unsigned* err) {
    const int64_t slot = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (slot >= npools * nslot) return;
    const int64_t b = slot / nslot, k = slot % nslot;
    if (k >= (int64_t)pool_counts[b]) return;
    const int bs = geo.bs;
    int64_t key = keys[slot];
    const bool key_ok = key >= 0 && key_in_domain(geo, key);
    const uint8_t* m = masks + slot * bs;
    uint32_t w = off[slot];
    for (int r = 0; r < bs; r += 32) {
        const int o = r + lane;
        const bool e = o < bs && (m[o] & 1);
        const unsigned bal = __ballot_sync(0xffffffffu, e);
        if (e) {
            const int64_t dst = (int64_t)w + __popc(bal & lanemask_lt());
            if (!key_ok) atomicOr(err, kErrOutOfDomain);
            out_lin[dst] = key_ok ? key * bs + o : -1;
            const int64_t src = slot * bs + o;
            for (int p = 0; p < pc.nprop; ++p) {
                const int es = pc.es[p];
                unsigned char* d = pc.dst[p] + dst * es;
                if (pc.src[p]) {
                    for (int q = 0; q < es; ++q) d[q] = pc.src[p][src * es + q];
                } else {
                    for (int q = 0; q < es; ++q) d[q] = (unsigned char)(pc.bck[p] >> (8 * q));
                }
            }
        }
        w += __popc(bal);
    }
}

}  // namespace sgb

using namespace sgb;

extern "C" {

const char* sgb_status_string(int s) {
    switch (s) {
        case SGB_OK: return "ok";
        case SGB_EINVAL: return "invalid argument";
        case SGB_ECUDA: return "CUDA error";
        case SGB_ENOMEM: return "out of device memory";
        case SGB_ERANGE: return "point outside the grid domain";
        case SGB_ESTATE: return "invalid state";
        case SGB_ETIMEOUT: return "device wait timed out";
        case SGB_ENOTSUP: return "not supported";
        default: return "unknown status";
    }
}

const char* sgb_last_error_string(void) { return g_last_error.c_str(); }

int sgb_version(void) { return 10000; }

int sgb_create(sgb_grid** out, int dim, int edge, const int64_t* size, int nprop, const int* prop_types, int device) {
    if (!out || !size || (nprop > 0 && !prop_types)) return SGB_EINVAL;
    *out = nullptr;
    if (dim != 3) {
        set_error("only dim == 3 grids are supported on the device");
        return SGB_ENOTSUP;
    }
    if (edge != 4 && edge != 8) {
        set_error("chunk edge must be 4 or 8");
        return SGB_ENOTSUP;
    }
    if (nprop < 1 || nprop > kMaxProps) return SGB_EINVAL;
    for (int p = 0; p < nprop; ++p)
        if (prop_types[p] < SGB_F32 || prop_types[p] > SGB_U8) return SGB_EINVAL;
    for (int d = 0; d < dim; ++d)
        if (size[d] <= 0) return SGB_EINVAL;
    DeviceGuard dg(device);
    SGB_CUDA(dg.status);
    sgb_grid* g = new sgb_grid();
    g->device = device;
    g->geo.dim = dim;
    g->geo.edge = edge;
    g->geo.bs = edge * edge * edge;
    for (int d = 0; d < 3; ++d) {
        g->geo.size[d] = d < dim ? size[d] : 1;
        g->geo.bsz[d] = g->geo.size[d] / edge + ((g->geo.size[d] % edge) != 0);  // grid_smb.hpp:48-57
    }
    g->nprop = nprop;
    for (int p = 0; p < nprop; ++p) g->ptype[p] = prop_types[p];
    cudaDeviceGetAttribute(&g->num_sms, cudaDevAttrMultiProcessorCount, device);
    int st = grid_reserve(g, 16, false);
    if (st == SGB_OK) st = g->err.ensure(16);
    if (st == SGB_OK && cudaMemset(g->err.p, 0, 16) != cudaSuccess) st = SGB_ECUDA;
    if (st == SGB_OK) st = write_background(g, 0, 0, g->data, g->mask);
    if (st == SGB_OK) st = cudaDeviceSynchronize() == cudaSuccess ? SGB_OK : SGB_ECUDA;
    if (st != SGB_OK) {
        sgb_destroy(g);
        return st;
    }
    *out = g;
    return SGB_OK;
}

int sgb_destroy(sgb_grid* g) {
    if (!g) return SGB_EINVAL;
    DeviceGuard dg(g->device);
    g->keys.release();
    g->keys2.release();
    g->mask.release();
    g->mask2.release();
    for (int p = 0; p < kMaxProps; ++p) {
        g->data[p].release();
        g->data2[p].release();
        g->pend_val[p].release();
    }
    g->pend_lin.release();
    g->nn[0].release();
    g->nn[1].release();
    g->nnhash.release();
    g->bits.release();
    g->epts.release();
    for (auto& L : g->links) {
        L.pad_pos.release();
        L.pad_off.release();
        L.scan.release();
        L.pos.release();
        L.off.release();
    }
    for (auto& b : g->scratch) b.release();
    g->hscratch.release();
    g->err.release();
    delete g;
    return SGB_OK;
}

int sgb_existence_changed(sgb_grid* g) {
    if (!g) return SGB_EINVAL;
    g->bits_valid = false;
    g->epts_valid = false;
    return SGB_OK;
}

int sgb_release_scratch(sgb_grid* g) {
    if (!g) return SGB_EINVAL;
    DeviceGuard dg(g->device);
    SGB_CUDA(dg.status);
    SGB_CUDA(cudaDeviceSynchronize());  // no kernel of this grid may still use the buffers
    g->keys2.release();
    g->mask2.release();
    for (int p = 0; p < kMaxProps; ++p) {
        g->data2[p].release();
        if (g->npend == 0) g->pend_val[p].release();
    }
    if (g->npend == 0) g->pend_lin.release();
    g->bits.release();
    g->bits_valid = false;
    g->epts.release();
    g->epts_valid = false;
    g->nnhash.release();
    g->nnhash_ok = false;
    for (auto& b : g->scratch) b.release();
    return SGB_OK;
}

int sgb_set_background(sgb_grid* g, int prop, const void* value) {
    if (!g || !value || prop < 0 || prop >= g->nprop) return SGB_EINVAL;
    std::memcpy(g->bck[prop], value, elem_size(g->ptype[prop]));
    const int bs = g->geo.bs, es = elem_size(g->ptype[prop]);
    SGB_TRY(fill(g->data[prop].as<unsigned char>() + (size_t)g->n * bs * es, bs, es, bck_pattern(g, prop), 0));
    SGB_TRY(sanitize_prop(g, prop, 0));  // points without EXIST read the new background
    SGB_CUDA(cudaStreamSynchronize(0));
    return SGB_OK;
}

int sgb_insert(sgb_grid* g, int64_t n, const int32_t* coords, const void* const* values, sgb_stream stream) {
    if (!g || n < 0 || (n > 0 && !coords)) return SGB_EINVAL;
    if (n == 0) return SGB_OK;
    cudaStream_t s = (cudaStream_t)stream;
    SGB_TRY(g->pend_lin.reserve((size_t)(g->npend + n) * 8));
    k_lin_from_coords<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(coords, n, g->geo,
                                                                   g->pend_lin.as<int64_t>() + g->npend,
                                                                   g->err.as<unsigned>());
    SGB_CUDA(cudaGetLastError());
    SGB_TRY(stage_values(g, n, values, s));
    g->npend += n;
    return SGB_OK;
}

int sgb_insert_lin(sgb_grid* g, int64_t n, const int64_t* lin, const void* const* values, sgb_stream stream) {
    if (!g || n < 0 || (n > 0 && !lin)) return SGB_EINVAL;
    if (n == 0) return SGB_OK;
    cudaStream_t s = (cudaStream_t)stream;
    SGB_TRY(g->pend_lin.reserve((size_t)(g->npend + n) * 8));
    k_check_lin<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(lin, n, g->geo, g->pend_lin.as<int64_t>() + g->npend,
                                                             g->err.as<unsigned>());
    SGB_CUDA(cudaGetLastError());
    SGB_TRY(stage_values(g, n, values, s));
    g->npend += n;
    return SGB_OK;
}

int sgb_insert_pools(sgb_grid* g, int64_t npools, int64_t nslot, const int32_t* counts, const int64_t* lin,
                     const void* const* values, sgb_stream stream) {
    if (!g || npools < 0 || nslot < 0 || (npools > 0 && (!counts || !lin))) return SGB_EINVAL;
    if (npools == 0) return SGB_OK;
    cudaStream_t s = (cudaStream_t)stream;
    DevBuf& cnt = g->scratch[9];
    DevBuf& off = g->scratch[10];
    SGB_TRY(cnt.ensure((size_t)npools * 4 + 16));
    SGB_TRY(off.ensure((size_t)npools * 4 + 16));
    k_clamp_counts<<<(unsigned)((npools + 255) / 256), 256, 0, s>>>(counts, npools, (int32_t)nslot, cnt.as<uint32_t>(),
                                                                     g->err.as<unsigned>());
    SGB_CUDA(cudaGetLastError());
    uint32_t* total = off.as<uint32_t>() + npools;
    SGB_TRY(scan_exclusive_u32(cnt.as<uint32_t>(), off.as<uint32_t>(), npools, total, &g->scratch[6], s));
    SGB_TRY(g->hscratch.ensure(64));
    SGB_CUDA(cudaMemcpyAsync(g->hscratch.p, total, 4, cudaMemcpyDeviceToHost, s));
    SGB_CUDA(cudaStreamSynchronize(s));
    const int64_t add = *(uint32_t*)g->hscratch.p;
    if (add == 0) return SGB_OK;
    SGB_TRY(g->pend_lin.reserve((size_t)(g->npend + add) * 8));
    PoolCopy pc{};
    pc.nprop = g->nprop;
    for (int p = 0; p < g->nprop; ++p) {
        const int es = elem_size(g->ptype[p]);
        SGB_TRY(g->pend_val[p].reserve((size_t)(g->npend + add) * es));
        pc.src[p] = values ? (const unsigned char*)values[p] : nullptr;
        if (pc.src[p]) g->pend_has[p] = true;
        pc.dst[p] = g->pend_val[p].as<unsigned char>() + (size_t)g->npend * es;
        pc.es[p] = es;
        pc.bck[p] = bck_pattern(g, p);
    }
    k_pool_copy<<<(unsigned)npools, 128, 0, s>>>(cnt.as<uint32_t>(), off.as<uint32_t>(), nslot, lin, g->geo,
                                                 g->pend_lin.as<int64_t>() + g->npend, pc, g->err.as<unsigned>());
    SGB_CUDA(cudaGetLastError());
    g->npend += add;
    return SGB_OK;
}

int sgb_insert_blocks(sgb_grid* g, int64_t npools, int64_t nslot, const int32_t* counts, const int64_t* keys,
                      const void* const* values, const uint8_t* masks, sgb_stream stream) {
    if (!g || npools < 0 || nslot <= 0 || nslot > (1 << 30) || (npools > 0 && (!counts || !keys || !masks)))
        return SGB_EINVAL;
    if (npools == 0) return SGB_OK;
    const int64_t nslots = npools * nslot;
    if (nslots * (int64_t)g->geo.bs >= (int64_t(1) << 32)) {
        set_error("sgb_insert_blocks: the block pools hold at most 2^32 - 1 chunk points");
        return SGB_ERANGE;
    }
    cudaStream_t s = (cudaStream_t)stream;
    DevBuf& cnt = g->scratch[9];
    DevBuf& per = g->scratch[7];
    DevBuf& off = g->scratch[8];
    SGB_TRY(cnt.ensure((size_t)npools * 4 + 16));
    SGB_TRY(per.ensure((size_t)nslots * 4 + 16));
    SGB_TRY(off.ensure((size_t)nslots * 4 + 16));
    k_clamp_counts<<<(unsigned)((npools + 255) / 256), 256, 0, s>>>(counts, npools, (int32_t)nslot, cnt.as<uint32_t>(),
                                                                     g->err.as<unsigned>());
    const unsigned wblocks = (unsigned)((nslots * 32 + 255) / 256);
    k_block_counts<<<wblocks, 256, 0, s>>>(cnt.as<uint32_t>(), npools, nslot, masks, g->geo.bs, per.as<uint32_t>());
    SGB_CUDA(cudaGetLastError());
    uint32_t* total = off.as<uint32_t>() + nslots;
    SGB_TRY(scan_exclusive_u32(per.as<uint32_t>(), off.as<uint32_t>(), nslots, total, &g->scratch[6], s));
    SGB_TRY(g->hscratch.ensure(64));
    SGB_CUDA(cudaMemcpyAsync(g->hscratch.p, total, 4, cudaMemcpyDeviceToHost, s));
    SGB_CUDA(cudaStreamSynchronize(s));
    const int64_t add = *(uint32_t*)g->hscratch.p;
    if (add == 0) return SGB_OK;
    SGB_TRY(g->pend_lin.reserve((size_t)(g->npend + add) * 8));
    PoolCopy pc{};
    pc.nprop = g->nprop;
    for (int p = 0; p < g->nprop; ++p) {
        const int es = elem_size(g->ptype[p]);
        SGB_TRY(g->pend_val[p].reserve((size_t)(g->npend + add) * es));
        pc.src[p] = values ? (const unsigned char*)values[p] : nullptr;
        if (pc.src[p]) g->pend_has[p] = true;
        pc.dst[p] = g->pend_val[p].as<unsigned char>() + (size_t)g->npend * es;
        pc.es[p] = es;
        pc.bck[p] = bck_pattern(g, p);
    }
    k_block_emit<<<wblocks, 256, 0, s>>>(cnt.as<uint32_t>(), npools, nslot, keys, masks, off.as<uint32_t>(), g->geo,
                                         g->pend_lin.as<int64_t>() + g->npend, pc, g->err.as<unsigned>());
    SGB_CUDA(cudaGetLastError());
    g->npend += add;
    return SGB_OK;
}

int sgb_set_linearizer(sgb_grid* g, int kind) {
    if (!g || (kind != SGB_LIN_SMB && kind != SGB_LIN_ZMB)) return SGB_EINVAL;
    if (g->n != 0 || g->npend != 0) {
        set_error("the chunk linearizer is chosen while the grid is empty");
        return SGB_ESTATE;
    }
    if (kind == SGB_LIN_ZMB) {
        if (g->geo.dim != 3) return SGB_ENOTSUP;
        for (int d = 0; d < 3; ++d)
            if (g->geo.bsz[d] > (int64_t(1) << 21)) {
                set_error("Morton chunk ids hold 21 bits per block coordinate");
                return SGB_ENOTSUP;
            }
    }
    g->geo.zorder = kind == SGB_LIN_ZMB;
    g->nn_valid[0] = g->nn_valid[1] = false;
    g->nnhash_ok = false;
    return SGB_OK;
}

int sgb_get_view(sgb_grid* g, int nn_kind, sgb_view* out, sgb_stream stream) {
    if (!g || !out || (nn_kind != SGB_NN_STAR && nn_kind != SGB_NN_FULL)) return SGB_EINVAL;
    cudaStream_t s = (cudaStream_t)stream;
    SGB_TRY(ensure_neighbours(g, nn_kind, s));
    for (int p = 0; p < g->nprop; ++p) SGB_TRY(ensure_clean(g, p, s));
    std::memset(out, 0, sizeof(*out));
    out->n = g->n;
    out->edge = g->geo.edge;
    out->bs = g->geo.bs;
    out->nprop = g->nprop;
    out->nn_kind = nn_kind;
    for (int d = 0; d < 3; ++d) {
        out->size[d] = g->geo.size[d];
        out->bsz[d] = g->geo.bsz[d];
    }
    out->zorder = g->geo.zorder;
    out->keys = g->keys.as<int64_t>();
    for (int p = 0; p < g->nprop; ++p) out->data[p] = g->data[p].p;
    out->mask = g->mask.as<uint8_t>();
    out->nn = g->nn[nn_kind].as<int32_t>();
    return SGB_OK;
}

int sgb_nchunks(const sgb_grid* g, int64_t* n) {
    if (!g || !n) return SGB_EINVAL;
    *n = g->n;
    return SGB_OK;
}

int sgb_index_buffer(sgb_grid* g, const int64_t** dev) {
    if (!g || !dev) return SGB_EINVAL;
    *dev = g->keys.as<int64_t>();
    return SGB_OK;
}

int sgb_data_buffer(sgb_grid* g, int prop, void** dev) {
    if (!g || !dev || prop < 0 || prop >= g->nprop) return SGB_EINVAL;
    *dev = g->data[prop].p;
    g->clean[prop] = false;  // the caller may write any point
    return SGB_OK;
}

int sgb_mask_buffer(sgb_grid* g, uint8_t** dev) {
    if (!g || !dev) return SGB_EINVAL;
    *dev = g->mask.as<uint8_t>();
    for (int p = 0; p < g->nprop; ++p) g->clean[p] = false;  // existence may change
    g->bits_valid = false;
    g->epts_valid = false;
    return SGB_OK;
}

static int load_map_impl(sgb_grid* g, int64_t n, const int64_t* keys, const void* const* data, const uint8_t* mask,
                         cudaMemcpyKind kind, cudaStream_t s) {
    if (!g || n < 0 || (n > 0 && (!keys || !data || !mask))) return SGB_EINVAL;
    SGB_TRY(grid_reserve(g, n, false));
    const int bs = g->geo.bs;
    if (n > 0) {
        SGB_CUDA(cudaMemcpyAsync(g->keys.p, keys, (size_t)n * 8, kind, s));
        for (int p = 0; p < g->nprop; ++p) {
            const int es = elem_size(g->ptype[p]);
            if (data[p]) SGB_CUDA(cudaMemcpyAsync(g->data[p].p, data[p], (size_t)n * bs * es, kind, s));
            else SGB_TRY(fill(g->data[p].p, n * bs, es, bck_pattern(g, p), s));  // not given: background
        }
        SGB_CUDA(cudaMemcpyAsync(g->mask.p, mask, (size_t)n * bs, kind, s));
    }
    g->n = n;
    SGB_TRY(write_background(g, n, s, g->data, g->mask));
    for (int p = 0; p < g->nprop; ++p) SGB_TRY(sanitize_prop(g, p, s));
    invalidate_derived(g);
    return SGB_OK;
}

int sgb_load_map(sgb_grid* g, int64_t n, const int64_t* keys, const void* const* data, const uint8_t* mask,
                 sgb_stream s) {
    return load_map_impl(g, n, keys, data, mask, cudaMemcpyHostToDevice, (cudaStream_t)s);
}

int sgb_load_map_dev(sgb_grid* g, int64_t n, const int64_t* keys, const void* const* data, const uint8_t* mask,
                     sgb_stream s) {
    return load_map_impl(g, n, keys, data, mask, cudaMemcpyDeviceToDevice, (cudaStream_t)s);
}

int sgb_download_map(sgb_grid* g, int64_t* keys, void* const* data, uint8_t* mask, sgb_stream stream) {
    if (!g) return SGB_EINVAL;
    cudaStream_t s = (cudaStream_t)stream;
    const int bs = g->geo.bs;
    if (keys && g->n) SGB_CUDA(cudaMemcpyAsync(keys, g->keys.p, (size_t)g->n * 8, cudaMemcpyDeviceToHost, s));
    if (data)
        for (int p = 0; p < g->nprop; ++p)
            if (data[p])
                SGB_CUDA(cudaMemcpyAsync(data[p], g->data[p].p, (size_t)(g->n + 1) * bs * elem_size(g->ptype[p]),
                                         cudaMemcpyDeviceToHost, s));
    if (mask) SGB_CUDA(cudaMemcpyAsync(mask, g->mask.p, (size_t)(g->n + 1) * bs, cudaMemcpyDeviceToHost, s));
    SGB_CUDA(cudaStreamSynchronize(s));
    return SGB_OK;
}

int sgb_count_existing(sgb_grid* g, int64_t* existing, int64_t* padding, sgb_stream stream) {
    if (!g) return SGB_EINVAL;
    cudaStream_t s = (cudaStream_t)stream;
    SGB_TRY(g->scratch[11].ensure(16));
    SGB_CUDA(cudaMemsetAsync(g->scratch[11].p, 0, 16, s));
    const int64_t total = g->n * g->geo.bs;
    if (total > 0) {
        int64_t blocks = (total + 255) / 256;
        if (blocks > 2048) blocks = 2048;
        k_count<<<(unsigned)blocks, 256, 0, s>>>(g->mask.as<uint8_t>(), total,
                                                 g->scratch[11].as<unsigned long long>());
        SGB_CUDA(cudaGetLastError());
    }
    SGB_TRY(g->hscratch.ensure(64));
    SGB_CUDA(cudaMemcpyAsync(g->hscratch.p, g->scratch[11].p, 16, cudaMemcpyDeviceToHost, s));
    SGB_CUDA(cudaStreamSynchronize(s));
    unsigned long long* h = (unsigned long long*)g->hscratch.p;
    if (existing) *existing = (int64_t)h[0];
    if (padding) *padding = (int64_t)h[1];
    return SGB_OK;
}

int sgb_existing_offsets(sgb_grid* g, int64_t* offsets, sgb_stream stream) {
    if (!g || !offsets) return SGB_EINVAL;
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t n = g->n;
    if (n * (int64_t)g->geo.bs >= (int64_t(1) << 32)) {
        // the counts are scanned in 32-bit words: larger totals would wrap
        set_error("sgb_existing_offsets scans 32-bit counts: at most 2^32 - 1 chunk points");
        return SGB_ERANGE;
    }
    DevBuf& counts = g->scratch[7];
    DevBuf& scanned = g->scratch[8];
    SGB_TRY(counts.ensure((size_t)(n + 1) * 4));
    SGB_TRY(scanned.ensure((size_t)(n + 2) * 4));
    if (n > 0) {
        k_chunk_counts<<<(unsigned)((n * 32 + 255) / 256), 256, 0, s>>>(g->mask.as<uint8_t>(), n, g->geo.bs,
                                                                       counts.as<uint32_t>());
        SGB_CUDA(cudaGetLastError());
    }
    uint32_t* total = scanned.as<uint32_t>() + n + 1;
    SGB_TRY(scan_exclusive_u32(counts.as<uint32_t>(), scanned.as<uint32_t>(), n, total, &g->scratch[6], s));
    k_offsets_i64<<<(unsigned)((n + 1 + 255) / 256), 256, 0, s>>>(scanned.as<uint32_t>(), total, n, offsets);
    SGB_CUDA(cudaGetLastError());
    return SGB_OK;
}

int sgb_get(sgb_grid* g, int64_t n, const int32_t* coords, int prop, void* out, sgb_stream stream) {
    if (!g || n < 0 || prop < 0 || prop >= g->nprop || (n > 0 && (!coords || !out))) return SGB_EINVAL;
    if (n == 0) return SGB_OK;
    cudaStream_t s = (cudaStream_t)stream;
    const unsigned blocks = (unsigned)((n + 255) / 256);
    const int64_t* k = g->keys.as<int64_t>();
    const uint8_t* m = g->mask.as<uint8_t>();
    switch (elem_size(g->ptype[prop])) {
        case 1: k_get<uint8_t><<<blocks, 256, 0, s>>>(coords, n, g->geo, k, g->n, g->data[prop].as<uint8_t>(), m, (uint8_t*)out); break;
        case 4: k_get<uint32_t><<<blocks, 256, 0, s>>>(coords, n, g->geo, k, g->n, g->data[prop].as<uint32_t>(), m, (uint32_t*)out); break;
        default: k_get<uint64_t><<<blocks, 256, 0, s>>>(coords, n, g->geo, k, g->n, g->data[prop].as<uint64_t>(), m, (uint64_t*)out); break;
    }
    SGB_CUDA(cudaGetLastError());
    return SGB_OK;
}

int sgb_check_device_errors(sgb_grid* g, sgb_stream stream) {
    if (!g) return SGB_EINVAL;
    cudaStream_t s = (cudaStream_t)stream;
    SGB_TRY(g->hscratch.ensure(64));
    SGB_CUDA(cudaMemcpyAsync(g->hscratch.p, g->err.p, 4, cudaMemcpyDeviceToHost, s));
    SGB_CUDA(cudaMemsetAsync(g->err.p, 0, 4, s));
    SGB_CUDA(cudaStreamSynchronize(s));
    unsigned e = *(unsigned*)g->hscratch.p;
    if (e & kErrWaitTimeout) {
        set_error("a device-side bounded wait gave up");
        return SGB_ETIMEOUT;
    }
    if (e & kErrOutOfDomain) {
        set_error("an inserted point lies outside the grid domain");
        return SGB_ERANGE;
    }
    if (e & kErrPoolOverflow) {
        set_error("an insert pool counted more points than its slots (the excess was dropped)");
        return SGB_ERANGE;
    }
    return SGB_OK;
}

int sgb_device_bytes(const sgb_grid* g, int64_t* bytes) {
    if (!g || !bytes) return SGB_EINVAL;
    size_t b = g->keys.bytes + g->keys2.bytes + g->mask.bytes + g->mask2.bytes + g->pend_lin.bytes + g->nn[0].bytes +
               g->nn[1].bytes + g->bits.bytes + g->err.bytes;
    for (int p = 0; p < kMaxProps; ++p) b += g->data[p].bytes + g->data2[p].bytes + g->pend_val[p].bytes;
    for (auto& s : g->scratch) b += s.bytes;
    *bytes = (int64_t)b;
    return SGB_OK;
}

int sgb_set_launch_config(sgb_grid* g, int ctas_per_sm, int stages) {
    if (!g || ctas_per_sm < -1 || ctas_per_sm > 16 || stages < -1 || (stages > 0 && (stages < 3 || stages > 16)))
        return SGB_EINVAL;
    if (ctas_per_sm) g->ctas_per_sm = ctas_per_sm < 0 ? 0 : ctas_per_sm;  // -1: automatic
    if (stages) g->stages = stages < 0 ? 0 : stages;  // -1: automatic depth
    return SGB_OK;
}

}  // extern "C"
