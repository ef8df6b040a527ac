// Internal definitions shared by the CUDA translation units of libsgb200.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/sgb200.h"

namespace sgb {

constexpr int kMaxProps = 8;

// Device error word bits (sgb_check_device_errors).
enum : unsigned {
    kErrWaitTimeout = 1u,   // a bounded mbarrier wait gave up
    kErrOutOfDomain = 2u,   // an inserted point lies outside the domain
    kErrPoolOverflow = 4u,  // an insert pool reported more points than it has slots
};

inline int elem_size(int t) { return t == SGB_F64 ? 8 : (t == SGB_U8 ? 1 : 4); }

void set_error(const std::string& msg);
int cuda_status(cudaError_t e, const char* what);

#define SGB_CUDA(call)                                          \
    do {                                                        \
        cudaError_t e_ = (call);                                \
        if (e_ != cudaSuccess) return ::sgb::cuda_status(e_, #call); \
    } while (0)

#define SGB_TRY(call)                 \
    do {                              \
        int s_ = (call);              \
        if (s_ != SGB_OK) return s_;  \
    } while (0)

// Makes `dev` the current device for the lifetime of the guard and gives the
// caller's current device back on every return path, so an entry point that
// works on a grid of another GPU leaves the caller's CUDA state as it was.
struct DeviceGuard {
    int prev = -1;
    cudaError_t status = cudaSuccess;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) status = cudaSetDevice(dev);
        else prev = -1;  // nothing to restore
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
    DeviceGuard(const DeviceGuard&) = delete;
    DeviceGuard& operator=(const DeviceGuard&) = delete;
};

// Grow-only device buffer.
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    // Growth in place: an address range reserved once (va, va_bytes) with physical memory mapped behind
    // p as the buffer grows, so that contents and address stay; `maps` holds the physical allocations
    // (driver handles and sizes) in address order.  Empty for buffers from cudaMalloc.
    unsigned long long va = 0;
    size_t va_bytes = 0;
    std::vector<std::pair<unsigned long long, size_t>> maps;
    // one owner per allocation: moves (std::swap of buffer sets) leave the source empty, copies are refused
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept { take(o); }
    DevBuf& operator=(DevBuf&& o) noexcept {
        if (this != &o) {
            release();
            take(o);
        }
        return *this;
    }
    ~DevBuf() = default;  // owners release explicitly (the grid and batch destructors)
    int reserve(size_t need);   // keeps contents
    int ensure(size_t need);    // may drop contents
    int grow(size_t need);      // may drop contents; grows to four times the need (tables that follow a growing map)
    // keeps contents; buffers past kInPlaceMinBytes grow in place (no free, no copy, same address) on the
    // current device, smaller ones as reserve()
    int grow_in_place(size_t need);
    void release();
    template <typename T>
    T* as() const { return static_cast<T*>(p); }

   private:
    void take(DevBuf& o) {
        p = o.p;
        bytes = o.bytes;
        va = o.va;
        va_bytes = o.va_bytes;
        maps = std::move(o.maps);
        o.p = nullptr;
        o.bytes = 0;
        o.va = 0;
        o.va_bytes = 0;
        o.maps.clear();
    }
};
constexpr size_t kInPlaceMinBytes = size_t(256) << 20;

// Pinned host staging for small device->host reads.
struct HostScratch {
    void* p = nullptr;
    size_t bytes = 0;
    int ensure(size_t need);
    void release();
};

struct Geometry {
    int dim = 3, edge = 8, bs = 512;
    int64_t size[3] = {1, 1, 1};
    int64_t bsz[3] = {1, 1, 1};
    int zorder = 0;  // chunk ids: 0 grid_smb (x fastest), 1 grid_zmb (Morton)
};

// Morton spreading / compaction of 21-bit coordinates (the published
// "magic bits" bit-interleaving method): bit i of v moves to bit 3i.
__host__ __device__ inline uint64_t morton_spread3(uint64_t v) {
    v &= 0x1fffffull;
    v = (v | v << 32) & 0x1f00000000ffffull;
    v = (v | v << 16) & 0x1f0000ff0000ffull;
    v = (v | v << 8) & 0x100f00f00f00f00full;
    v = (v | v << 4) & 0x10c30c30c30c30c3ull;
    v = (v | v << 2) & 0x1249249249249249ull;
    return v;
}
__host__ __device__ inline uint64_t morton_compact3(uint64_t v) {
    v &= 0x1249249249249249ull;
    v = (v ^ (v >> 2)) & 0x10c30c30c30c30c3ull;
    v = (v ^ (v >> 4)) & 0x100f00f00f00f00full;
    v = (v ^ (v >> 8)) & 0x1f0000ff0000ffull;
    v = (v ^ (v >> 16)) & 0x1f00000000ffffull;
    v = (v ^ (v >> 32)) & 0x1fffffull;
    return v;
}

// Chunk id of an in-domain block coordinate: grid_smb::BlockLinId
// (src/Grid/Geometry/grid_smb.hpp:280-299) or grid_zmb::BlockLinId = lin_zid
// (src/Grid/Geometry/grid_zmb.hpp:100-104, src/util/zmorton.hpp:72-98).
__host__ __device__ inline int64_t block_key(const Geometry& g, int64_t bx, int64_t by, int64_t bz) {
    if (g.zorder)
        return (int64_t)(morton_spread3((uint64_t)bx) | morton_spread3((uint64_t)by) << 1 |
                         morton_spread3((uint64_t)bz) << 2);
    return bx + g.bsz[0] * (by + g.bsz[1] * bz);
}

// Block coordinate of a chunk id (BlockInvLinId of either linearizer).
__host__ __device__ inline void block_coords(const Geometry& g, int64_t key, int64_t* bc) {
    if (g.zorder) {
        bc[0] = (int64_t)morton_compact3((uint64_t)key);
        bc[1] = (int64_t)morton_compact3((uint64_t)key >> 1);
        bc[2] = (int64_t)morton_compact3((uint64_t)key >> 2);
        return;
    }
    if (key >= 0 && key <= 0xffffffffLL && g.bsz[0] <= 0xffffffffLL && g.bsz[1] <= 0xffffffffLL) {
        // the same quotients in 32-bit arithmetic (a 64-bit division is several times dearer)
        const uint32_t k = (uint32_t)key, b0 = (uint32_t)g.bsz[0], b1 = (uint32_t)g.bsz[1];
        const uint32_t q = k / b0;
        bc[0] = (int64_t)(k - q * b0);
        bc[1] = (int64_t)(q % b1);
        bc[2] = (int64_t)(q / b1);
        return;
    }
    bc[0] = key % g.bsz[0];
    bc[1] = (key / g.bsz[0]) % g.bsz[1];
    bc[2] = key / (g.bsz[0] * g.bsz[1]);
}

// Lowest point of a chunk.
__host__ __device__ inline void chunk_origin(const Geometry& g, int64_t key, int64_t* o) {
    block_coords(g, key, o);
    for (int d = 0; d < 3; ++d) o[d] *= g.edge;
}

// Number of chunk ids the linearizer can produce for the domain (ids are below it).
__host__ __device__ inline int64_t key_space(const Geometry& g) {
    if (!g.zorder) return g.bsz[0] * g.bsz[1] * g.bsz[2];
    int64_t m = g.bsz[0] > g.bsz[1] ? g.bsz[0] : g.bsz[1];
    m = m > g.bsz[2] ? m : g.bsz[2];
    int64_t p = 1;
    while (p < m) p <<= 1;
    return p * p * p;
}

// Chunk id and offset in the chunk of an in-domain point: grid_smb::LinId
// (src/Grid/Geometry/grid_smb.hpp:176-190) / grid_zmb::LinId
// (src/Grid/Geometry/grid_zmb.hpp:63-76); the offset is x fastest for both.
__host__ __device__ inline void point_key(const Geometry& g, const int64_t* c, int64_t* key, int64_t* local) {
    const int e = g.edge;
    if (g.zorder) {
        *key = block_key(g, c[0] / e, c[1] / e, c[2] / e);
        *local = c[0] % e + e * (c[1] % e + e * (c[2] % e));
        return;
    }
    int64_t b = c[g.dim - 1] / e, l = c[g.dim - 1] % e;
    for (int d = g.dim - 2; d >= 0; --d) {
        b = b * g.bsz[d] + c[d] / e;
        l = l * e + c[d] % e;
    }
    *key = b;
    *local = l;
}

// Is a chunk id one of a block inside the domain?
__host__ __device__ inline bool key_in_domain(const Geometry& g, int64_t key) {
    if (key < 0 || key >= key_space(g)) return false;
    if (!g.zorder) return true;
    int64_t bc[3];
    block_coords(g, key, bc);
    return bc[0] < g.bsz[0] && bc[1] < g.bsz[1] && bc[2] < g.bsz[2];
}

// Launch parameters of the fixed-function stencils.
struct StencilParams {
    float dt, Du, Dv, F, nFK;
    float bck[2];   // backgrounds of the source properties
    float bckd[2];  // backgrounds of the destination properties
    float coeff[27];
    int64_t box_lo[3], box_hi[3];
    int has_box;
};

// Per-grid entry of a stencil launch.  A grid takes part in global step t
// when start <= t < start + nsteps; it then reads ping-pong buffer
// (t - start) & 1 and writes the other one.  A single-grid launch is the
// entry {start 0, nsteps 1} at t = 0.  bck[b][j] is the background of the
// j-th field of ping-pong buffer b (buffer 0 = the src properties, 1 = dst).
struct GridInfo {
    int64_t start;
    int64_t nsteps;
    float dt, Du, Dv, F, nFK;
    float bck[2][2];
};

// Field pointers of a launch: [ping-pong buffer][source property].
struct FieldSet {
    const float* in[2][2];
    float* out[2][2];
};

// Links of one direction (construct_link_dw / construct_link_up).
struct LinkSet {
    DevBuf pad_pos, pad_off;  // padding points: int32 chunk position, int16 offset
    DevBuf scan;              // uint32 [npad + 1]: first link of each padding point, nlinks last
    DevBuf pos, off;          // links: int32 chunk position, int16 offset in the other grid
    int64_t npad = 0, nlinks = 0;
};

}  // namespace sgb

struct sgb_grid {
    sgb::Geometry geo;
    int device = 0;
    int nprop = 0;
    int ptype[sgb::kMaxProps] = {};
    unsigned char bck[sgb::kMaxProps][8] = {};

    int64_t n = 0;        // chunks
    int64_t cap = 0;      // chunk capacity of the buffers below (excluding background)
    sgb::DevBuf keys;     // int64 [cap]
    sgb::DevBuf data[sgb::kMaxProps];  // [(cap+1) * bs]
    sgb::DevBuf mask;     // [(cap+1) * bs]
    // second set of buffers for flushes that add chunks
    sgb::DevBuf keys2, data2[sgb::kMaxProps], mask2;

    // staged inserts
    int64_t npend = 0;
    sgb::DevBuf pend_lin;                    // int64 [npend]
    sgb::DevBuf pend_val[sgb::kMaxProps];    // [npend]
    bool pend_has[sgb::kMaxProps] = {};

    // neighbour tables (int32, -1 = absent); index 0 NNStar (8/chunk), 1 NNFull (27/chunk)
    sgb::DevBuf nn[2];
    bool nn_valid[2] = {false, false};
    sgb::DevBuf nnhash;   // open-addressing hash of the chunk keys used by the neighbour search
    bool nnhash_ok = false;  // built for the current keys (any key change invalidates both nn tables)
    sgb::DevBuf bits;     // uint64 existence bitmaps, bs/64 words per chunk
    bool bits_valid = false;
    // existing-point list (e_points): uint32 chunk position * bs + offset
    sgb::DevBuf epts;
    int64_t nepts = 0;
    bool epts_valid = false;
    // multi-resolution links: [0] down, [1] up
    sgb::LinkSet links[2];

    // clean[p]: every point of property p whose mask byte is 0 holds the
    // background value.  The reference substitutes the background for such
    // points whenever it reads them (loadGhostBlock, BlockMapGpu_ker::get);
    // keeping them filled lets the stencils read chunk data without a mask
    // test per neighbour.  Cleared when the caller gets a writable pointer.
    bool clean[sgb::kMaxProps] = {true, true, true, true, true, true, true, true};

    // flush / scan / sort scratch
    sgb::DevBuf scratch[12];
    sgb::HostScratch hscratch;

    sgb::DevBuf err;      // unsigned device error word
    int num_sms = 148;
    int ctas_per_sm = 0;  // 0: automatic per stencil kind (auto_ctas_per_sm)
    int stages = 0;       // 0: deepest staging ring that keeps ctas_per_sm CTAs resident
};

namespace sgb {

// neighbours.cu
int ensure_neighbours(sgb_grid* g, int nn, cudaStream_t s);
int ensure_bits(sgb_grid* g, cudaStream_t s);

// points.cu
int ensure_point_list(sgb_grid* g, cudaStream_t s);
int launch_points_box27(sgb_grid* g, const int* src, const int* dst, const StencilParams& prm, cudaStream_t s);
int launch_points_box27_sparse(sgb_grid* g, const int* src, const int* dst, const StencilParams& prm,
                               cudaStream_t s);

// stencil.cu
int launch_stencil(sgb_grid* g, int kind, const int* src, const int* dst, const StencilParams& prm,
                   cudaStream_t s);
int make_params(sgb_grid* g, int kind, const int* src, const int* dst, const float* params, int nparams,
                const int64_t* box, StencilParams& prm);

// scan.cu
int scan_exclusive_u32(const uint32_t* in, uint32_t* out, int64_t n, uint32_t* total_dev, DevBuf* tmp,
                       cudaStream_t s);

// buffers
int grid_reserve(sgb_grid* g, int64_t chunks, bool keep);
// fill the mask-0 points of property p with its background (sets clean[p])
int sanitize_prop(sgb_grid* g, int p, cudaStream_t s);
// fill every point (n + 1 chunks) of property p with its background
int fill_background_all(sgb_grid* g, int p, cudaStream_t s);
int ensure_clean(sgb_grid* g, int p, cudaStream_t s);
// fill count elements of esize bytes with the low esize bytes of pattern
int fill(void* dst, int64_t count, int esize, uint64_t pattern, cudaStream_t s);
// the background of property p as an element_size-byte pattern
uint64_t bck_pattern(const sgb_grid* g, int p);
int write_background(sgb_grid* g, int64_t pos, cudaStream_t s, DevBuf* data, DevBuf& mask);

}  // namespace sgb
