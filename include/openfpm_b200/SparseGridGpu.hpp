// C++ drop-in front-end for the SparseGridGpu hot path over libsgb200.
//
// Mirrors the reference class template
//   SparseGridGpu<dim, aggregate<T...>, blockEdgeSize, threadBlockSize, indexT>
// (src/SparseGridGpu/SparseGridGpu.hpp:483-493) for dim = 3 and 8^3 / 4^3
// chunks: the host methods keep the reference's names and argument meaning,
// the device view returned by toKernel() offers init / insert<p> /
// flush_block_insert / get<p> to user kernels, and the conv family takes user
// __device__ lambdas.  Fixed-function stencils (HeatStencil, Conv3x3x3) run
// the library's kernels; conv lambdas run a header kernel instantiated in the
// caller's translation unit.  Compile user code with nvcc (-std=c++17,
// --extended-lambda) and link libsgb200.so.
//
// Errors: every failing library call throws openfpm_b200::sgb_error carrying
// the sgb_status and the library's message (the reference prints and
// continues, SparseGridGpu.hpp:2347-2352).
#pragma once

#if !defined(__CUDACC__)
#error "SparseGridGpu.hpp holds device code: compile with nvcc"
#endif

#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <stdexcept>
#include <string>
#include <tuple>
#include <type_traits>
#include <utility>
#include <vector>

#include "../sgb200.h"

// Position of a chunk in the block map, as the reference's stencil functors receive it
// (openfpm::sparse_index, src/Vector/map_vector_sparse.hpp).
namespace openfpm {
template <typename T>
struct sparse_index {
    T id;
};
}  // namespace openfpm

namespace openfpm_b200 {

// ------------------------------------------------------------------ support types
struct sgb_error : std::runtime_error {
    int status;
    sgb_error(int s, const std::string& what)
        : std::runtime_error(what + ": " + sgb_status_string(s) + " (" + sgb_last_error_string() + ")"), status(s) {}
};

inline void check(int s, const char* what) {
    if (s != SGB_OK) throw sgb_error(s, what);
}

template <typename... T>
struct aggregate {
    using type = std::tuple<T...>;
    static constexpr unsigned max_prop = sizeof...(T);
};

template <unsigned dim, typename T = long>
struct grid_key_dx {
    T k[dim];
    __host__ __device__ grid_key_dx() : k{} {}
    __host__ __device__ grid_key_dx(std::initializer_list<T> l) : k{} {
        unsigned i = 0;
        for (T v : l)
            if (i < dim) k[i++] = v;
    }
    __host__ __device__ T get(unsigned i) const { return k[i]; }
    __host__ __device__ void set_d(unsigned i, T v) { k[i] = v; }
};

template <unsigned dim, typename T>
struct Box {
    T lo[dim], hi[dim];
    __host__ __device__ T getLow(unsigned i) const { return lo[i]; }
    __host__ __device__ T getHigh(unsigned i) const { return hi[i]; }
    __host__ __device__ void setLow(unsigned i, T v) { lo[i] = v; }
    __host__ __device__ void setHigh(unsigned i, T v) { hi[i] = v; }
};

template <unsigned dim, typename T>
struct Point {
    T x[dim];
    __host__ __device__ T get(unsigned i) const { return x[i]; }
};

namespace gpu {
struct ofp_context_t {};
}  // namespace gpu

// The sub-grid iterator's box (SparseGridGpu_iterator_sub): inclusive start / stop.
template <unsigned dim>
struct SparseGridGpu_iterator_sub {
    grid_key_dx<dim> start, stop;
    const grid_key_dx<dim>& getStart() const { return start; }
    const grid_key_dx<dim>& getStop() const { return stop; }
};

// Byte offsets into a pack buffer (the reference's Pack_stat / Unpack_stat).
struct Pack_stat {
    size_t off = 0;
    size_t getOffset() const { return off; }
};
struct Unpack_stat {
    size_t off = 0;
    size_t getOffset() const { return off; }
    void addOffset(size_t b) { off += b; }
};

// A device byte buffer standing in for ExtPreAlloc<CudaMemory>.
class CudaMemory {
   public:
    CudaMemory() = default;
    CudaMemory(const CudaMemory&) = delete;
    CudaMemory& operator=(const CudaMemory&) = delete;
    ~CudaMemory() {
        if (p_) cudaFree(p_);
    }
    bool resize(size_t n) {
        if (n <= sz_) return true;
        void* q = nullptr;
        if (cudaMalloc(&q, n) != cudaSuccess) return false;
        if (p_) cudaFree(p_);
        p_ = q;
        sz_ = n;
        return true;
    }
    void* getDevicePointer() const { return p_; }
    size_t size() const { return sz_; }

   private:
    void* p_ = nullptr;
    size_t sz_ = 0;
};

enum flush_type { FLUSH_ON_HOST = 0, FLUSH_ON_DEVICE = 1 };
enum StencilMode { STENCIL_MODE_INPLACE = 1, STENCIL_MODE_INPLACE_NO_SHARED = 3 };
enum class tag_boundaries { NO_CALCULATE_EXISTING_POINTS, CALCULATE_EXISTING_POINTS };
struct No_check {};
enum mask_sparse { NOT_EXIST = 0, EXIST = 1, PADDING = 2, EXIST_AND_PADDING = 3 };

template <unsigned dim>
struct NNStar {
    static constexpr int kind = SGB_NN_STAR;
    static constexpr int nNN = 8;  // 2^dim table entries per chunk, the 2*dim faces first
};
template <unsigned dim>
struct NNFull {
    static constexpr int kind = SGB_NN_FULL;
    static constexpr int nNN = 27;  // 3^dim
    // NNFull::getNNindex_offset (src/SparseGridGpu/SparseGridGpu.hpp:331-355): the neighbour slot
    // (dx + 3 dy + 9 dz, d in {0, 1, 2}) and the offset inside that chunk of a local coordinate that
    // may lie one chunk outside; true when it does
    template <unsigned E, typename I>
    __host__ __device__ static bool getNNindex_offset(const I (&c)[3], unsigned& nn_index, unsigned& offset_nn) {
        bool out = false;
        nn_index = 0;
        offset_nn = 0;
        unsigned cnt = 1, cnt_off = 1;
        for (int i = 0; i < 3; ++i) {
            const int p = 1 - (int)(c[i] < 0) + (int)(c[i] >= (int)E);
            nn_index += p * cnt;
            offset_nn += (unsigned)((int)c[i] + (1 - p) * (int)E) * cnt_off;
            cnt *= 3;
            cnt_off *= E;
            out |= p != 1;
        }
        return out;
    }
};

// IntPow<base, exp>::value (src/util/mathutil.hpp)
template <unsigned base, unsigned exp>
struct IntPow {
    static constexpr unsigned value = base * IntPow<base, exp - 1>::value;
};
template <unsigned base>
struct IntPow<base, 0> {
    static constexpr unsigned value = 1;
};

// The aggregate a device view exposes as AggregateType / AggregateBlockType: the grid's
// properties stored as chunks of BS points, with the mask block last (index pMask).
template <typename AggregateT, unsigned BS>
struct block_aggregate {
    using scalars = typename AggregateT::type;
    static constexpr unsigned nprop = std::tuple_size<scalars>::value;
    static constexpr unsigned size = BS;
};
namespace detail {
template <typename A, unsigned p, bool mask = (p == A::nprop)>
struct scalar_of {
    using type = typename std::tuple_element<p, typename A::scalars>::type;
};
template <typename A, unsigned p>
struct scalar_of<A, p, true> {
    using type = unsigned char;
};
}  // namespace detail
// ScalarTypeOf<AggregateBlockType, p>: the point type of property p (unsigned char for the mask)
template <typename A, unsigned p>
using ScalarTypeOf = typename detail::scalar_of<A, p>::type;
// BlockTypeOf<AggregateType, p>: a chunk of property p; ::size points
template <typename A, unsigned p>
struct BlockTypeOf {
    using scalar_type = ScalarTypeOf<A, p>;
    static constexpr unsigned size = A::size;
};

// Result of getNNPoint: the chunk position (the background chunk when the neighbour chunk is
// absent) and the point's offset inside it (block_offset, SparseGridGpu_ker.cuh)
template <typename I>
struct block_offset {
    I pos;
    I off;
};

// flush reductions (src/Vector/cuda/map_vector_sparse_cuda_kernels.cuh:51-352)
template <unsigned p> struct sRight_ { static constexpr unsigned prop = p; static constexpr int op = SGB_OP_RIGHT; };
template <unsigned p> struct sLeft_ { static constexpr unsigned prop = p; static constexpr int op = SGB_OP_LEFT; };
template <unsigned p> struct sadd_ { static constexpr unsigned prop = p; static constexpr int op = SGB_OP_ADD; };
template <unsigned p> struct smax_ { static constexpr unsigned prop = p; static constexpr int op = SGB_OP_MAX; };
template <unsigned p> struct smin_ { static constexpr unsigned prop = p; static constexpr int op = SGB_OP_MIN; };
template <unsigned p> struct sBitwiseOr_ { static constexpr unsigned prop = p; static constexpr int op = SGB_OP_OR; };

// fixed-function stencils of the reference's tests
template <unsigned dim, unsigned p_src, unsigned p_dst>
struct HeatStencil {
    static constexpr int kind = SGB_HEAT7;
    static constexpr unsigned src = p_src, dst = p_dst;
};
template <unsigned dim, unsigned p_src, unsigned p_dst>
struct Conv3x3x3 {
    static constexpr int kind = SGB_BOX27;
    static constexpr unsigned src = p_src, dst = p_dst;
};
template <unsigned dim, unsigned p_src, unsigned p_dst>
struct Conv3x3x3_noshared {
    static constexpr int kind = SGB_BOX27_NS;
    static constexpr unsigned src = p_src, dst = p_dst;
};
struct conv_coeff {
    float coeff[3][3][3];
};

template <unsigned dim, typename T>
struct cross_stencil {
    T xm[dim];
    T xp[dim];
};

// Layout of a chunk plus its one-point halo in shared memory: E + 2 planes of E + 2 rows, row (j, k)
// starting at element RS * (j + 1) + PS * (k + 1) and holding x = -1 .. E at its elements X0 - 1 ..
// X0 + E, so that its E interior elements start on a 16-byte boundary (they are copied 16 bytes at a
// time).  The row stride RS is the smallest multiple of X0 above E + 1: a row's x = E element may sit
// in the next row's first X0 - 1 elements, which that row leaves unused.
template <typename T, int E>
struct tile_layout {
    static constexpr int X0 = sizeof(T) >= 16 ? 1 : 16 / (int)sizeof(T);
    static constexpr int RS = ((E + 2 + X0 - 1) / X0) * X0;
    static constexpr int T2 = E + 2;
    static constexpr int PS = RS * T2;
    // one past the last element (x = E of row (E, E)), rounded up to X0
    static constexpr int SIZE = ((X0 + E + RS * (T2 - 1) + PS * (T2 - 1) + 1 + X0 - 1) / X0) * X0;
    __host__ __device__ static constexpr int index(int i, int j, int k) { return X0 + i + RS * (j + 1) + PS * (k + 1); }
};

// halo-indexed tile accessor (src/SparseGrid/cp_block.hpp:14-97): u(i, j, k)
// for local coordinates i, j, k in [-1, edge]
template <typename T, int E>
struct cp_block {
    T* ptr;
    __device__ T& operator()(int i, int j, int k) const { return ptr[tile_layout<T, E>::index(i, j, k)]; }
};

// chunk data handle passed to conv2_b functions: block.template get<p>()[offset]
template <int NPROP>
struct data_block {
    void* const* data;
    int64_t chunk;
    int bs;
    template <unsigned p, typename T = float>
    __device__ T* get() const {
        return static_cast<T*>(data[p]) + chunk * bs;
    }
};

namespace detail {
// chunk ids of the two linearizers (grid_smb: block x fastest; grid_zmb:
// 3-D Morton code of the block coordinate, 21 bits per coordinate)
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
__host__ __device__ inline int64_t block_key(int zorder, const int64_t* bsz, int64_t bx, int64_t by, int64_t bz) {
    if (zorder) return (int64_t)(morton_spread3(bx) | morton_spread3(by) << 1 | morton_spread3(bz) << 2);
    return bx + bsz[0] * (by + bsz[1] * bz);
}
__host__ __device__ inline void block_coords(int zorder, const int64_t* bsz, int64_t key, int64_t* bc) {
    if (zorder) {
        bc[0] = (int64_t)morton_compact3((uint64_t)key);
        bc[1] = (int64_t)morton_compact3((uint64_t)key >> 1);
        bc[2] = (int64_t)morton_compact3((uint64_t)key >> 2);
        return;
    }
    if (key >= 0 && key <= 0xffffffffLL && bsz[0] <= 0xffffffffLL && bsz[1] <= 0xffffffffLL) {
        // the same quotients in 32-bit arithmetic (a 64-bit division is a long software sequence)
        const uint32_t k = (uint32_t)key, b0 = (uint32_t)bsz[0], b1 = (uint32_t)bsz[1];
        const uint32_t q = k / b0;
        bc[0] = (int64_t)(k - q * b0);
        bc[1] = (int64_t)(q % b1);
        bc[2] = (int64_t)(q / b1);
        return;
    }
    bc[0] = key % bsz[0];
    bc[1] = (key / bsz[0]) % bsz[1];
    bc[2] = key / (bsz[0] * bsz[1]);
}
template <typename T> struct sgb_type_of;
template <> struct sgb_type_of<float> { static constexpr int value = SGB_F32; };
template <> struct sgb_type_of<int> { static constexpr int value = SGB_I32; };
template <> struct sgb_type_of<double> { static constexpr int value = SGB_F64; };
template <> struct sgb_type_of<unsigned char> { static constexpr int value = SGB_U8; };

template <typename Tuple> struct types_of;
template <typename... T>
struct types_of<std::tuple<T...>> {
    static std::vector<int> get() { return {sgb_type_of<T>::value...}; }
};

__device__ __forceinline__ int64_t find_key(const int64_t* keys, int64_t n, int64_t key) {
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (keys[mid] < key) lo = mid + 1;
        else hi = mid;
    }
    return (lo < n && keys[lo] == key) ? lo : -1;
}

// per-CTA slot counters of the insert pools (vct_atomic_add in the reference):
// point slots of insert<p>, chunk slots of insertBlock
static __shared__ int sgb_pool_counter;
static __shared__ int sgb_block_counter;

// cp.async copies of one element (4 or 8 bytes) into shared memory; other sizes are copied by the
// thread itself
template <typename T>
__device__ __forceinline__ void async_copy_elem(T* dst_smem, const T* src) {
    if constexpr (sizeof(T) == 4 || sizeof(T) == 8) {
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"((unsigned)__cvta_generic_to_shared(dst_smem)),
                     "l"(src), "n"((int)sizeof(T))
                     : "memory");
    } else {
        *dst_smem = *src;
    }
}
__device__ __forceinline__ void async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void async_wait_group() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// 16-byte cp.async copy into shared memory (both addresses 16-byte aligned)
template <typename T>
__device__ __forceinline__ void async_copy16(T* dst_smem, const T* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((unsigned)__cvta_generic_to_shared(dst_smem)),
                 "l"(src)
                 : "memory");
}

// Copy plan of one field's halo tile for thread `tid` of NT.  Work items are numbered with the
// 16-byte pieces of the row interiors first (rows (j, k) = -1 .. E, j fastest), then the two x-halo
// elements of every row (every element of every row when a row interior is not a multiple of 16
// bytes); a thread takes items tid, tid + NT, ...  An item's place in the tile, its offset inside the
// source chunk and the neighbour-table slot it reads (0 .. 26, SELF for the chunk itself) are the
// same for every chunk, so each thread works them out once.
template <typename T, int E, int NT>
struct tile_plan {
    using LT = tile_layout<T, E>;
    static constexpr int T2 = E + 2, ROWS = T2 * T2, BS = E * E * E, SELF = 27;
    static constexpr bool VEC = sizeof(T) <= 16 && (E * sizeof(T)) % 16 == 0;
    static constexpr int PER = VEC ? 16 / (int)sizeof(T) : 1;  // elements of a piece
    static constexpr int VPR = VEC ? E / PER : 0;               // pieces per row interior
    static constexpr int NVEC = ROWS * VPR;
    static constexpr int NITEM = NVEC + ROWS * (VEC ? 2 : E + 2);
    static constexpr int ITEMS = (NITEM + NT - 1) / NT;
    static_assert(BS <= 65536, "a chunk's element offsets are kept in 16 bits");
    int toff[ITEMS];  // element offset in the tile; -1: no item
    int soff[ITEMS];  // element offset in the source chunk | slot << 16

    __device__ static int slot_of(int kn, int dx, int dy, int dz) {
        const int nz = (dx != 0) + (dy != 0) + (dz != 0);
        if (nz == 0) return SELF;
        if (kn == 27) return (dx + 1) + 3 * (dy + 1) + 9 * (dz + 1);
        return nz > 1 ? 0 : dx ? (dx < 0 ? 0 : 1) : dy ? (dy < 0 ? 2 : 3) : (dz < 0 ? 4 : 5);
    }
    __device__ void init(int tid, int kn) {
#pragma unroll
        for (int q = 0; q < ITEMS; ++q) {
            const int w = tid + q * NT;
            toff[q] = -1;
            soff[q] = 0;
            if (w >= NITEM) continue;
            int r, i;
            if (w < NVEC) {
                r = w / (VPR > 0 ? VPR : 1);
                i = (w % (VPR > 0 ? VPR : 1)) * PER;
            } else if (VEC) {
                r = (w - NVEC) / 2;
                i = (w - NVEC) % 2 ? E : -1;
            } else {
                r = (w - NVEC) / (E + 2);
                i = (w - NVEC) % (E + 2) - 1;
            }
            const int j = r % T2 - 1, k = r / T2 - 1;
            const int dx = i < 0 ? -1 : (i >= E ? 1 : 0), dy = j < 0 ? -1 : (j >= E ? 1 : 0),
                      dz = k < 0 ? -1 : (k >= E ? 1 : 0);
            const int lx = (i + E) % E, ly = (j + E) % E, lz = (k + E) % E;
            toff[q] = LT::index(i, j, k);
            soff[q] = (lx + E * (ly + E * lz)) | slot_of(kn, dx, dy, dz) << 16;
        }
    }
    // issue this thread's copies of chunk table `nnrow` (slot SELF: the chunk) into tiles[0 .. NF - 1]
    // from fields srcs[0 .. NF - 1] of this type (background bks[f] where the source chunk is absent)
    template <int NF>
    __device__ void issue(int tid, const int32_t* nnrow, T* const* tiles, const T* const* srcs, const T* bks) const {
#pragma unroll
        for (int q = 0; q < ITEMS; ++q) {
            if (toff[q] < 0) continue;
            const int sc = nnrow[soff[q] >> 16];
            const int64_t so = (int64_t)sc * BS + (soff[q] & 0xffff);
            if (VEC && tid + q * NT < NVEC) {
                if (sc >= 0) {
#pragma unroll
                    for (int f = 0; f < NF; ++f) async_copy16(tiles[f] + toff[q], srcs[f] + so);
                } else {
#pragma unroll
                    for (int e = 0; e < PER; ++e)
#pragma unroll
                        for (int f = 0; f < NF; ++f) tiles[f][toff[q] + e] = bks[f];
                }
            } else {
                if (sc >= 0) {
#pragma unroll
                    for (int f = 0; f < NF; ++f) async_copy_elem(tiles[f] + toff[q], srcs[f] + so);
                } else {
#pragma unroll
                    for (int f = 0; f < NF; ++f) tiles[f][toff[q]] = bks[f];
                }
            }
        }
    }
};

// threads per CTA of the conv kernel: two warps share a chunk (fewer threads per chunk spend fewer
// instructions on the per-chunk work, and more registers per thread keep more points in flight)
constexpr int kConvThreads = 64;

// Conv kernel for user lambdas, over up to three source fields (NP) of any types: each CTA (two warps,
// eight points a thread in 8^3 chunks) takes chunks blockIdx.x, + gridDim.x, ... and keeps two halo
// tiles per source field in shared memory (tile_layout).  While one chunk is computed from one tile,
// the next chunk's tile is gathered into the other by cp.async copies, row by row: the E interior
// elements of a row in 16-byte copies from the chunk the row lies in (the chunk itself, a face
// neighbour, or for rows along a halo edge the edge neighbour under NNFull and neighbour 0, the -x
// chunk, at the wrapped coordinate under NNStar, as the reference's ghost-layer map gives them), the
// two x-halo elements one by one.  Absent chunks give the background.  One barrier per chunk: a thread
// waits for its own copies of the chunk, the barrier makes every thread's copies visible and closes the
// reads of the other tile, and only then is the next chunk's gather issued.  The lambda runs for every
// active point inside the box (conv_cross writes every point of the chunk).
template <int E, int NP, int MODE, typename T0, typename T1, typename T2, typename U0, typename U1, typename U2,
          typename F>
__global__ void __launch_bounds__(kConvThreads, 8)
    conv_kernel(sgb_view v, int src0, int src1, int src2, int dst0, int dst1, int dst2, Box<3, int> box, int full_box,
                T0 bk0, T1 bk1, T2 bk2, F f) {
    constexpr int NT = kConvThreads;
    using L0 = tile_layout<T0, E>;
    using P0 = tile_plan<T0, E, NT>;
    using P1 = tile_plan<T1, E, NT>;
    using P2 = tile_plan<T2, E, NT>;
    // source fields of one type share their copy items
    constexpr bool SAME = (NP < 2 || std::is_same<T0, T1>::value) && (NP < 3 || std::is_same<T0, T2>::value);
    constexpr int BS = E * E * E, NPT = (BS + NT - 1) / NT;
    constexpr int NB = 2;  // halo tiles per field: chunks s + 1 .. s + NB - 1 are in flight while s computes
    constexpr int M = NB + 1;    // slots of per-chunk metadata (neighbour row, box)
    constexpr bool BITS = E <= 10;  // box as one bit per in-box x, y and z, or lo / hi per dimension
    constexpr int NBW = BITS ? 1 : 6;
    __shared__ __align__(16) T0 tile0[NB][L0::SIZE];
    __shared__ __align__(16) T1 tile1[NB][NP >= 2 ? tile_layout<T1, E>::SIZE : 16];
    __shared__ __align__(16) T2 tile2[NB][NP >= 3 ? tile_layout<T2, E>::SIZE : 16];
    __shared__ int32_t nnrow[M][28];
    __shared__ int32_t boxc[M][NBW];
    const T0* s0 = static_cast<const T0*>(v.data[src0]);
    const T1* s1 = static_cast<const T1*>(v.data[src1]);
    const T2* s2 = static_cast<const T2*>(v.data[src2]);
    U0* const d0g = static_cast<U0*>(v.data[dst0]);
    U1* const d1g = static_cast<U1*>(v.data[dst1]);
    U2* const d2g = static_cast<U2*>(v.data[dst2]);
    const int kn = v.nn_kind == SGB_NN_FULL ? 27 : 8;
    const int tid = threadIdx.x;
    const int64_t stride = gridDim.x, c0 = blockIdx.x;
    if (c0 >= v.n) return;
    // this CTA's chunks are c0, c0 + stride, ...: chunk number s is at position c0 + s * stride
    const int64_t nmine = (v.n - c0 + stride - 1) / stride;
    auto pos = [&](int64_t s) { return c0 + s * stride; };
    P0 plan0;
    P1 plan1;
    P2 plan2;
    plan0.init(tid, kn);
    if (NP >= 2 && !SAME) plan1.init(tid, kn);
    if (NP >= 3 && !SAME) plan2.init(tid, kn);
    auto gather = [&](int64_t s) {  // chunk number s into tile s % NB (its metadata in slot s % M)
        if (s < nmine) {
            const int b = (int)(s % NB), m = (int)(s % M);
            if constexpr (SAME) {
                T0* const tiles[3] = {tile0[b], reinterpret_cast<T0*>(tile1[b]), reinterpret_cast<T0*>(tile2[b])};
                const T0* const srcs[3] = {s0, reinterpret_cast<const T0*>(s1), reinterpret_cast<const T0*>(s2)};
                const T0 bks[3] = {bk0, (T0)bk1, (T0)bk2};
                plan0.template issue<NP>(tid, nnrow[m], tiles, srcs, bks);
            } else {
                T0* const t0s[1] = {tile0[b]};
                const T0* const s0s[1] = {s0};
                plan0.template issue<1>(tid, nnrow[m], t0s, s0s, &bk0);
                if constexpr (NP >= 2) {
                    T1* const t1s[1] = {tile1[b]};
                    const T1* const s1s[1] = {s1};
                    plan1.template issue<1>(tid, nnrow[m], t1s, s1s, &bk1);
                }
                if constexpr (NP >= 3) {
                    T2* const t2s[1] = {tile2[b]};
                    const T2* const s2s[1] = {s2};
                    plan2.template issue<1>(tid, nnrow[m], t2s, s2s, &bk2);
                }
            }
        }
        async_commit();  // one group per chunk number, empty past the end
    };
    auto row_of = [&](int64_t s) { return (s < nmine && tid < kn) ? v.nn[pos(s) * kn + tid] : -1; };
    auto box_of = [&](int64_t key, int32_t* out) {
        int64_t bcd[3];
        detail::block_coords(v.zorder, v.bsz, key, bcd);
        uint32_t w = 0;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const int64_t o = bcd[d] * E, l = box.lo[d] - o, h = box.hi[d] - o;
            const int lo = l < 0 ? 0 : (l > E ? E : (int)l), hi = h < -1 ? -1 : (h >= E ? E - 1 : (int)h);
            if constexpr (BITS) {
                if (hi >= lo) w |= (((1u << (hi + 1)) - 1) & ~((1u << lo) - 1)) << (d * E);
            } else {
                out[2 * d] = lo;
                out[2 * d + 1] = hi;
            }
        }
        if constexpr (BITS) out[0] = (int32_t)w;
    };
    // metadata of chunk number s into slot s % M: its neighbour row (loaded earlier into `row`), its own
    // position, and (thread 0, unless the box holds the whole grid) its box from `key`
    auto publish = [&](int64_t s, int32_t row, int64_t key) {
        if (s >= nmine) return;
        const int m = (int)(s % M);
        if (tid < kn) nnrow[m][tid] = row;
        if (tid == 0) {
            nnrow[m][P0::SELF] = (int32_t)pos(s);
            if (!full_box) box_of(key, boxc[m]);
        }
    };
    // point q of this thread, q = 0 .. NPT - 1 (offset in the chunk; i, j, k its coordinates).  In 8^3
    // chunks a warp takes x = 0 .. 7 of one row j in four planes k: with the tile's 12-element rows and
    // 120-element planes (24 banks apart) the warp's reads of the points and of each of their six
    // neighbours fall on 32 distinct banks.
    auto point = [&](int q, int& i, int& j, int& k) {
        const int w = tid + q * NT;
        i = w % E;
        j = E == 8 ? (w >> 5) & 7 : (w / E) % E;
        k = E == 8 ? ((w >> 3) & 3) + 4 * (w >> 8) : w / (E * E);
        return i + E * (j + E * k);
    };
    int pi[NPT], pj[NPT], pk[NPT], pp[NPT];  // this thread's points, worked out once
#pragma unroll
    for (int q = 0; q < NPT; ++q) pp[q] = point(q, pi[q], pj[q], pk[q]);
    uint8_t m_cur[NPT], m_next[NPT];
    auto masks_of = [&](int64_t s, uint8_t* m) {
#pragma unroll
        for (int q = 0; q < NPT; ++q) {
            const int pnt = pp[q];
            m[q] = (s < nmine && (BS % NT == 0 || tid + q * NT < BS)) ? v.mask[pos(s) * BS + pnt] : (uint8_t)0;
        }
    };
    auto key_of = [&](int64_t s) { return (tid == 0 && !full_box && s < nmine) ? v.keys[pos(s)] : (int64_t)0; };
    // prologue: chunk numbers 0 .. NB - 2 in flight
    for (int64_t s = 0; s < NB - 1; ++s) publish(s, row_of(s), key_of(s));
    int32_t row = row_of(NB - 1);
    int64_t key = key_of(NB - 1);
    masks_of(0, m_cur);
    __syncthreads();
    for (int64_t s = 0; s < NB - 1; ++s) gather(s);
    for (int64_t it = 0; it < nmine; ++it) {
        // slot (it + NB - 1) % M last served chunk it - 2, whose readers are all behind the last barrier
        publish(it + NB - 1, row, key);
        row = row_of(it + NB);
        key = key_of(it + NB);
        if constexpr (NB == 2) async_wait_group<0>();
        else async_wait_group<NB - 2>();  // this thread's copies of chunk it
        __syncthreads();  // everyone's copies of chunk it landed; everyone is done with chunk it - 1's tile
        gather(it + NB - 1);
        masks_of(it + 1, m_next);
        const int b = (int)(it % NB), mslot = (int)(it % M);
        uint32_t bw = ~0u;
        int lo[3] = {0, 0, 0}, hi[3] = {E - 1, E - 1, E - 1};
        if (!full_box) {
            if constexpr (BITS) {
                bw = (uint32_t)boxc[mslot][0];
            } else {
#pragma unroll
                for (int d = 0; d < 3; ++d) lo[d] = boxc[mslot][2 * d], hi[d] = boxc[mslot][2 * d + 1];
            }
        }
        const T0* t0 = tile0[b];
        const int64_t c = pos(it);
        U0* const d0 = d0g + c * BS;  // this chunk's destination points
        U1* const d1 = d1g + c * BS;
        U2* const d2 = d2g + c * BS;
#pragma unroll
        for (int q = 0; q < NPT; ++q) {
            if (BS % NT != 0 && tid + q * NT >= BS) break;
            const int i = pi[q], j = pj[q], k = pk[q], pnt = pp[q];
            bool in;
            if constexpr (BITS) {
                const uint32_t pm = (1u << i) | (1u << (E + j)) | (1u << (2 * E + k));
                in = (bw & pm) == pm;
            } else {
                in = i >= lo[0] && i <= hi[0] && j >= lo[1] && j <= hi[1] && k >= lo[2] && k <= hi[2];
            }
            const bool act = (m_cur[q] & 3) == 1 && in;
            const int g = pnt;
            if constexpr (MODE == 0) {  // conv_cross: storeBlock of the whole chunk
                const int cc = L0::index(i, j, k);
                T0 res = t0[cc];
                if (act) {
                    cross_stencil<3, T0> cs;
                    cs.xm[0] = t0[cc - 1];
                    cs.xp[0] = t0[cc + 1];
                    cs.xm[1] = t0[cc - L0::RS];
                    cs.xp[1] = t0[cc + L0::RS];
                    cs.xm[2] = t0[cc - L0::PS];
                    cs.xp[2] = t0[cc + L0::PS];
                    T0 u = t0[cc];
                    res = f(u, cs);
                }
                d0[g] = (U0)res;
            } else if (act) {
                cp_block<T0, E> u{const_cast<T0*>(t0)};
                cp_block<T1, E> w{const_cast<T1*>(tile1[NP >= 2 ? b : 0])};
                if constexpr (MODE == 1) {  // conv
                    d0[g] = (U0)f(u, i, j, k);
                } else if constexpr (MODE == 2) {  // conv2
                    U0 r1 = 0;
                    U1 r2 = 0;
                    f(r1, r2, u, w, i, j, k);
                    d0[g] = r1;
                    d1[g] = r2;
                } else if constexpr (MODE == 3) {  // conv2_b
                    U0 r1 = 0;
                    U1 r2 = 0;
                    data_block<8> blk{v.data, c, BS};
                    f(r1, r2, u, w, blk, pnt, i, j, k);
                    d0[g] = r1;
                    d1[g] = r2;
                } else if constexpr (MODE == 4) {  // conv_cross_b: the chunk's data block and the point's offset
                    data_block<8> blk{v.data, c, BS};
                    d0[g] = (U0)f(u, blk, pnt, i, j, k);
                } else {  // conv3_b: three fields
                    cp_block<T2, E> x3{const_cast<T2*>(tile2[NP >= 3 ? b : 0])};
                    U0 r1 = 0;
                    U1 r2 = 0;
                    U2 r3 = 0;
                    data_block<8> blk{v.data, c, BS};
                    f(r1, r2, r3, u, w, x3, blk, pnt, i, j, k);
                    d0[g] = r1;
                    d1[g] = r2;
                    d2[g] = r3;
                }
            }
        }
#pragma unroll
        for (int q = 0; q < NPT; ++q) m_cur[q] = m_next[q];
    }
    async_wait_group<0>();
}

}  // namespace detail

// The chunk slot that insertBlock hands to a CTA: ec.template get<p>()[offset] is
// property p of the slot's point `offset`, ec.template get<pMask>()[offset] its
// mask byte (the encap of the reference's blockMap.insert, BlockMapGpu_ker.cuh:199-227).
// The same encap over a grid chunk is the data block a stencil functor gets
// (dataBlockLoad / dataBlockStore).
template <typename AggregateT, unsigned BS>
struct block_encap {
    using props = typename AggregateT::type;
    static constexpr unsigned nprop = std::tuple_size<props>::value;
    void* val[8];   // arrays of the properties (pools or grid data)
    uint8_t* mask;  // mask array
    int64_t slot;   // slot or chunk position in those arrays
    template <unsigned p>
    __device__ auto get() const {
        if constexpr (p == nprop) {
            return mask + slot * BS;
        } else {
            using T = typename std::tuple_element<p, props>::type;
            return static_cast<T*>(val[p]) + slot * BS;
        }
    }
};

// BlockMapGpu_ker<>::setExist / setPadding / unsetPadding / exist
// (src/SparseGridGpu/BlockMapGpu_ker.cuh): mask byte helpers of user kernels.
template <typename A = void, unsigned B = 0, typename C = void>
struct BlockMapGpu_ker {
    static __device__ __forceinline__ void setExist(unsigned char& m) { m |= 1; }
    static __device__ __forceinline__ void unsetExist(unsigned char& m) { m &= ~1; }
    static __device__ __forceinline__ void setPadding(unsigned char& m) { m |= 2; }
    static __device__ __forceinline__ void unsetPadding(unsigned char& m) { m &= ~2; }
    static __device__ __forceinline__ bool exist(unsigned char m) { return m & 1; }
    static __device__ __forceinline__ bool isPadding(unsigned char m) { return m & 2; }
};

// ------------------------------------------------------------------ device view
// Returned by SparseGridGpu::toKernel(); passed by value to user kernels.
template <typename AggregateT, unsigned E>
struct SparseGridGpu_ker {
    sgb_view v;
    unsigned long long bck[8];  // background of every property, as raw bytes (device remove)
    int64_t* pool_lin;
    void* pool_val[8];
    int32_t* pool_cnt;
    int nslot;
    // chunk-slot pools of insertBlock: key, per-property values, mask bytes, per-CTA count
    int64_t* blk_key;
    void* blk_val[8];
    uint8_t* blk_mask;
    int32_t* blk_cnt;
    int nblkslot;
    using props = typename AggregateT::type;
    using AggregateType = block_aggregate<AggregateT, E * E * E>;
    using AggregateBlockType = AggregateType;
    using indexT_ = long;
    static constexpr unsigned blockEdgeSize_ = E;
    static constexpr unsigned d = 3;
    static constexpr unsigned dims = 3;
    static constexpr unsigned pMask = std::tuple_size<props>::value;
    static constexpr unsigned blockSize = E * E * E;

    __host__ __device__ static constexpr unsigned getBlockEdgeSize() { return E; }

    // grid_smb::LinId (src/Grid/Geometry/grid_smb.hpp:176-190)
    template <typename CoordT>
    __device__ int64_t getLinId(const grid_key_dx<3, CoordT>& c) const {
        const int64_t b = detail::block_key(v.zorder, v.bsz, c.get(0) / E, c.get(1) / E, c.get(2) / E);
        const int64_t l = ((c.get(2) % E) * E + c.get(1) % E) * E + c.get(0) % E;
        return b * (E * E * E) + l;
    }

    // grid_smb::BlockLinId of a block coordinate (src/Grid/Geometry/grid_smb.hpp:280-299)
    template <typename CoordT>
    __device__ int64_t getBlockLinId(const grid_key_dx<3, CoordT>& blockCoord) const {
        return detail::block_key(v.zorder, v.bsz, blockCoord.get(0), blockCoord.get(1), blockCoord.get(2));
    }

    // global coordinate of point `offset` of the chunk at block coordinate blockCoord
    // (SparseGridGpu_ker::getGlobalCoord)
    template <typename CoordT>
    __device__ grid_key_dx<3, CoordT> getGlobalCoord(const grid_key_dx<3, CoordT>& blockCoord, unsigned offset) const {
        grid_key_dx<3, CoordT> k;
        k.set_d(0, blockCoord.get(0) * E + offset % E);
        k.set_d(1, blockCoord.get(1) * E + (offset / E) % E);
        k.set_d(2, blockCoord.get(2) * E + offset / (E * E));
        return k;
    }

    // vector_sparse_gpu_ker::init (map_vector_sparse_cuda_ker.cuh:129-140)
    __device__ void init() const {
        if (threadIdx.x == 0 && threadIdx.y == 0 && threadIdx.z == 0) {
            detail::sgb_pool_counter = 0;
            detail::sgb_block_counter = 0;
        }
        __syncthreads();
    }

    // insertBlock(blockId, stride) (BlockMapGpu_ker.cuh:199-227): every thread of the CTA calls
    // it; the thread with threadIdx.x % stride == 0 takes one chunk slot of this CTA's pool for
    // chunk id blockId, and the threads with the same threadIdx.x / stride get its encap.
    // Points written through the encap whose mask byte has EXIST set are inserted at the next
    // flush, in (CTA, slot, offset) order after the CTA's insert<p> points.  A CTA that takes
    // more slots than the pool holds makes the next flush fail (SGB_ERANGE).
    template <unsigned nChunksPerBlocks = 1>
    __device__ block_encap<AggregateT, E * E * E> insertBlock(int64_t blockId, unsigned stride = 8192) const {
        __shared__ int slot_of[nChunksPerBlocks];
        const unsigned group = threadIdx.x / stride;
        const int64_t blk = blockIdx.x + (int64_t)gridDim.x * (blockIdx.y + (int64_t)gridDim.y * blockIdx.z);
        if (threadIdx.x % stride == 0 && threadIdx.y == 0 && threadIdx.z == 0) {
            int slot = atomicAdd(&detail::sgb_block_counter, 1);
            slot = slot < nblkslot ? slot : nblkslot - 1;  // an overflowing pool is reported at flush
            blk_key[blk * nblkslot + slot] = blockId;
            slot_of[group] = slot;
        }
        __syncthreads();
        block_encap<AggregateT, E * E * E> ec;
        for (int p = 0; p < 8; ++p) ec.val[p] = blk_val[p];
        ec.mask = blk_mask;
        ec.slot = blk * nblkslot + slot_of[group];
        return ec;
    }

    // insert<p>(coord): one slot of this CTA's pool (map_vector_sparse_cuda_ker.cuh:309-318)
    template <unsigned p, typename CoordT>
    __device__ typename std::tuple_element<p, props>::type& insert(const grid_key_dx<3, CoordT>& coord) const {
        using T = typename std::tuple_element<p, props>::type;
        const int64_t blk = blockIdx.x + (int64_t)gridDim.x * (blockIdx.y + (int64_t)gridDim.y * blockIdx.z);
        int slot = atomicAdd(&detail::sgb_pool_counter, 1);
        const bool ok = slot < nslot;
        slot = ok ? slot : nslot - 1;  // an overflowing pool is reported at flush
        const int64_t idx = blk * nslot + slot;
        pool_lin[idx] = getLinId(coord);
        return static_cast<T*>(pool_val[p])[idx];
    }

    // flush_block_insert (map_vector_sparse_cuda_ker.cuh:424-439)
    __device__ void flush_block_insert() const {
        __syncthreads();
        if (threadIdx.x == 0 && threadIdx.y == 0 && threadIdx.z == 0) {
            const int64_t blk = blockIdx.x + (int64_t)gridDim.x * (blockIdx.y + (int64_t)gridDim.y * blockIdx.z);
            pool_cnt[blk] = detail::sgb_pool_counter;
            if (blk_cnt) blk_cnt[blk] = detail::sgb_block_counter;
        }
    }

    // get<p>(coord): value, or the background when the point does not exist
    // remove(coord) (SparseGridGpu_ker.cuh:664-668 -> BlockMapGpu_ker::remove, BlockMapGpu_ker.cuh:
    // 310-331): the point's mask byte is cleared (no effect if its chunk is absent); its properties
    // get their backgrounds, which the grid keeps in every non-existing point
    template <typename CoordT>
    __device__ void remove(const grid_key_dx<3, CoordT>& coord) const {
        const int64_t lin = getLinId(coord), bs = E * E * E;
        const int64_t pos = detail::find_key(v.keys, v.n, lin / bs);
        if (pos < 0) return;
        const int64_t idx = pos * bs + lin % bs;
        const_cast<uint8_t*>(v.mask)[idx] = 0;
        clear_props(idx, std::make_index_sequence<std::tuple_size<props>::value>{});
    }
    template <size_t... I>
    __device__ void clear_props(int64_t idx, std::index_sequence<I...>) const {
        (clear_prop<I>(idx), ...);
    }
    template <size_t I>
    __device__ void clear_prop(int64_t idx) const {
        using T = typename std::tuple_element<I, props>::type;
        T b;
        memcpy(&b, &bck[I], sizeof(T));
        static_cast<T*>(v.data[I])[idx] = b;
    }

    template <unsigned p, typename CoordT>
    __device__ typename std::tuple_element<p, props>::type get(const grid_key_dx<3, CoordT>& coord) const {
        using T = typename std::tuple_element<p, props>::type;
        const int64_t lin = getLinId(coord), bs = E * E * E;
        int64_t pos = detail::find_key(v.keys, v.n, lin / bs);
        if (pos < 0) pos = v.n;
        const int64_t idx = pos * bs + lin % bs;
        return (v.mask[idx] & 1) ? static_cast<const T*>(v.data[p])[idx]
                                 : static_cast<const T*>(v.data[p])[v.n * bs + lin % bs];
    }

    template <typename CoordT>
    __device__ bool isPadding(const grid_key_dx<3, CoordT>& coord) const {
        const int64_t lin = getLinId(coord), bs = E * E * E;
        const int64_t pos = detail::find_key(v.keys, v.n, lin / bs);
        return pos >= 0 && (v.mask[pos * bs + lin % bs] & 3) == 3;
    }

    // ---------------------------------------------------------------- stencil functor interface
    // (SparseGridGpu_ker.cuh:297-372, 551-604, 877-896) for functors applied by applyStencils<S>
    static __device__ __forceinline__ bool exist(unsigned char m) { return m & 1; }
    static __device__ __forceinline__ bool isPaddingMask(unsigned char m) { return m & 2; }

    // point coordinate of a linear point id (grid_smb::InvLinId, grid_smb.hpp:263-277)
    __device__ grid_key_dx<3, int> getCoord(int64_t linId) const {
        constexpr int64_t bs = E * E * E;
        int64_t bc[3];
        detail::block_coords(v.zorder, v.bsz, linId / bs, bc);
        const int o = (int)(linId % bs);
        grid_key_dx<3, int> k;
        k.set_d(0, (int)(bc[0] * E + o % E));
        k.set_d(1, (int)(bc[1] * E + (o / E) % E));
        k.set_d(2, (int)(bc[2] * E + o / (E * E)));
        return k;
    }

    // the chunk at position pos as a data block (dataBuffer.get(pos) in the reference)
    __device__ block_encap<AggregateT, E * E * E> getDataBlock(int64_t pos) const {
        block_encap<AggregateT, E * E * E> ec;
        for (int p = 0; p < 8; ++p) ec.val[p] = v.data[p];
        ec.mask = const_cast<uint8_t*>(v.mask);
        ec.slot = pos;
        return ec;
    }

    // enlarged-block (chunk plus one-point halo, (E+2)^3) indexing
    static __host__ __device__ constexpr unsigned getEnlargedBlockSize() { return (E + 2) * (E + 2) * (E + 2); }
    __device__ grid_key_dx<3, int> getCoordInEnlargedBlock(unsigned offset) const {
        grid_key_dx<3, int> k;
        k.set_d(0, (int)(offset % E) + 1);
        k.set_d(1, (int)((offset / E) % E) + 1);
        k.set_d(2, (int)(offset / (E * E)) + 1);
        return k;
    }
    __device__ unsigned getLinIdInEnlargedBlock(unsigned offset) const {
        return (offset % E + 1) + (E + 2) * (((offset / E) % E + 1) + (E + 2) * (offset / (E * E) + 1));
    }
    template <typename C>
    __device__ unsigned getNeighbourLinIdInEnlargedBlock(const grid_key_dx<3, C>& base, unsigned dimension,
                                                          char offset) const {
        int c[3] = {(int)base.get(0), (int)base.get(1), (int)base.get(2)};
        c[dimension] += offset;
        return (unsigned)(c[0] + (int)(E + 2) * (c[1] + (int)(E + 2) * c[2]));
    }
    template <typename C>
    __device__ unsigned getNeighbourLinIdInEnlargedBlock(const grid_key_dx<3, C>& base,
                                                          const grid_key_dx<3, C>& offsets) const {
        const int c0 = (int)(base.get(0) + offsets.get(0)), c1 = (int)(base.get(1) + offsets.get(1)),
                  c2 = (int)(base.get(2) + offsets.get(2));
        return (unsigned)(c0 + (int)(E + 2) * (c1 + (int)(E + 2) * c2));
    }

    template <unsigned p>
    __device__ ScalarTypeOf<AggregateType, p> background() const {
        ScalarTypeOf<AggregateType, p> b;
        memcpy(&b, &bck[p], sizeof(b));
        return b;
    }

    // chunk position of the halo cell (dx, dy, dz) of chunk `chunk` (nz of them non-zero), -1 when
    // absent.  NNFull: the 26 neighbours.  NNStar (NNStar::getNNskin, SparseGridGpu_ker_util.hpp:
    // 114-139): faces read their neighbour; edge and corner cells read neighbour 0, the -x chunk,
    // at the wrapped local coordinate, as the reference's ghost-layer map does.
    __device__ int64_t halo_chunk(int64_t chunk, int dx, int dy, int dz, int nz) const {
        if (v.nn_kind == SGB_NN_FULL) return v.nn[chunk * 27 + (dx + 1) + 3 * (dy + 1) + 9 * (dz + 1)];
        const int slot = nz > 1 ? 0 : (dx ? (dx < 0 ? 0 : 1) : dy ? (dy < 0 ? 2 : 3) : (dz < 0 ? 4 : 5));
        return v.nn[chunk * 8 + slot];
    }

    // loadGhostBlock<p> (SparseGridGpu_ker.cuh:551-571 -> loadGhostBlock_impl, SparseGridGpu_ker_util.hpp:
    // 487-564): every thread of the CTA fills cells of the (E+2)^3 tile of chunk pos with property p;
    // a cell whose source mask byte is 0 (or whose chunk is absent) takes the background (the mask
    // property takes the mask byte itself).  The optional mask tile receives the mask bytes.
    template <unsigned p, typename AggrWrapperT>
    __device__ void loadGhostBlock(const AggrWrapperT&, openfpm::sparse_index<unsigned> pos,
                                   ScalarTypeOf<AggregateType, p>* sharedRegion) const {
        load_tile<p>(pos.id, sharedRegion, nullptr);
    }
    template <unsigned p, typename AggrWrapperT>
    __device__ void loadGhostBlock(const AggrWrapperT&, openfpm::sparse_index<unsigned> pos,
                                   ScalarTypeOf<AggregateType, p>* sharedRegion, unsigned char* mask) const {
        load_tile<p>(pos.id, sharedRegion, mask);
    }
    template <unsigned p>
    __device__ void load_tile(int64_t chunk, ScalarTypeOf<AggregateType, p>* tile, unsigned char* mtile) const {
        using T = ScalarTypeOf<AggregateType, p>;
        constexpr int TE = E + 2, TT = TE * TE * TE, BS = E * E * E;
        const int nthr = blockDim.x * blockDim.y * blockDim.z;
        const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
        T b{};
        if constexpr (p != pMask) b = background<p>();
        for (int cell = tid; cell < TT; cell += nthr) {
            const int tx = cell % TE, ty = (cell / TE) % TE, tz = cell / (TE * TE);
            const int dx = tx == 0 ? -1 : (tx == TE - 1 ? 1 : 0), dy = ty == 0 ? -1 : (ty == TE - 1 ? 1 : 0),
                      dz = tz == 0 ? -1 : (tz == TE - 1 ? 1 : 0);
            const int nz = (dx != 0) + (dy != 0) + (dz != 0);
            const int64_t sc = nz ? halo_chunk(chunk, dx, dy, dz, nz) : chunk;
            const int lx = (tx - 1 + E) % E, ly = (ty - 1 + E) % E, lz = (tz - 1 + E) % E;
            uint8_t m = 0;
            T val = b;
            if (sc >= 0) {
                const int64_t idx = sc * BS + lx + E * (ly + E * lz);
                m = v.mask[idx];
                if constexpr (p == pMask) val = m;
                else if (m != 0) val = static_cast<const T*>(v.data[p])[idx];
            }
            tile[cell] = val;
            if (mtile) mtile[cell] = m;
        }
    }

    // storeBlock<p> (SparseGridGpu_ker.cuh:598-604, 877-896): thread `offset` writes its point of the
    // tile into the chunk.  Points that do not exist receive this property's background (the
    // reference writes the tile value, the source's background there; every read of a point that
    // does not exist returns the background, so the two cannot be told apart).
    template <unsigned p, typename AggrWrapperT>
    __device__ void storeBlock(AggrWrapperT& block, ScalarTypeOf<AggregateType, p>* sharedRegion) const {
        constexpr unsigned BS = E * E * E;
        const unsigned pos = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
        if (pos < BS) {
            const unsigned char m = block.template get<pMask>()[pos];
            block.template get<p>()[pos] = m ? sharedRegion[getLinIdInEnlargedBlock(pos)] : background<p>();
        }
    }

    // getNNPoint<NN> (SparseGridGpu_ker.cuh:297-327): the chunk position and offset of the point at
    // `mov` from point `offset` of chunk pos (at most one chunk away); an absent chunk is the
    // background chunk.  NN is the grid's neighbourhood (NNFull, setNNType<NNFull<3>>).
    template <typename NN_type, typename I>
    __device__ block_offset<I> getNNPoint(openfpm::sparse_index<unsigned> pos, unsigned offset,
                                          const grid_key_dx<3, I>& mov) const {
        I c[3];
        for (int i = 0; i < 3; ++i) {
            c[i] = mov.get(i) + (I)(offset % E);
            offset /= E;
        }
        unsigned nn_index = 0, offset_nn = 0;
        const bool out = NN_type::template getNNindex_offset<E>(c, nn_index, offset_nn);
        int64_t nnb = pos.id;
        if (out) {
            const int32_t q = v.nn[nn_index + NN_type::nNN * (int64_t)pos.id];
            nnb = q < 0 ? v.n : q;
        }
        return block_offset<I>{(I)nnb, (I)offset_nn};
    }
    // get<p>(block_offset): the value stored at that chunk position and offset
    template <unsigned p, typename I>
    __device__ ScalarTypeOf<AggregateType, p> get(const block_offset<I>& bo) const {
        return static_cast<const ScalarTypeOf<AggregateType, p>*>(v.data[p])[(int64_t)bo.pos * (E * E * E) + bo.off];
    }
};

// ------------------------------------------------------------------ user stencil functors
namespace detail {
template <typename S, typename = void>
struct is_fixed_stencil : std::false_type {};
template <typename S>
struct is_fixed_stencil<S, std::void_t<decltype(S::kind)>> : std::true_type {};

// applyStencilInPlace (SparseGridGpu_kernels.cuh:1045-1094): one CTA of BS threads per chunk,
// thread `offset` one point; the point's mask is cleared outside the inclusive box; the functor
// gets the view, the chunk id and position, the point's offset and coordinate, the chunk's data
// block (to load from and store to) and the mask byte.
template <typename S, typename Ker, typename... Args>
__global__ void apply_stencil_inplace(Box<3, int> bx, Ker sg, Args... args) {
    constexpr unsigned BS = Ker::blockSize;
    const unsigned dataBlockPos = blockIdx.x;
    const unsigned offset = threadIdx.x;
    if (dataBlockPos >= sg.v.n) return;
    auto dataBlock = sg.getDataBlock(dataBlockPos);
    const int64_t dataBlockId = sg.v.keys[dataBlockPos];
    grid_key_dx<3, int> pointCoord = sg.getCoord(dataBlockId * BS + offset);
    unsigned char curMask = 0;
    if (offset < BS) {
        curMask = sg.v.mask[(int64_t)dataBlockPos * BS + offset];
        for (int i = 0; i < 3; ++i)
            if (pointCoord.get(i) < bx.getLow(i) || pointCoord.get(i) > bx.getHigh(i)) curMask = 0;
    }
    openfpm::sparse_index<unsigned> sdataBlockPos;
    sdataBlockPos.id = dataBlockPos;
    S::stencil(sg, (unsigned)dataBlockId, sdataBlockPos, offset, pointCoord, dataBlock, dataBlock, curMask, args...);
}

// applyStencilInPlaceNoShared (SparseGridGpu_kernels.cuh:1096-1150): one thread per existing point
// of the existing-point list (chunk position * BS + offset), no shared-memory tiles.
template <typename S, typename Ker, typename... Args>
__global__ void apply_stencil_noshared(Box<3, int> bx, Ker sg, const uint32_t* ids, int64_t nids, Args... args) {
    constexpr unsigned BS = Ker::blockSize;
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= nids) return;
    const uint32_t id = ids[t];
    const unsigned dataBlockPos = id / BS, offset = id % BS;
    auto dataBlock = sg.getDataBlock(dataBlockPos);
    const int64_t dataBlockId = sg.v.keys[dataBlockPos];
    grid_key_dx<3, int> pointCoord = sg.getCoord(dataBlockId * BS + offset);
    unsigned char curMask = sg.v.mask[(int64_t)dataBlockPos * BS + offset];
    for (int i = 0; i < 3; ++i)
        if (pointCoord.get(i) < bx.getLow(i) || pointCoord.get(i) > bx.getHigh(i)) curMask = 0;
    openfpm::sparse_index<unsigned> sdataBlockPos;
    sdataBlockPos.id = dataBlockPos;
    S::stencil(sg, (unsigned)dataBlockId, sdataBlockPos, offset, pointCoord, dataBlock, dataBlock, curMask, args...);
}
}  // namespace detail

// ------------------------------------------------------------------ host class
// layout and linearizer tags of the reference's template parameters
template <typename T>
struct memory_traits_inte {};
template <unsigned dim, unsigned blockEdgeSize, typename indexT = long>
struct grid_smb {
    static constexpr int zorder = 0;
};
template <unsigned dim, unsigned blockEdgeSize, typename indexT = long>
struct grid_zmb {
    static constexpr int zorder = 1;
};

template <unsigned dim, typename AggregateT, unsigned blockEdgeSize = 8, unsigned threadBlockSize = 512,
          typename indexT = long, template <typename> class layout_base = memory_traits_inte,
          typename linearizer = grid_smb<dim, blockEdgeSize, indexT>>
class SparseGridGpu {
    static_assert(dim == 3, "this build runs 3-D sparse grids");
    static_assert(blockEdgeSize == 8 || blockEdgeSize == 4, "chunk edge 8 or 4");
    using props = typename AggregateT::type;
    static constexpr unsigned nprop = std::tuple_size<props>::value;
    static constexpr unsigned bs = blockEdgeSize * blockEdgeSize * blockEdgeSize;

    sgb_grid* g_ = nullptr;
    size_t size_[3];
    unsigned long long bck_raw_[8] = {};  // backgrounds as raw bytes, for the view's device remove
    int nn_kind_ = SGB_NN_STAR;  // setNNType
    // device insert pools
    int64_t npools_ = 0, nslot_ = 0;
    int64_t* pool_lin_ = nullptr;
    void* pool_val_[8] = {};
    int32_t* pool_cnt_ = nullptr;
    // insertBlock chunk-slot pools
    int64_t nblkslot_ = 0;
    int64_t* blk_key_ = nullptr;
    void* blk_val_[8] = {};
    uint8_t* blk_mask_ = nullptr;
    int32_t* blk_cnt_ = nullptr;
    // host copies filled by deviceToHost
    std::vector<int64_t> h_keys_;
    std::vector<std::vector<unsigned char>> h_data_;
    std::vector<uint8_t> h_mask_;

    void free_pools() {
        if (pool_lin_) cudaFree(pool_lin_);
        for (auto& p : pool_val_)
            if (p) cudaFree(p), p = nullptr;
        if (pool_cnt_) cudaFree(pool_cnt_);
        pool_lin_ = nullptr;
        pool_cnt_ = nullptr;
        for (auto& p : blk_val_)
            if (p) cudaFree(p), p = nullptr;
        if (blk_key_) cudaFree(blk_key_);
        if (blk_mask_) cudaFree(blk_mask_);
        if (blk_cnt_) cudaFree(blk_cnt_);
        blk_key_ = nullptr;
        blk_mask_ = nullptr;
        blk_cnt_ = nullptr;
        npools_ = nslot_ = nblkslot_ = 0;
    }

    template <typename... ops>
    static std::vector<int> op_list() {
        std::vector<int> o(nprop, SGB_OP_NONE);
        int dummy[] = {0, (o[ops::prop] = ops::op, 0)...};
        (void)dummy;
        return o;
    }

   public:
    static constexpr unsigned dims = dim;
    static constexpr unsigned blockEdgeSize_ = blockEdgeSize;
    using device_grid_type = SparseGridGpu_ker<AggregateT, blockEdgeSize>;

    // SparseGridGpu(const size_t (&res)[dim], unsigned stencilSupportRadius = 1) (SparseGridGpu.hpp:1694-1698)
    explicit SparseGridGpu(const size_t (&res)[dim], unsigned stencilSupportRadius = 1, int device = 0) {
        if (stencilSupportRadius != 1) throw sgb_error(SGB_ENOTSUP, "stencilSupportRadius");
        int64_t sz[3];
        for (unsigned d = 0; d < 3; ++d) size_[d] = res[d], sz[d] = (int64_t)res[d];
        auto types = detail::types_of<props>::get();
        check(sgb_create(&g_, 3, blockEdgeSize, sz, (int)nprop, types.data(), device), "sgb_create");
        if (linearizer::zorder) check(sgb_set_linearizer(g_, SGB_LIN_ZMB), "sgb_set_linearizer");
    }
    SparseGridGpu(const SparseGridGpu&) = delete;
    SparseGridGpu& operator=(const SparseGridGpu&) = delete;
    ~SparseGridGpu() {
        free_pools();
        if (g_) sgb_destroy(g_);
    }

    sgb_grid* handle() const { return g_; }
    static constexpr unsigned getBlockEdgeSize() { return blockEdgeSize; }
    constexpr unsigned getBlockSize() const { return bs; }

    template <unsigned p>
    void setBackgroundValue(typename std::tuple_element<p, props>::type v) {
        check(sgb_set_background(g_, p, &v), "setBackgroundValue");
        bck_raw_[p] = 0;
        std::memcpy(&bck_raw_[p], &v, sizeof(v));
    }

    // setGPUInsertBuffer(nBlock, nSlot) (SparseGridGpu.hpp:2270-2277)
    void setGPUInsertBuffer(int64_t nBlock, int64_t nSlot) {
        free_pools();
        npools_ = nBlock;
        nslot_ = nSlot;
        const size_t n = (size_t)nBlock * nSlot;
        if (cudaMalloc(&pool_lin_, n * 8) != cudaSuccess || cudaMalloc(&pool_cnt_, nBlock * 4) != cudaSuccess)
            throw sgb_error(SGB_ENOMEM, "setGPUInsertBuffer");
        auto types = detail::types_of<props>::get();
        for (unsigned p = 0; p < nprop; ++p) {
            const size_t es = types[p] == SGB_F64 ? 8 : (types[p] == SGB_U8 ? 1 : 4);
            if (cudaMalloc(&pool_val_[p], n * es) != cudaSuccess) throw sgb_error(SGB_ENOMEM, "setGPUInsertBuffer");
        }
        cudaMemset(pool_cnt_, 0, nBlock * 4);
        // insertBlock takes whole chunk slots, as every insert does in the reference: up to nSlot per
        // CTA, bounded so that the chunk-slot pools stay within 512 MiB (at least one slot per CTA)
        size_t per_slot = bs;  // mask bytes
        for (unsigned p = 0; p < nprop; ++p) per_slot += (size_t)bs * (types[p] == SGB_F64 ? 8 : (types[p] == SGB_U8 ? 1 : 4));
        const size_t cap = (size_t)512 << 20;
        nblkslot_ = std::max<int64_t>(1, std::min<int64_t>(nSlot, (int64_t)(cap / std::max<size_t>(1, per_slot * nBlock))));
        const size_t nb = (size_t)nBlock * nblkslot_;
        if (cudaMalloc(&blk_key_, nb * 8) != cudaSuccess || cudaMalloc(&blk_mask_, nb * bs) != cudaSuccess ||
            cudaMalloc(&blk_cnt_, nBlock * 4) != cudaSuccess)
            throw sgb_error(SGB_ENOMEM, "setGPUInsertBuffer (block slots)");
        for (unsigned p = 0; p < nprop; ++p) {
            const size_t es = types[p] == SGB_F64 ? 8 : (types[p] == SGB_U8 ? 1 : 4);
            if (cudaMalloc(&blk_val_[p], nb * bs * es) != cudaSuccess)
                throw sgb_error(SGB_ENOMEM, "setGPUInsertBuffer (block slots)");
        }
        cudaMemset(blk_mask_, 0, nb * bs);  // initializeInsertBuffer (BlockMapGpu_kernels.cuh:110-139)
        cudaMemset(blk_cnt_, 0, nBlock * 4);
    }
    void setGPUInsertBuffer(dim3 nBlock, dim3 nSlot) {
        setGPUInsertBuffer((int64_t)nBlock.x * nBlock.y * nBlock.z, (int64_t)nSlot.x * nSlot.y * nSlot.z);
    }

    device_grid_type toKernel() {
        device_grid_type k{};
        check(sgb_get_view(g_, nn_kind_, &k.v, nullptr), "toKernel");
        // the kernel may remove points: cached existence data is rebuilt when next needed
        check(sgb_existence_changed(g_), "toKernel");
        for (unsigned p = 0; p < nprop && p < 8; ++p) k.bck[p] = bck_raw_[p];
        k.pool_lin = pool_lin_;
        for (int p = 0; p < 8; ++p) k.pool_val[p] = pool_val_[p];
        k.pool_cnt = pool_cnt_;
        k.nslot = (int)nslot_;
        k.blk_key = blk_key_;
        for (int p = 0; p < 8; ++p) k.blk_val[p] = blk_val_[p];
        k.blk_mask = blk_mask_;
        k.blk_cnt = blk_cnt_;
        k.nblkslot = (int)nblkslot_;
        return k;
    }

    // flush<v_reduce...>(ctx, opt) (SparseGridGpu.hpp:772-779)
    template <typename... v_reduce>
    void flush(gpu::ofp_context_t&, flush_type = FLUSH_ON_DEVICE) {
        if (npools_) {
            check(sgb_insert_pools(g_, npools_, nslot_, pool_cnt_, pool_lin_, pool_val_, nullptr), "flush (pools)");
            cudaMemset(pool_cnt_, 0, npools_ * 4);
            check(sgb_insert_blocks(g_, npools_, nblkslot_, blk_cnt_, blk_key_, blk_val_, blk_mask_, nullptr),
                  "flush (block slots)");
            cudaMemset(blk_cnt_, 0, npools_ * 4);
            cudaMemset(blk_mask_, 0, (size_t)npools_ * nblkslot_ * bs);
        }
        auto ops = op_list<v_reduce...>();
        check(sgb_flush(g_, ops.data(), nullptr), "flush");
    }

    template <typename NN = NNStar<dim>>
    void findNeighbours() {
        check(sgb_find_neighbours(g_, NN::kind, nullptr), "findNeighbours");
    }
    template <typename NN>
    void setNNType() {
        nn_kind_ = NN::kind;
    }
    template <typename NN = NNStar<dim>>
    void tagBoundaries(gpu::ofp_context_t&, No_check = No_check(),
                       tag_boundaries opt = tag_boundaries::NO_CALCULATE_EXISTING_POINTS) {
        check(sgb_tag_boundaries(g_, NN::kind, nullptr), "tagBoundaries");
        if (opt == tag_boundaries::CALCULATE_EXISTING_POINTS)
            check(sgb_calc_existing_points(g_, nullptr, nullptr), "tagBoundaries (existing points)");
        cudaDeviceSynchronize();  // as the reference (SparseGridGpu.hpp:2393)
    }

    Box<dim, int> getBox() const {
        Box<dim, int> b;
        for (unsigned d = 0; d < dim; ++d) b.lo[d] = 0, b.hi[d] = (int)size_[d];
        return b;
    }

    // applyStencils<S>(box, mode, args...) (SparseGridGpu.hpp:2704-2734).  HeatStencil, Conv3x3x3 and
    // Conv3x3x3_noshared run the library's fixed-function kernels; any other S is a user functor
    // with the reference's contract (typedef stencil_type, static __device__ stencil(sparseGrid,
    // dataBlockId, dataBlockIdPos, offset, pointCoord, dataBlockLoad, dataBlockStore, curMask,
    // args...)), run one CTA per chunk (STENCIL_MODE_INPLACE) or one thread per existing point
    // (STENCIL_MODE_INPLACE_NO_SHARED, after tagBoundaries(..., CALCULATE_EXISTING_POINTS)).
    template <typename S, typename... Args>
    void applyStencils(const Box<dim, int>& box, StencilMode mode, Args... args) {
        if constexpr (detail::is_fixed_stencil<S>::value) {
            apply_fixed<S>(box, args...);
        } else {
            apply_user<S>(box, mode, args...);
        }
    }

    // conv family with user __device__ functions (SparseGridGpu.hpp:2568-2683)
    template <unsigned p_src, unsigned p_dst, unsigned stencil_size, typename F>
    void conv_cross(grid_key_dx<3> start, grid_key_dx<3> stop, F f) {
        launch_conv<1, 0, p_src, p_src, p_dst, p_dst>(start, stop, f);
    }
    template <unsigned p_src, unsigned p_dst, unsigned stencil_size, typename F>
    void conv(grid_key_dx<3> start, grid_key_dx<3> stop, F f) {
        launch_conv<1, 1, p_src, p_src, p_dst, p_dst>(start, stop, f);
    }
    // conv_cross_b (SparseGridGpu.hpp:2606-2621): f(cp_block, data_block, offset, i, j, k) over the
    // NNStar halo (edge and corner cells read neighbour 0 as the reference's ghost-layer map does),
    // written at active points
    template <unsigned p_src, unsigned p_dst, unsigned stencil_size, typename F>
    void conv_cross_b(grid_key_dx<3> start, grid_key_dx<3> stop, F f) {
        const int keep = nn_kind_;
        nn_kind_ = SGB_NN_STAR;
        launch_conv<1, 4, p_src, p_src, p_dst, p_dst>(start, stop, f);
        nn_kind_ = keep;
    }
    template <unsigned s1, unsigned s2, unsigned d1, unsigned d2, unsigned stencil_size, typename F>
    void conv2(grid_key_dx<3> start, grid_key_dx<3> stop, F f) {
        launch_conv<2, 2, s1, s2, d1, d2>(start, stop, f);
    }
    template <unsigned s1, unsigned s2, unsigned d1, unsigned d2, unsigned stencil_size, typename F>
    void conv2_b(grid_key_dx<3> start, grid_key_dx<3> stop, F f) {
        launch_conv<2, 3, s1, s2, d1, d2>(start, stop, f);
    }
    // conv3_b (SparseGridGpu.hpp:2646-2663): f(r1, r2, r3, u, v, w, data_block, offset, i, j, k) over three
    // source fields, the results written at active points
    template <unsigned s1, unsigned s2, unsigned s3, unsigned d1, unsigned d2, unsigned d3, unsigned stencil_size,
              typename F>
    void conv3_b(grid_key_dx<3> start, grid_key_dx<3> stop, F f) {
        launch_conv<3, 5, s1, s2, d1, d2, s3, d3>(start, stop, f);
    }

    // deviceToHost<p...>(): the block map and listed properties to host copies
    template <unsigned... prp>
    void deviceToHost() {
        int64_t n;
        sgb_nchunks(g_, &n);
        h_keys_.resize(n);
        h_mask_.resize((n + 1) * bs);
        auto types = detail::types_of<props>::get();
        h_data_.assign(nprop, {});
        std::vector<void*> ptrs(nprop, nullptr);
        for (unsigned p = 0; p < nprop; ++p) {
            const size_t es = types[p] == SGB_F64 ? 8 : (types[p] == SGB_U8 ? 1 : 4);
            h_data_[p].resize((n + 1) * bs * es);
            ptrs[p] = h_data_[p].data();
        }
        check(sgb_download_map(g_, h_keys_.data(), ptrs.data(), h_mask_.data(), nullptr), "deviceToHost");
    }

    // host get<p>(coord) after deviceToHost (BlockMapGpu.hpp:108-126)
    template <unsigned p, typename CoordT>
    typename std::tuple_element<p, props>::type get(const grid_key_dx<dim, CoordT>& c) const {
        using T = typename std::tuple_element<p, props>::type;
        int64_t bsz[3];
        for (int d = 0; d < 3; ++d) bsz[d] = ((int64_t)size_[d] + blockEdgeSize - 1) / blockEdgeSize;
        const int64_t b = detail::block_key(linearizer::zorder, bsz, c.get(0) / blockEdgeSize, c.get(1) / blockEdgeSize,
                                            c.get(2) / blockEdgeSize);
        const int64_t l = ((c.get(2) % blockEdgeSize) * blockEdgeSize + c.get(1) % blockEdgeSize) * blockEdgeSize +
                          c.get(0) % blockEdgeSize;
        const int64_t n = (int64_t)h_keys_.size();
        int64_t lo = 0, hi = n;
        while (lo < hi) {
            int64_t mid = (lo + hi) / 2;
            if (h_keys_[mid] < b) lo = mid + 1;
            else hi = mid;
        }
        const int64_t pos = (lo < n && h_keys_[lo] == b) ? lo : n;
        const T* d = reinterpret_cast<const T*>(h_data_[p].data());
        return (h_mask_[pos * bs + l] & 1) ? d[pos * bs + l] : d[n * bs + l];
    }
    template <typename CoordT>
    unsigned char getFlag(const grid_key_dx<dim, CoordT>& c) const {
        int64_t bsz[3];
        for (int d = 0; d < 3; ++d) bsz[d] = ((int64_t)size_[d] + blockEdgeSize - 1) / blockEdgeSize;
        const int64_t b = detail::block_key(linearizer::zorder, bsz, c.get(0) / blockEdgeSize, c.get(1) / blockEdgeSize,
                                            c.get(2) / blockEdgeSize);
        const int64_t l = ((c.get(2) % blockEdgeSize) * blockEdgeSize + c.get(1) % blockEdgeSize) * blockEdgeSize +
                          c.get(0) % blockEdgeSize;
        for (size_t i = 0; i < h_keys_.size(); ++i)
            if (h_keys_[i] == b) return h_mask_[i * bs + l];
        return 0;
    }

    // write / write_with_spacing_offset (SparseGridGpu.hpp:3844-3903): every point whose mask
    // byte is not 0 at coord * spacing + offset * spacing, its properties and its mask byte, as a
    // binary legacy VTK poly-data file of vertices (the reference passes the same data to
    // openfpm_io's VTKWriter).  Reads the device data itself.
    bool write(const std::string& output) {
        const double one[3] = {1, 1, 1}, zero[3] = {0, 0, 0};
        return write_impl(output, one, zero);
    }
    bool write_with_spacing_offset(const std::string& output, Point<dim, double> spacing, Point<dim, double> offset) {
        return write_impl(output, spacing.x, offset.x);
    }

    // insertFlush<p>(coord) (SparseGridGpu.hpp:2779-2846): insert a point into the host copy
    // made by deviceToHost (its chunk is created with background values if missing), mark it
    // existing and return its value for the caller to fill; hostToDevice() uploads the copy
    template <unsigned p, typename CoordT>
    typename std::tuple_element<p, props>::type& insertFlush(const grid_key_dx<dim, CoordT>& c) {
        using T = typename std::tuple_element<p, props>::type;
        if (h_data_.size() != nprop || h_mask_.empty()) deviceToHost<>();  // no host copy yet
        int64_t bsz[3];
        for (int d = 0; d < 3; ++d) bsz[d] = ((int64_t)size_[d] + blockEdgeSize - 1) / blockEdgeSize;
        const int64_t b = detail::block_key(linearizer::zorder, bsz, c.get(0) / blockEdgeSize, c.get(1) / blockEdgeSize,
                                            c.get(2) / blockEdgeSize);
        const int64_t l = ((c.get(2) % blockEdgeSize) * blockEdgeSize + c.get(1) % blockEdgeSize) * blockEdgeSize +
                          c.get(0) % blockEdgeSize;
        auto it = std::lower_bound(h_keys_.begin(), h_keys_.end(), b);
        const int64_t pos = it - h_keys_.begin();
        if (it == h_keys_.end() || *it != b) {
            // a new chunk at pos: background values (the background chunk's, last), mask 0
            const int64_t n = (int64_t)h_keys_.size();
            h_keys_.insert(it, b);
            h_mask_.insert(h_mask_.begin() + pos * bs, bs, (uint8_t)0);
            for (unsigned q = 0; q < nprop; ++q) {
                const size_t es = h_data_[q].size() / ((n + 1) * bs);
                std::vector<unsigned char> bck(h_data_[q].end() - es * bs, h_data_[q].end());
                h_data_[q].insert(h_data_[q].begin() + pos * bs * es, bck.begin(), bck.end());
            }
        }
        h_mask_[pos * bs + l] = 1;
        return reinterpret_cast<T*>(h_data_[p].data())[pos * bs + l];
    }

    // hostToDevice(): upload the host copy (deviceToHost, insertFlush) as the grid's block map
    void hostToDevice() {
        const int64_t n = (int64_t)h_keys_.size();
        std::vector<const void*> ptrs(nprop);
        for (unsigned q = 0; q < nprop; ++q) ptrs[q] = h_data_[q].data();
        check(sgb_load_map(g_, n, h_keys_.data(), ptrs.data(), h_mask_.data(), nullptr), "hostToDevice");
    }

    // measureBlockOccupancy / measureBlockOccupancyMemory (SparseGridGpu.hpp:2485-2554): mean and
    // sample standard deviation over the chunks of the fraction of active (existing and not
    // padding) / existing points
    void measureBlockOccupancy(double& mean, double& deviation) const { occupancy(true, mean, deviation); }
    void measureBlockOccupancyMemory(double& mean, double& deviation) const { occupancy(false, mean, deviation); }

    // swap (SparseGridGpu.hpp:3403-3408)
    void swap(SparseGridGpu& o) {
        std::swap(g_, o.g_);
        for (int d = 0; d < 3; ++d) std::swap(size_[d], o.size_[d]);
        std::swap(nn_kind_, o.nn_kind_);
        for (int p = 0; p < 8; ++p) std::swap(bck_raw_[p], o.bck_raw_[p]);
        std::swap(npools_, o.npools_);
        std::swap(nslot_, o.nslot_);
        std::swap(pool_lin_, o.pool_lin_);
        for (int p = 0; p < 8; ++p) std::swap(pool_val_[p], o.pool_val_[p]);
        std::swap(pool_cnt_, o.pool_cnt_);
        h_keys_.swap(o.h_keys_);
        h_data_.swap(o.h_data_);
        h_mask_.swap(o.h_mask_);
        rem_sects_.swap(o.rem_sects_);
        pack_subs_.swap(o.pack_subs_);
    }

    // removeUnusedBuffers (SparseGridGpu.hpp:3739-3742)
    void removeUnusedBuffers() { check(sgb_release_scratch(g_), "removeUnusedBuffers"); }

    // private_get_neighborhood_array: the device neighbour table of the current NN type (int32,
    // -1 absent), valid until the next flush
    const int32_t* private_get_neighborhood_array() {
        sgb_view v;
        check(sgb_get_view(g_, nn_kind_, &v, nullptr), "private_get_neighborhood_array");
        return v.nn;
    }

    // remove(box): queue a section whose points removePoints deletes (SparseGridGpu.hpp:3528-3531)
    void remove(const Box<dim, int>& section_to_delete) { rem_sects_.push_back(section_to_delete); }

    // removePoints(ctx) (SparseGridGpu.hpp:3417-3489): the chunks stay, their points in the boxes go
    void removePoints(gpu::ofp_context_t&) {
        if (rem_sects_.empty()) return;
        std::vector<int64_t> b;
        for (const auto& bx : rem_sects_)
            for (int k = 0; k < 2; ++k)
                for (unsigned d = 0; d < dim; ++d) b.push_back(k == 0 ? bx.getLow(d) : bx.getHigh(d));
        check(sgb_remove_boxes(g_, (int64_t)rem_sects_.size(), b.data(), nullptr), "removePoints");
        rem_sects_.clear();
    }

    // The existing points in the order getIterator() visits them (chunk order, then offset order);
    // with start / stop only those inside that inclusive box (the sub-iterator).
    std::vector<grid_key_dx<dim, int>> existingPoints() const { return existing_points_impl(nullptr); }
    std::vector<grid_key_dx<dim, int>> existingPoints(const grid_key_dx<dim>& start, const grid_key_dx<dim>& stop) const {
        int64_t b[6];
        for (unsigned d = 0; d < 3; ++d) b[d] = start.get(d), b[3 + d] = stop.get(d);
        return existing_points_impl(b);
    }

    // ---- multi-resolution links (SparseGridGpu.hpp:2113-2262)
    void construct_link_dw(SparseGridGpu& grid_dw, const Box<dim, int>& db, Point<dim, int> p_dw,
                           gpu::ofp_context_t&) {
        int64_t b[6], sh[3];
        for (unsigned d = 0; d < 3; ++d) b[d] = db.getLow(d), b[3 + d] = db.getHigh(d), sh[d] = p_dw.get(d);
        check(sgb_construct_link_dw(g_, grid_dw.handle(), b, sh, nullptr), "construct_link_dw");
    }
    void construct_link_up(SparseGridGpu& grid_up, const Box<dim, int>& db, Point<dim, int> p_up,
                           gpu::ofp_context_t&) {
        int64_t b[6], sh[3];
        for (unsigned d = 0; d < 3; ++d) b[d] = db.getLow(d), b[3 + d] = db.getHigh(d), sh[d] = p_up.get(d);
        check(sgb_construct_link_up(g_, grid_up.handle(), b, sh, nullptr), "construct_link_up");
    }
    // getDownLinks / getDownLinksOffsets and the up pair, as one device view per direction
    sgb_links getDownLinks() const { return links(0); }
    sgb_links getUpLinks() const { return links(1); }

    // getIterator(start, stop): the sub-grid iterator of the inclusive box
    SparseGridGpu_iterator_sub<dim> getIterator(const grid_key_dx<dim>& start, const grid_key_dx<dim>& stop) const {
        return SparseGridGpu_iterator_sub<dim>{start, stop};
    }

    // ---- ghost-exchange packing (SparseGridGpu.hpp:3041-3370 pack side, 1420-1615 and 3665-3750 unpack)
    void packReset() { pack_subs_.clear(); }

    // packRequest(sub_it, req): queue the box; the size comes with packCalculate
    template <int... prp>
    void packRequest(const SparseGridGpu_iterator_sub<dim>& sub_it, size_t&) {
        pack_subs_.push_back(sub_it);
    }

    // packCalculate<prp...>(req, ctx): req += bytes to pack the queued boxes with prp...
    template <int... prp>
    void packCalculate(size_t& req, gpu::ofp_context_t&) {
        const int props[] = {prp..., 0};
        const std::vector<int64_t> b = pack_rows();
        std::vector<int64_t> sizes(pack_subs_.size());
        if (!sizes.empty())
            check(sgb_pack_request(g_, (int64_t)sizes.size(), b.data(), (int)sizeof...(prp), props, sizes.data(),
                                   nullptr),
                  "packCalculate");
        for (int64_t v : sizes) req += (size_t)v;
    }

    // pack<prp...>(mem, sub_it, sts): in the reference this only queues; the
    // bytes are written by packFinalize, here too
    template <int... prp>
    void pack(CudaMemory&, const SparseGridGpu_iterator_sub<dim>&, Pack_stat&) {}

    // packFinalize<prp...>(mem, sts): pack every queued box, back to back from sts's offset
    template <int... prp>
    void packFinalize(CudaMemory& mem, Pack_stat& sts, int = 0, bool = false) {
        const int props[] = {prp..., 0};
        const std::vector<int64_t> b = pack_rows();
        int64_t written = 0;
        check(sgb_pack(g_, (int64_t)pack_subs_.size(), b.data(), (int)sizeof...(prp), props,
                       (unsigned char*)mem.getDevicePointer() + sts.off, (int64_t)(mem.size() - sts.off), &written,
                       nullptr),
              "packFinalize");
        sts.off += (size_t)written;
    }

    // removeAddUnpackReset / unpack / removeAddUnpackFinalize: remove(box)
    // sections, unpack one packed box per call into the box of sub_it, then
    // apply the removals and merge the unpacked points
    void removeAddUnpackReset() { rem_sects_.clear(); }

    template <unsigned... prp>
    void unpack(CudaMemory& mem, const SparseGridGpu_iterator_sub<dim>& sub_it, Unpack_stat& ps,
                gpu::ofp_context_t&) {
        const int props[] = {(int)prp..., 0};
        int64_t start[3] = {0, 0, 0};
        for (unsigned d = 0; d < dim; ++d) start[d] = sub_it.getStart().get(d);
        int64_t used = 0;
        check(sgb_unpack(g_, (const unsigned char*)mem.getDevicePointer() + ps.off, (int64_t)(mem.size() - ps.off),
                         (int)sizeof...(prp), props, start, &used, nullptr),
              "unpack");
        ps.addOffset((size_t)used);
    }

    template <unsigned... prp>
    void removeAddUnpackFinalize(gpu::ofp_context_t& ctx, int) {
        removePoints(ctx);
        std::array<int, 8> ops{};
        const int listed[] = {(int)prp..., -1};
        for (int k = 0; k < (int)sizeof...(prp); ++k) ops[listed[k]] = SGB_OP_RIGHT;
        check(sgb_flush(g_, ops.data(), nullptr), "removeAddUnpackFinalize");
    }

    size_t countExistingElements() const {
        int64_t e = 0;
        check(sgb_count_existing(g_, &e, nullptr, nullptr), "countExistingElements");
        return (size_t)e;
    }
    size_t countBoundaryElements() const {
        int64_t p = 0;
        check(sgb_count_existing(g_, nullptr, &p, nullptr), "countBoundaryElements");
        return (size_t)p;
    }
    size_t size() const { return countExistingElements(); }

    // device buffers (private_get_index_array / private_get_data_array)
    const int64_t* private_get_index_array() const {
        const int64_t* p = nullptr;
        sgb_index_buffer(g_, &p);
        return p;
    }
    template <unsigned p>
    void* private_get_data_array() const {
        void* d = nullptr;
        sgb_data_buffer(g_, p, &d);
        return d;
    }
    int64_t nchunks() const {
        int64_t n = 0;
        sgb_nchunks(g_, &n);
        return n;
    }

   private:
    std::vector<Box<dim, int>> rem_sects_;
    std::vector<SparseGridGpu_iterator_sub<dim>> pack_subs_;

    template <typename T>
    static void put_be(std::ofstream& f, T v) {
        unsigned char b[sizeof(T)];
        std::memcpy(b, &v, sizeof(T));
        for (int i = (int)sizeof(T) - 1; i >= 0; --i) f.put((char)b[i]);
    }
    template <size_t... I>
    void write_props(std::ofstream& f, const std::vector<size_t>& sel, std::index_sequence<I...>) {
        (write_prop<I>(f, sel), ...);
    }
    template <size_t p>
    void write_prop(std::ofstream& f, const std::vector<size_t>& sel) {
        using T = typename std::tuple_element<p, props>::type;
        const char* vt = std::is_same<T, float>::value ? "float"
                         : std::is_same<T, double>::value ? "double"
                         : std::is_same<T, int>::value ? "int" : "unsigned_char";
        f << "SCALARS attr" << p << " " << vt << "\nLOOKUP_TABLE default\n";
        const T* d = reinterpret_cast<const T*>(h_data_[p].data());
        for (size_t i : sel) put_be(f, d[i]);
        f << "\n";
    }
    bool write_impl(const std::string& output, const double* sp, const double* of) {
        deviceToHost<>();
        int64_t bsz[3];
        for (int d = 0; d < 3; ++d) bsz[d] = ((int64_t)size_[d] + blockEdgeSize - 1) / blockEdgeSize;
        std::vector<size_t> sel;
        for (size_t i = 0; i < h_keys_.size() * bs; ++i)
            if (h_mask_[i] != 0) sel.push_back(i);
        std::ofstream f(output, std::ios::binary);
        if (!f) return false;
        f << "# vtk DataFile Version 3.0\nsparse_grid\nBINARY\nDATASET POLYDATA\nPOINTS " << sel.size() << " float\n";
        for (size_t i : sel) {
            int64_t bc[3];
            detail::block_coords(linearizer::zorder, bsz, h_keys_[i / bs], bc);
            const int64_t o = (int64_t)(i % bs);
            const int64_t c[3] = {bc[0] * blockEdgeSize + o % blockEdgeSize,
                                  bc[1] * blockEdgeSize + (o / blockEdgeSize) % blockEdgeSize,
                                  bc[2] * blockEdgeSize + o / (blockEdgeSize * blockEdgeSize)};
            for (int d = 0; d < 3; ++d) put_be(f, (float)((double)c[d] * sp[d] + of[d] * sp[d]));
        }
        f << "\nVERTICES " << sel.size() << " " << 2 * sel.size() << "\n";
        for (size_t k = 0; k < sel.size(); ++k) put_be(f, (int32_t)1), put_be(f, (int32_t)k);
        f << "\nPOINT_DATA " << sel.size() << "\n";
        write_props(f, sel, std::make_index_sequence<nprop>{});
        f << "SCALARS mask unsigned_char\nLOOKUP_TABLE default\n";
        for (size_t i : sel) f.put((char)h_mask_[i]);
        f << "\n";
        return (bool)f;
    }

    void occupancy(bool active_only, double& mean, double& deviation) const {
        int64_t n = 0;
        sgb_nchunks(g_, &n);
        std::vector<uint8_t> m((n + 1) * bs);
        check(sgb_download_map(g_, nullptr, nullptr, m.data(), nullptr), "measureBlockOccupancy");
        std::vector<double> occ((size_t)n);
        for (int64_t c = 0; c < n; ++c) {
            size_t k = 0;
            for (unsigned i = 0; i < bs; ++i) {
                const uint8_t b = m[c * bs + i];
                k += active_only ? ((b & 1) && !(b & 2)) : (b & 1) != 0;
            }
            occ[c] = (double)k / bs;
        }
        mean = 0;
        for (double x : occ) mean += x;
        mean /= (double)n;
        deviation = 0;
        for (double x : occ) deviation += (x - mean) * (x - mean);
        deviation = std::sqrt(deviation / (double)(n - 1));
    }

    sgb_links links(int up) const {
        sgb_links l{};
        check(sgb_get_links(g_, up, &l), "links");
        return l;
    }

    std::vector<int64_t> pack_rows() const {
        std::vector<int64_t> b;
        for (const auto& it : pack_subs_) {
            for (unsigned d = 0; d < 3; ++d) b.push_back(d < dim ? (int64_t)it.getStart().get(d) : 0);
            for (unsigned d = 0; d < 3; ++d) b.push_back(d < dim ? (int64_t)it.getStop().get(d) : 0);
        }
        return b;
    }

    std::vector<grid_key_dx<dim, int>> existing_points_impl(const int64_t* box) const {
        int64_t cnt = 0;
        check(sgb_existing_points(g_, box, nullptr, 0, &cnt, nullptr), "existingPoints");
        std::vector<grid_key_dx<dim, int>> out(cnt);
        if (cnt == 0) return out;
        int32_t* d = nullptr;
        if (cudaMalloc(&d, (size_t)cnt * 12) != cudaSuccess) throw sgb_error(SGB_ENOMEM, "existingPoints");
        int st = sgb_existing_points(g_, box, d, cnt, &cnt, nullptr);
        std::vector<int32_t> h((size_t)cnt * 3);
        if (st == SGB_OK) cudaMemcpy(h.data(), d, h.size() * 4, cudaMemcpyDeviceToHost);
        cudaFree(d);
        check(st, "existingPoints");
        for (int64_t i = 0; i < cnt; ++i)
            for (unsigned k = 0; k < dim; ++k) out[i].set_d(k, h[i * 3 + k]);
        return out;
    }

    void run_fixed(int kind, unsigned s, unsigned d, const float* prm, int nprm, const Box<dim, int>& box) {
        int src[2] = {(int)s, 0}, dst[2] = {(int)d, 0};
        int64_t b[6];
        for (unsigned i = 0; i < 3; ++i) b[i] = box.lo[i], b[3 + i] = box.hi[i];
        check(sgb_apply_stencil(g_, kind, src, dst, prm, nprm, b, nullptr), "applyStencils");
    }

    template <typename S>
    void apply_fixed(const Box<dim, int>& box, float dt) {
        static_assert(S::kind == SGB_HEAT7, "HeatStencil takes dt");
        run_fixed(S::kind, S::src, S::dst, &dt, 1, box);
    }
    template <typename S>
    void apply_fixed(const Box<dim, int>& box, double dt) {
        apply_fixed<S>(box, (float)dt);
    }
    template <typename S>
    void apply_fixed(const Box<dim, int>& box, const conv_coeff& cc) {
        static_assert(S::kind == SGB_BOX27 || S::kind == SGB_BOX27_NS, "Conv3x3x3 takes conv_coeff");
        float c[27];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                for (int k = 0; k < 3; ++k) c[i * 9 + j * 3 + k] = cc.coeff[i][j][k];
        run_fixed(S::kind, S::src, S::dst, c, 27, box);
    }

    template <typename S, typename... Args>
    void apply_user(const Box<dim, int>& box, StencilMode mode, Args... args) {
        using NN = typename S::stencil_type;
        device_grid_type k{};
        check(sgb_get_view(g_, NN::kind, &k.v, nullptr), "applyStencils");
        if (k.v.n == 0) return;
        for (unsigned p = 0; p < nprop && p < 8; ++p) k.bck[p] = bck_raw_[p];
        if (mode == STENCIL_MODE_INPLACE_NO_SHARED) {
            const uint32_t* ids = nullptr;
            int64_t nids = 0;
            check(sgb_existing_point_list(g_, &ids, &nids, nullptr), "applyStencils (existing points)");
            if (nids > 0)
                detail::apply_stencil_noshared<S><<<(unsigned)((nids + 127) / 128), 128>>>(box, k, ids, nids, args...);
        } else {
            detail::apply_stencil_inplace<S><<<(unsigned)k.v.n, bs>>>(box, k, args...);
        }
        check(cudaGetLastError() == cudaSuccess ? SGB_OK : SGB_ECUDA, "applyStencils launch");
        // a functor may store into any point of any property: the library refills the backgrounds
        // of points that do not exist before its own kernels rely on them
        for (unsigned p = 0; p < nprop; ++p) {
            void* d = nullptr;
            check(sgb_data_buffer(g_, (int)p, &d), "applyStencils");
        }
    }

    template <int NP, int MODE, unsigned s1, unsigned s2, unsigned d1, unsigned d2, unsigned s3 = s1, unsigned d3 = d1,
              typename F>
    void launch_conv(grid_key_dx<3> start, grid_key_dx<3> stop, F f) {
        using T0 = typename std::tuple_element<s1, props>::type;
        using T1 = typename std::tuple_element<s2, props>::type;
        using T2 = typename std::tuple_element<s3, props>::type;
        using U0 = typename std::tuple_element<d1, props>::type;
        using U1 = typename std::tuple_element<d2, props>::type;
        using U2 = typename std::tuple_element<d3, props>::type;
        sgb_view v;
        check(sgb_get_view(g_, nn_kind_, &v, nullptr), "conv");
        if (v.n == 0) return;
        Box<3, int> box;
        for (int i = 0; i < 3; ++i) box.lo[i] = (int)start.get(i), box.hi[i] = (int)stop.get(i);
        T0 b0;
        T1 b1;
        T2 b2;
        std::memcpy(&b0, &bck_raw_[s1], sizeof(T0));
        std::memcpy(&b1, &bck_raw_[s2], sizeof(T1));
        std::memcpy(&b2, &bck_raw_[s3], sizeof(T2));
        // every existing point lies in [0, size): a box that holds all of it needs no per-chunk test
        int full_box = 1;
        for (int i = 0; i < 3; ++i) full_box &= box.lo[i] <= 0 && (int64_t)box.hi[i] >= (int64_t)size_[i] - 1;
        auto kern = detail::conv_kernel<blockEdgeSize, NP, MODE, T0, T1, T2, U0, U1, U2, F>;
        int dev = 0, sms = 148, per_sm = 1;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, detail::kConvThreads, 0);
        // one wave of resident CTAs, each walking its share of the chunks
        const int64_t cap = (int64_t)sms * (per_sm > 0 ? per_sm : 1);
        const unsigned blocks = (unsigned)(v.n < cap ? v.n : cap);
        kern<<<blocks, detail::kConvThreads>>>(v, (int)s1, (int)s2, (int)s3, (int)d1, (int)d2, (int)d3, box, full_box,
                                               b0, b1, b2, f);
        check(cudaGetLastError() == cudaSuccess ? SGB_OK : SGB_ECUDA, "conv launch");
        if (MODE == 0) {
            // storeBlock semantics put source values into the destination's
            // non-existing points: have the library restore its backgrounds
            void* d = nullptr;
            check(sgb_data_buffer(g_, (int)d1, &d), "conv");
        }
    }
};

// SparseGridGpu_z (src/SparseGridGpu/SparseGridGpu.hpp:3948-3960): chunk ids by Morton code
template <unsigned dim, typename AggregateT, unsigned blockEdgeSize = 8, unsigned threadBlockSize = 512,
          typename indexT = long, template <typename> class layout_base = memory_traits_inte,
          typename linearizer = grid_zmb<dim, blockEdgeSize, indexT>>
using SparseGridGpu_z = SparseGridGpu<dim, AggregateT, blockEdgeSize, threadBlockSize, indexT, layout_base, linearizer>;

}  // namespace openfpm_b200
