// Drop-in test of include/openfpm_b200/SparseGridGpu.hpp: user code written
// against the reference's SparseGridGpu interface (device insert pools,
// flush<smax_<0>>, tagBoundaries, applyStencils<HeatStencil / Conv3x3x3>,
// conv / conv_cross / conv2 / conv2_b with __device__ lambdas, toKernel().get,
// deviceToHost + get) compiled with nvcc and run on the GPU.  Follows the
// reference's tests src/SparseGridGpu/tests/SparseGridGpu_tests.cu (insert
// kernels 15-60, conv_cross / conv / conv2 at 499-720, Conv3x3x3 at 887-952).
//
// Each check compares two routes that must agree bit for bit: the header's
// device-side paths against the C ABI calls that the Python parity tests pin
// to the CPU oracle.  Prints "ok <name>" per check; exit status 0 when all
// pass.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iterator>
#include <string>
#include <unistd.h>
#include <vector>

#include "openfpm_b200/SparseGridGpu.hpp"

using namespace openfpm_b200;

static int g_fail = 0;
#define CHECK(cond, name)                                      \
    do {                                                       \
        if (cond) std::printf("ok %s\n", name);                \
        else {                                                 \
            std::printf("FAIL %s (line %d)\n", name, __LINE__); \
            ++g_fail;                                          \
        }                                                      \
    } while (0)

constexpr int N = 64;  // domain edge
typedef aggregate<float, float, float, float, float, float> Agg6;
typedef SparseGridGpu<3, Agg6, 8> Grid6;

__host__ __device__ inline bool in_shape(int x, int y, int z) {
    const int dx = x - 30, dy = y - 33, dz = z - 29;
    const int r2 = dx * dx + dy * dy + dz * dz;
    return r2 <= 22 * 22 && r2 >= 6 * 6;  // a thick shell: chunks with holes and missing neighbours
}
__host__ __device__ inline float val_a(int x, int y, int z) { return 0.01f * (float)((x * 7 + y * 13 + z * 29) % 97); }
__host__ __device__ inline float val_b(int x, int y, int z) { return 0.02f * (float)((x * 11 + y * 5 + z * 3) % 89); }

// insert<p> twice per point (the larger value must win under smax_), one
// CTA per 8^3 box as the reference's insertConstantValue kernels
template <unsigned p, typename Ker>
__global__ void insert_shape(Ker g) {
    g.init();
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y,
              z = blockIdx.z * blockDim.z + threadIdx.z;
    if (in_shape(x, y, z)) {
        grid_key_dx<3, int> c({x, y, z});
        g.template insert<p>(c) = p == 0 ? val_a(x, y, z) : val_b(x, y, z);
        g.template insert<p>(c) = (p == 0 ? val_a(x, y, z) : val_b(x, y, z)) * 0.5f;
    }
    g.flush_block_insert();
}

template <typename Ker>
__global__ void read_all(Ker g, float* out) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y,
              z = blockIdx.z * blockDim.z + threadIdx.z;
    grid_key_dx<3, int> c({x, y, z});
    out[x + N * (y + N * z)] = g.template get<0>(c);
}

struct HostMap {
    std::vector<int64_t> keys;
    std::vector<std::vector<float>> data;
    std::vector<uint8_t> mask;
};

static HostMap download(sgb_grid* g, int nprop) {
    HostMap m;
    int64_t n = 0;
    sgb_nchunks(g, &n);
    m.keys.resize(n);
    m.mask.resize((n + 1) * 512);
    m.data.assign(nprop, std::vector<float>((n + 1) * 512));
    std::vector<void*> ptrs(nprop);
    for (int p = 0; p < nprop; ++p) ptrs[p] = m.data[p].data();
    check(sgb_download_map(g, m.keys.data(), ptrs.data(), m.mask.data(), nullptr), "download");
    return m;
}

// bitwise equality of property pa of a and pb of b over points selected by `sel(mask byte)`
template <typename Sel>
static bool same(const HostMap& a, int pa, const HostMap& b, int pb, Sel sel) {
    if (a.keys != b.keys) return false;
    const size_t n = a.keys.size() * 512;
    for (size_t i = 0; i < n; ++i)
        if (sel(a.mask[i]) && std::memcmp(&a.data[pa][i], &b.data[pb][i], 4) != 0) return false;
    return true;
}

static bool existing(uint8_t m) { return (m & 1) != 0; }
static bool active(uint8_t m) { return (m & 3) == 1; }

// The staged C ABI route: the same points in a plain insert list
static void insert_via_abi(sgb_grid* g) {
    std::vector<int32_t> coords;
    std::vector<float> va;
    for (int z = 0; z < N; ++z)
        for (int y = 0; y < N; ++y)
            for (int x = 0; x < N; ++x)
                if (in_shape(x, y, z)) {
                    for (int rep = 0; rep < 2; ++rep) {
                        coords.insert(coords.end(), {x, y, z});
                        va.push_back(rep == 0 ? val_a(x, y, z) : val_a(x, y, z) * 0.5f);
                    }
                }
    const int64_t n = (int64_t)va.size();
    int32_t* dc;
    float* dv;
    cudaMalloc(&dc, coords.size() * 4);
    cudaMalloc(&dv, va.size() * 4);
    cudaMemcpy(dc, coords.data(), coords.size() * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(dv, va.data(), va.size() * 4, cudaMemcpyHostToDevice);
    const void* vals[6] = {dv, nullptr, nullptr, nullptr, nullptr, nullptr};
    check(sgb_insert(g, n, dc, vals, nullptr), "sgb_insert");
    int ops[6] = {SGB_OP_MAX, SGB_OP_NONE, SGB_OP_NONE, SGB_OP_NONE, SGB_OP_NONE, SGB_OP_NONE};
    check(sgb_flush(g, ops, nullptr), "sgb_flush");
    cudaDeviceSynchronize();
    cudaFree(dc);
    cudaFree(dv);
}

// remove<>(coord) from a device kernel: the points of the shape with an even coordinate sum
// (SparseGridGpu_testKernels.cuh:318-357 removeSphere3D_even_radiusV)
template <typename Ker>
__global__ void remove_even(Ker g) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y,
              z = blockIdx.z * blockDim.z + threadIdx.z;
    if (in_shape(x, y, z) && (x + y + z) % 2 == 0) g.remove(grid_key_dx<3, int>({x, y, z}));
}

// insertBlock as the reference's insertSphere3D (SparseGridGpu_testKernels.cuh:144-200): one CTA
// per 8^3 block of a box starting at `start`, every thread one point; blocks holding a point of the
// shell r2 <= r < r1 around the box centre take a chunk slot and write their points
template <unsigned p, typename Ker>
__global__ void insert_sphere_blocks(Ker sg, grid_key_dx<3, int> start, float r1, float r2, float value) {
    constexpr unsigned pMask = Ker::pMask;
    grid_key_dx<3, long> blk({(long)(blockIdx.x + start.get(0) / 8), (long)(blockIdx.y + start.get(1) / 8),
                              (long)(blockIdx.z + start.get(2) / 8)});
    const unsigned offset = threadIdx.x;
    __shared__ bool is_block_empty;
    if (threadIdx.x == 0) is_block_empty = true;
    sg.init();
    const auto blockId = sg.getBlockLinId(blk);
    const grid_key_dx<3, long> keyg = sg.getGlobalCoord(blk, offset);
    const long x = keyg.get(0) - (start.get(0) + gridDim.x / 2 * 8);
    const long y = keyg.get(1) - (start.get(1) + gridDim.y / 2 * 8);
    const long z = keyg.get(2) - (start.get(2) + gridDim.z / 2 * 8);
    const float radius = sqrtf((float)(x * x + y * y + z * z));
    const bool is_active = radius < r1 && radius >= r2;
    if (is_active) is_block_empty = false;
    __syncthreads();
    if (!is_block_empty) {
        auto ec = sg.insertBlock(blockId);
        if (is_active) {
            ec.template get<p>()[offset] = value + (float)(keyg.get(0) + 3 * keyg.get(1));
            BlockMapGpu_ker<>::setExist(ec.template get<pMask>()[offset]);
        }
    }
    __syncthreads();
    sg.flush_block_insert();
}

// insertBlock with two properties per point as insertConstantValue2 (SparseGridGpu_tests.cu:14-43)
template <unsigned p1, unsigned p2, typename Ker>
__global__ void insert_constant_blocks(Ker sg, float value) {
    constexpr unsigned pMask = Ker::pMask;
    sg.init();
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y,
              z = blockIdx.z * blockDim.z + threadIdx.z;
    grid_key_dx<3, int> coord({x, y, z});
    const int64_t pos = sg.getLinId(coord);
    const int64_t dataBlockId = pos / 512;
    const unsigned offset = (unsigned)(pos % 512);
    auto ec = sg.insertBlock(dataBlockId);  // thread (0, 0, 0) takes the CTA's slot
    ec.template get<p1>()[offset] = value;
    ec.template get<p2>()[offset] = value;
    BlockMapGpu_ker<>::setExist(ec.template get<pMask>()[offset]);
    __syncthreads();
    sg.flush_block_insert();
}

// ---- user stencil functors with the reference's contract (applyStencils<S> with any S)
// BoundaryStencilSetXRescaled (SparseGridGpu_testKernels.cuh:36-80), in 3-D
template <unsigned dim, unsigned p_src, unsigned p_dst, typename ScalarT = float>
struct UserBoundarySetXRescaled {
    typedef NNStar<dim> stencil_type;
    static constexpr unsigned supportRadius = 1;
    template <typename SparseGridT, typename DataBlockWrapperT>
    static inline __device__ void stencil(SparseGridT& sparseGrid, const unsigned dataBlockId,
                                          openfpm::sparse_index<unsigned> dataBlockIdPos, unsigned offset,
                                          grid_key_dx<dim, int>& pointCoord, DataBlockWrapperT& dataBlockLoad,
                                          DataBlockWrapperT& dataBlockStore, unsigned char curMask, ScalarT minX,
                                          ScalarT maxX, ScalarT minValue, ScalarT maxValue) {
        if (curMask == mask_sparse::EXIST_AND_PADDING) {
            const ScalarT x = pointCoord.get(0);
            auto value = maxValue * (x - minX) / (maxX - minX - 1);
            if (x < minX) value = minValue;
            else if (x > maxX) value = maxValue;
            dataBlockStore.template get<p_dst>()[offset] = value;
        }
    }
};

// HeatStencil (SparseGridGpu_util_test.cuh:201-290) as user code: loadGhostBlock, enlarged-block
// indexing, storeBlock
template <unsigned dim, unsigned p_src, unsigned p_dst>
struct UserHeatStencil {
    typedef NNStar<dim> stencil_type;
    static constexpr unsigned supportRadius = 1;
    template <typename SparseGridT, typename DataBlockWrapperT>
    static inline __device__ void stencil(SparseGridT& sparseGrid, const unsigned dataBlockId,
                                          const openfpm::sparse_index<unsigned> dataBlockIdPos, const unsigned offset,
                                          const grid_key_dx<dim, int>& pointCoord,
                                          const DataBlockWrapperT& dataBlockLoad, DataBlockWrapperT& dataBlockStore,
                                          unsigned char curMask, float dt) {
        typedef typename SparseGridT::AggregateBlockType AggregateT;
        typedef ScalarTypeOf<AggregateT, p_src> ScalarT;
        constexpr unsigned enlargedBlockSize = IntPow<SparseGridT::getBlockEdgeSize() + 2 * supportRadius, dim>::value;
        __shared__ ScalarT enlargedBlock[enlargedBlockSize];
        sparseGrid.template loadGhostBlock<p_src>(dataBlockLoad, dataBlockIdPos, enlargedBlock);
        __syncthreads();
        decltype(sparseGrid.getLinIdInEnlargedBlock(0)) linId = 0;
        ScalarT res = 0;
        if ((curMask & mask_sparse::EXIST) && !(curMask & mask_sparse::PADDING)) {
            const auto coord = sparseGrid.getCoordInEnlargedBlock(offset);
            linId = sparseGrid.getLinIdInEnlargedBlock(offset);
            ScalarT cur = enlargedBlock[linId];
            ScalarT laplacian = -2.0 * dim * cur;
            for (int d = 0; d < dim; ++d) {
                auto nPlusId = sparseGrid.getNeighbourLinIdInEnlargedBlock(coord, d, 1);
                auto nMinusId = sparseGrid.getNeighbourLinIdInEnlargedBlock(coord, d, -1);
                ScalarT neighbourPlus = enlargedBlock[nPlusId];
                ScalarT neighbourMinus = enlargedBlock[nMinusId];
                laplacian += neighbourMinus + neighbourPlus;
            }
            res = cur + dt * laplacian;
        }
        __syncthreads();
        if ((curMask & mask_sparse::EXIST) && !(curMask & mask_sparse::PADDING)) enlargedBlock[linId] = res;
        __syncthreads();
        sparseGrid.template storeBlock<p_dst>(dataBlockStore, enlargedBlock);
    }
};

// Conv3x3x3 (SparseGridGpu_tests.cu:887-952) as user code over an NNFull tile
template <unsigned dim, unsigned p_src, unsigned p_dst>
struct UserConv3x3x3 {
    typedef NNFull<dim> stencil_type;
    static constexpr unsigned supportRadius = 1;
    template <typename SparseGridT, typename DataBlockWrapperT>
    static inline __device__ void stencil(SparseGridT& sparseGrid, const unsigned dataBlockId,
                                          openfpm::sparse_index<unsigned> dataBlockIdPos, unsigned offset,
                                          grid_key_dx<dim, int>& pointCoord, DataBlockWrapperT& dataBlockLoad,
                                          DataBlockWrapperT& dataBlockStore, unsigned char curMask, conv_coeff& cc) {
        typedef typename SparseGridT::AggregateBlockType AggregateT;
        typedef ScalarTypeOf<AggregateT, p_src> ScalarT;
        constexpr unsigned enlargedBlockSize = IntPow<SparseGridT::getBlockEdgeSize() + 2 * supportRadius, dim>::value;
        __shared__ ScalarT enlargedBlock[enlargedBlockSize];
        sparseGrid.template loadGhostBlock<p_src>(dataBlockLoad, dataBlockIdPos, enlargedBlock);
        __syncthreads();
        if ((curMask & mask_sparse::EXIST) && !(curMask & mask_sparse::PADDING)) {
            const auto coord = sparseGrid.getCoordInEnlargedBlock(offset);
            ScalarT tot = 0.0;
            for (int i = 0; i < dim; ++i)
                for (int j = 0; j < dim; ++j)
                    for (int k = 0; k < dim; ++k) {
                        grid_key_dx<dim, int> key;
                        key.set_d(0, i - 1);
                        key.set_d(1, j - 1);
                        key.set_d(2, k - 1);
                        auto nPlusId = sparseGrid.getNeighbourLinIdInEnlargedBlock(coord, key);
                        tot += enlargedBlock[nPlusId] * cc.coeff[i][j][k];
                    }
            dataBlockStore.template get<p_dst>()[offset] = tot;
        }
    }
};

// Conv3x3x3_noshared (SparseGridGpu_tests.cu:955-1010) as user code: getNNPoint + get
template <unsigned dim, unsigned p_src, unsigned p_dst>
struct UserConv3x3x3NoShared {
    typedef NNFull<dim> stencil_type;
    static constexpr unsigned supportRadius = 1;
    template <typename SparseGridT, typename DataBlockWrapperT>
    static inline __device__ void stencil(SparseGridT& sparseGrid, const unsigned dataBlockId,
                                          openfpm::sparse_index<unsigned> dataBlockIdPos, unsigned offset,
                                          grid_key_dx<dim, int>& pointCoord, DataBlockWrapperT& dataBlockLoad,
                                          DataBlockWrapperT& dataBlockStore, unsigned char curMask, conv_coeff& cc) {
        typedef typename SparseGridT::AggregateBlockType AggregateT;
        typedef ScalarTypeOf<AggregateT, p_src> ScalarT;
        if ((curMask & mask_sparse::EXIST) && !(curMask & mask_sparse::PADDING)) {
            ScalarT tot = 0.0;
            for (int i = 0; i < dim; ++i)
                for (int j = 0; j < dim; ++j)
                    for (int k = 0; k < dim; ++k) {
                        grid_key_dx<dim, int> key;
                        key.set_d(0, k - 1);
                        key.set_d(1, j - 1);
                        key.set_d(2, i - 1);
                        block_offset<int> pos = sparseGrid.template getNNPoint<stencil_type>(dataBlockIdPos, offset, key);
                        tot += sparseGrid.template get<p_src>(pos) * cc.coeff[i][j][k];
                    }
            dataBlockStore.template get<p_dst>()[offset] = tot;
        }
    }
};

// loadGhostBlock with a mask tile: writes into p_dst, at every existing point, the number of its 26
// halo neighbours whose mask byte is set (exercises the NNStar edge / corner rule when run on NNStar)
template <unsigned p_src, unsigned p_dst>
struct UserCountTile {
    typedef NNStar<3> stencil_type;
    template <typename SparseGridT, typename DataBlockWrapperT>
    static inline __device__ void stencil(SparseGridT& sparseGrid, const unsigned, openfpm::sparse_index<unsigned> pos,
                                          unsigned offset, grid_key_dx<3, int>&, DataBlockWrapperT& load,
                                          DataBlockWrapperT& store, unsigned char curMask) {
        __shared__ float tile[1000];
        __shared__ unsigned char mtile[1000];
        sparseGrid.template loadGhostBlock<p_src>(load, pos, tile, mtile);
        __syncthreads();
        if (curMask & 1) {
            const auto c = sparseGrid.getCoordInEnlargedBlock(offset);
            float acc = 0;
            for (int dz = -1; dz <= 1; ++dz)
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dx = -1; dx <= 1; ++dx) {
                        grid_key_dx<3, int> o;
                        o.set_d(0, dx);
                        o.set_d(1, dy);
                        o.set_d(2, dz);
                        const unsigned id = sparseGrid.getNeighbourLinIdInEnlargedBlock(c, o);
                        acc += (mtile[id] & 1) ? tile[id] : 0.0f;
                    }
            store.template get<p_dst>()[offset] = acc;
        }
    }
};

int main() {
    const size_t sz[3] = {N, N, N};
    gpu::ofp_context_t ctx;

    // ---------------------------------------------------------------- insert + flush
    Grid6 grid(sz);
    grid.setBackgroundValue<0>(0.0f);
    grid.setGPUInsertBuffer(dim3(N / 8, N / 8, N / 8), dim3(1024, 1, 1));
    insert_shape<0><<<dim3(N / 8, N / 8, N / 8), dim3(8, 8, 8)>>>(grid.toKernel());
    grid.flush<smax_<0>>(ctx, FLUSH_ON_DEVICE);

    Grid6 ref(sz);
    ref.setBackgroundValue<0>(0.0f);
    insert_via_abi(ref.handle());

    HostMap A = download(grid.handle(), 6), B = download(ref.handle(), 6);
    CHECK(A.keys == B.keys && A.mask == B.mask && same(A, 0, B, 0, existing), "insert_pools_flush_smax");
    size_t npts = 0;
    for (int z = 0; z < N; ++z)
        for (int y = 0; y < N; ++y)
            for (int x = 0; x < N; ++x) npts += in_shape(x, y, z);
    CHECK(grid.countExistingElements() == npts, "countExistingElements");

    // ---------------------------------------------------------------- device get / host get
    float* dout;
    cudaMalloc(&dout, (size_t)N * N * N * 4);
    read_all<<<dim3(N / 8, N / 8, N / 8), dim3(8, 8, 8)>>>(grid.toKernel(), dout);
    std::vector<float> hout((size_t)N * N * N);
    cudaMemcpy(hout.data(), dout, hout.size() * 4, cudaMemcpyDeviceToHost);
    cudaFree(dout);
    grid.deviceToHost<0>();
    bool get_ok = true;
    for (int z = 0; z < N && get_ok; ++z)
        for (int y = 0; y < N; ++y)
            for (int x = 0; x < N; ++x) {
                const float h = grid.get<0>(grid_key_dx<3, int>({x, y, z}));
                const float expect = in_shape(x, y, z) ? val_a(x, y, z) : 0.0f;
                if (h != hout[x + N * (y + N * z)] || h != expect) get_ok = false;
            }
    CHECK(get_ok, "toKernel_get_matches_host_get");

    grid.tagBoundaries<NNStar<3>>(ctx);
    ref.tagBoundaries<NNStar<3>>(ctx);
    CHECK(grid.countBoundaryElements() == ref.countBoundaryElements() && grid.countBoundaryElements() > 0,
          "tagBoundaries");

    // second field for the two-field stencils: prop 1 = val_b on the same points
    {
        HostMap m = download(grid.handle(), 6);
        const int64_t n = (int64_t)m.keys.size();
        for (int64_t c = 0; c < n; ++c) {
            const int64_t k = m.keys[c];
            const int bx = (int)(k % (N / 8)), by = (int)((k / (N / 8)) % (N / 8)), bz = (int)(k / (N / 8 * N / 8));
            for (int o = 0; o < 512; ++o)
                m.data[1][c * 512 + o] = val_b(bx * 8 + o % 8, by * 8 + (o / 8) % 8, bz * 8 + o / 64);
        }
        std::vector<const void*> ptrs(6);
        for (int p = 0; p < 6; ++p) ptrs[p] = m.data[p].data();
        check(sgb_load_map(grid.handle(), n, m.keys.data(), ptrs.data(), m.mask.data(), nullptr), "load_map");
    }
    const Box<3, int> all = grid.getBox();
    const grid_key_dx<3> lo({0, 0, 0}), hi({N - 1, N - 1, N - 1});

    // ---------------------------------------------------------------- HeatStencil vs conv_cross
    grid.applyStencils<HeatStencil<3, 0, 2>>(all, STENCIL_MODE_INPLACE, 0.1f);
    // (HeatStencil's rounding as nvcc compiles the reference's functor: -6 u fused with the x pair)
    grid.conv_cross<0, 3, 1>(lo, hi, [] __device__(float& u, cross_stencil<3, float>& cs) {
        float lap = __fmaf_rn(-6.0f, u, __fadd_rn(cs.xm[0], cs.xp[0]));
        lap = __fadd_rn(lap, __fadd_rn(cs.xm[1], cs.xp[1]));
        lap = __fadd_rn(lap, __fadd_rn(cs.xm[2], cs.xp[2]));
        return __fmaf_rn(0.1f, lap, u);
    });
    cudaDeviceSynchronize();
    HostMap H = download(grid.handle(), 6);
    CHECK(same(H, 2, H, 3, existing), "heat_vs_conv_cross");

    // ---------------------------------------------------------------- conv (cp_block) vs HeatStencil, in a box
    Box<3, int> box;
    for (int d = 0; d < 3; ++d) box.setLow(d, 11 + d), box.setHigh(d, 47 - 2 * d);
    grid.applyStencils<HeatStencil<3, 0, 2>>(box, STENCIL_MODE_INPLACE, 0.05f);
    grid.conv<0, 3, 1>(grid_key_dx<3>({11, 12, 13}), grid_key_dx<3>({47, 45, 43}),
                       [] __device__(cp_block<float, 8>& u, int i, int j, int k) {
                           const float c = u(i, j, k);
                           float lap = __fmaf_rn(-6.0f, c, __fadd_rn(u(i - 1, j, k), u(i + 1, j, k)));
                           lap = __fadd_rn(lap, __fadd_rn(u(i, j - 1, k), u(i, j + 1, k)));
                           lap = __fadd_rn(lap, __fadd_rn(u(i, j, k - 1), u(i, j, k + 1)));
                           return __fmaf_rn(0.05f, lap, c);
                       });
    cudaDeviceSynchronize();
    HostMap C = download(grid.handle(), 6);
    {
        // active points inside the box: both wrote the update
        bool ok = C.keys == H.keys;
        const int64_t n = (int64_t)C.keys.size();
        int64_t cnt = 0;
        for (int64_t c = 0; c < n && ok; ++c) {
            const int64_t k = C.keys[c];
            const int bx = (int)(k % (N / 8)), by = (int)((k / (N / 8)) % (N / 8)), bz = (int)(k / (N / 8 * N / 8));
            for (int o = 0; o < 512; ++o) {
                const int x = bx * 8 + o % 8, y = by * 8 + (o / 8) % 8, z = bz * 8 + o / 64;
                const bool inb = x >= 11 && x <= 47 && y >= 12 && y <= 45 && z >= 13 && z <= 43;
                const size_t i = c * 512 + o;
                if (active(C.mask[i]) && inb) {
                    ++cnt;
                    if (std::memcmp(&C.data[2][i], &C.data[3][i], 4) != 0) ok = false;
                }
            }
        }
        CHECK(ok && cnt > 0, "heat_box_vs_conv_box");
    }

    // ---------------------------------------------------------------- Gray-Scott: GS7 vs conv2 and conv2_b
    const float Du = 0.16f, Dv = 0.08f, F = 0.035f, K = 0.065f, dt = 1.0f;
    {
        int src[2] = {0, 1}, dst[2] = {2, 3};
        float prm[5] = {Du, Dv, F, K, dt};
        check(sgb_apply_stencil(grid.handle(), SGB_GS7, src, dst, prm, 5, nullptr, nullptr), "gs7");
    }
    auto gs = [=] __device__(float& uo, float& vo, cp_block<float, 8>& u, cp_block<float, 8>& v, int i, int j,
                             int k) {
        auto lap = [](cp_block<float, 8>& f, int i, int j, int k) {
            float l = __fmul_rn(-6.0f, f(i, j, k));
            l = __fadd_rn(l, __fadd_rn(f(i - 1, j, k), f(i + 1, j, k)));
            l = __fadd_rn(l, __fadd_rn(f(i, j - 1, k), f(i, j + 1, k)));
            return __fadd_rn(l, __fadd_rn(f(i, j, k - 1), f(i, j, k + 1)));
        };
        const float uc = u(i, j, k), vc = v(i, j, k);
        const float uvv = __fmul_rn(__fmul_rn(uc, vc), vc);
        float du = __fmaf_rn(Du, lap(u, i, j, k), -uvv);
        du = __fmaf_rn(F, __fsub_rn(1.0f, uc), du);
        float dv = __fmaf_rn(Dv, lap(v, i, j, k), uvv);
        dv = __fmaf_rn(-(F + K), vc, dv);
        uo = __fmaf_rn(dt, du, uc);
        vo = __fmaf_rn(dt, dv, vc);
    };
    grid.conv2<0, 1, 4, 5, 1>(lo, hi, gs);
    cudaDeviceSynchronize();
    HostMap G = download(grid.handle(), 6);
    CHECK(same(G, 2, G, 4, active) && same(G, 3, G, 5, active), "gs7_vs_conv2");
    grid.conv2_b<0, 1, 4, 5, 1>(lo, hi,
                               [=] __device__(float& uo, float& vo, cp_block<float, 8>& u, cp_block<float, 8>& v,
                                              data_block<8>& blk, int offset, int i, int j, int k) {
                                   // the centre value through the chunk handle, as conv2_b users read it
                                   const float uc = blk.get<0>()[offset];
                                   float uu, vv;
                                   gs(uu, vv, u, v, i, j, k);
                                   uo = uc == u(i, j, k) ? uu : -1.0f;
                                   vo = vv;
                               });
    cudaDeviceSynchronize();
    HostMap G2 = download(grid.handle(), 6);
    CHECK(same(G2, 2, G2, 4, active) && same(G2, 3, G2, 5, active), "gs7_vs_conv2_b");

    // conv3_b (SparseGridGpu.hpp:2646-2663): the Gray-Scott pair on u, v plus a third field read with
    // its halo; the pair must equal GS7, the third result a conv of the same expression
    auto halo3 = [] __device__(cp_block<float, 8>& w, int i, int j, int k) {
        return __fadd_rn(__fadd_rn(w(i - 1, j, k), w(i, j + 1, k)), __fadd_rn(w(i, j, k - 1), w(i, j, k)));
    };
    grid.conv3_b<0, 1, 2, 4, 5, 3, 1>(lo, hi,
                                     [=] __device__(float& uo, float& vo, float& wo, cp_block<float, 8>& u,
                                                    cp_block<float, 8>& v, cp_block<float, 8>& w, data_block<8>&,
                                                    int, int i, int j, int k) {
                                         gs(uo, vo, u, v, i, j, k);
                                         wo = halo3(w, i, j, k);
                                     });
    cudaDeviceSynchronize();
    HostMap G3 = download(grid.handle(), 6);
    grid.conv<2, 3, 1>(lo, hi, [=] __device__(cp_block<float, 8>& w, int i, int j, int k) { return halo3(w, i, j, k); });
    cudaDeviceSynchronize();
    HostMap G4 = download(grid.handle(), 6);
    CHECK(same(G3, 4, G2, 2, active) && same(G3, 5, G2, 3, active) && same(G3, 3, G4, 3, active),
          "conv3_b_vs_gs7_and_conv");

    // ---------------------------------------------------------------- Conv3x3x3 vs conv over NNFull
    conv_coeff cc;
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b)
            for (int d = 0; d < 3; ++d) cc.coeff[a][b][d] = 0.01f * (float)(1 + a + 3 * b + 9 * d);
    grid.applyStencils<Conv3x3x3<3, 0, 2>>(all, STENCIL_MODE_INPLACE, cc);
    grid.setNNType<NNFull<3>>();
    grid.conv<0, 3, 1>(lo, hi, [cc] __device__(cp_block<float, 8>& u, int i, int j, int k) {
        float tot = 0.0f;
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b)
                for (int d = 0; d < 3; ++d) tot = __fmaf_rn(u(i + a - 1, j + b - 1, k + d - 1), cc.coeff[a][b][d], tot);
        return tot;
    });
    cudaDeviceSynchronize();
    HostMap Q = download(grid.handle(), 6);
    CHECK(same(Q, 2, Q, 3, active), "conv3x3x3_vs_conv_nnfull");

    // ------------------------------------------- Conv3x3x3_noshared (point list) vs conv over NNFull
    // SparseGridGpu_tests.cu:1073-1141: tagBoundaries with CALCULATE_EXISTING_POINTS, then
    // applyStencils in STENCIL_MODE_INPLACE_NO_SHARED; coefficient [i][j][k] with i along z
    grid.tagBoundaries<NNFull<3>>(ctx, No_check(), tag_boundaries::CALCULATE_EXISTING_POINTS);
    grid.applyStencils<Conv3x3x3_noshared<3, 0, 2>>(all, STENCIL_MODE_INPLACE_NO_SHARED, cc);
    grid.conv<0, 3, 1>(lo, hi, [cc] __device__(cp_block<float, 8>& u, int i, int j, int k) {
        float tot = 0.0f;
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b)
                for (int d = 0; d < 3; ++d) tot = __fmaf_rn(u(i + d - 1, j + b - 1, k + a - 1), cc.coeff[a][b][d], tot);
        return tot;
    });
    cudaDeviceSynchronize();
    HostMap Q2 = download(grid.handle(), 6);
    CHECK(same(Q2, 2, Q2, 3, active), "conv3x3x3_noshared_vs_conv_nnfull");

    // ---------------------------------------------------------------- removePoints + iterator
    {
        const auto before = grid.existingPoints();
        Box<3, int> rb;
        for (int d = 0; d < 3; ++d) rb.setLow(d, 20), rb.setHigh(d, 35);
        grid.remove(rb);
        grid.removePoints(ctx);
        const auto after = grid.existingPoints();
        size_t inside = 0;
        for (const auto& k : before) {
            bool in = true;
            for (int d = 0; d < 3; ++d) in = in && k.get(d) >= 20 && k.get(d) <= 35;
            inside += in;
        }
        const auto sub = grid.existingPoints(grid_key_dx<3>({0, 0, 0}), grid_key_dx<3>({15, 63, 63}));
        bool sub_ok = true;
        for (const auto& k : sub) sub_ok = sub_ok && k.get(0) <= 15;
        CHECK(before.size() == npts && inside > 0 && after.size() == npts - inside &&
                  grid.countExistingElements() == after.size() && sub_ok && !sub.empty(),
              "removePoints_and_iterator");
    }

    // ---------------------------------------------------------------- pack / unpack (ghost exchange)
    {
        // SparseGridGpu_tests.cu:1533-1700: pack two sub-boxes with properties 0 and 1,
        // unpack them into another grid, the first one shifted by +3 in x
        const grid_key_dx<3> a0({8, 10, 12}), a1({30, 40, 33}), b0({36, 0, 0}), b1({50, 63, 63});
        auto it1 = grid.getIterator(a0, a1);
        auto it2 = grid.getIterator(b0, b1);
        size_t req = 0;
        grid.packReset();
        grid.packRequest<0, 1>(it1, req);
        grid.packRequest<0, 1>(it2, req);
        grid.packCalculate<0, 1>(req, ctx);
        CudaMemory mem;
        mem.resize(req);
        Pack_stat sts;
        grid.pack<0, 1>(mem, it1, sts);
        grid.pack<0, 1>(mem, it2, sts);
        grid.packFinalize<0, 1>(mem, sts);

        Grid6 dst(sz);
        dst.setBackgroundValue<0>(0.0f);
        Unpack_stat ps;
        dst.removeAddUnpackReset();
        auto d1 = dst.getIterator(grid_key_dx<3>({11, 10, 12}), grid_key_dx<3>({33, 40, 33}));
        auto d2 = dst.getIterator(b0, b1);
        dst.remove(Box<3, int>{{11, 10, 12}, {33, 40, 33}});
        dst.unpack<0, 1>(mem, d1, ps, ctx);
        dst.remove(Box<3, int>{{36, 0, 0}, {50, 63, 63}});
        dst.unpack<0, 1>(mem, d2, ps, ctx);
        dst.removeAddUnpackFinalize<0, 1>(ctx, 0);

        const auto s1 = grid.existingPoints(a0, a1), s2 = grid.existingPoints(b0, b1);
        grid.deviceToHost<0, 1>();
        dst.deviceToHost<0, 1>();
        bool vals_ok = true;
        for (const auto& k : s1) {
            const grid_key_dx<3, int> t({k.get(0) + 3, k.get(1), k.get(2)});
            vals_ok = vals_ok && dst.get<0>(t) == grid.get<0>(k) && dst.get<1>(t) == grid.get<1>(k);
        }
        for (const auto& k : s2) vals_ok = vals_ok && dst.get<0>(k) == grid.get<0>(k) && dst.get<1>(k) == grid.get<1>(k);
        CHECK(req > 0 && sts.getOffset() == req && ps.getOffset() == req && !s1.empty() && !s2.empty() && vals_ok &&
                  dst.countExistingElements() == s1.size() + s2.size(),
              "pack_unpack");
    }

    // ---------------------------------------------------------------- host-side API
    {
        // measureBlockOccupancy: mean over chunks of the active fraction
        HostMap H = download(grid.handle(), 6);
        size_t act_pts = 0;
        for (size_t i = 0; i < H.keys.size() * 512; ++i) act_pts += active(H.mask[i]);
        double mean = 0, dev = 0;
        grid.measureBlockOccupancy(mean, dev);
        const bool occ_ok = std::fabs(mean * (double)H.keys.size() * 512 - (double)act_pts) < 1e-6 && dev >= 0;
        CHECK(occ_ok, "measureBlockOccupancy");

        // conv_cross_b: the face stencil equals conv over NNStar; the data block reads other properties
        grid.setNNType<NNStar<3>>();
        grid.conv_cross_b<0, 4, 1>(lo, hi, [] __device__(cp_block<float, 8>& u, data_block<8>&, int, int i, int j,
                                                         int k) {
            return __fadd_rn(__fadd_rn(u(i - 1, j, k), u(i + 1, j, k)), __fadd_rn(u(i, j - 1, k), u(i, j, k + 1)));
        });
        grid.conv<0, 5, 1>(lo, hi, [] __device__(cp_block<float, 8>& u, int i, int j, int k) {
            return __fadd_rn(__fadd_rn(u(i - 1, j, k), u(i + 1, j, k)), __fadd_rn(u(i, j - 1, k), u(i, j, k + 1)));
        });
        cudaDeviceSynchronize();
        HostMap C1 = download(grid.handle(), 6);
        const bool cb1 = same(C1, 4, C1, 5, active);
        grid.conv_cross_b<0, 4, 1>(lo, hi, [] __device__(cp_block<float, 8>&, data_block<8>& blk, int off, int, int,
                                                         int) { return blk.template get<1>()[off]; });
        cudaDeviceSynchronize();
        HostMap C2 = download(grid.handle(), 6);
        CHECK(cb1 && same(C2, 4, C2, 1, active), "conv_cross_b");

        // insertFlush on the host copy, then hostToDevice
        Grid6 h(sz);
        h.setBackgroundValue<0>(0.0f);
        h.deviceToHost<>();
        h.insertFlush<0>(grid_key_dx<3, int>({3, 4, 5})) = 7.5f;
        h.insertFlush<0>(grid_key_dx<3, int>({60, 61, 62})) = -2.0f;
        h.insertFlush<0>(grid_key_dx<3, int>({4, 4, 5})) = 1.25f;  // same chunk as the first point
        h.hostToDevice();
        h.deviceToHost<0>();
        const bool ins_ok = h.countExistingElements() == 3 && h.nchunks() == 2 &&
                            h.get<0>(grid_key_dx<3, int>({3, 4, 5})) == 7.5f &&
                            h.get<0>(grid_key_dx<3, int>({60, 61, 62})) == -2.0f &&
                            h.get<0>(grid_key_dx<3, int>({4, 4, 5})) == 1.25f &&
                            h.get<0>(grid_key_dx<3, int>({5, 4, 5})) == 0.0f;
        CHECK(ins_ok, "insertFlush_hostToDevice");

        // swap and removeUnusedBuffers: the grids trade contents; a flush and a stencil still run
        const size_t na = grid.countExistingElements(), nb = h.countExistingElements();
        grid.swap(h);
        const bool sw = grid.countExistingElements() == nb && h.countExistingElements() == na;
        grid.swap(h);
        grid.removeUnusedBuffers();
        grid.applyStencils<HeatStencil<3, 0, 1>>(grid.getBox(), STENCIL_MODE_INPLACE, 0.1f);
        cudaDeviceSynchronize();
        CHECK(sw && grid.countExistingElements() == na && grid.private_get_neighborhood_array() != nullptr,
              "swap_removeUnusedBuffers");
    }

    // ---------------------------------------------------------------- device remove
    {
        // remove from a kernel, then the heat stencil: equal to a grid that never had those points
        Grid6 rg(sz), og(sz);
        rg.setBackgroundValue<0>(0.25f);
        og.setBackgroundValue<0>(0.25f);
        rg.setGPUInsertBuffer(dim3(N / 8, N / 8, N / 8), dim3(1024, 1, 1));
        insert_shape<0><<<dim3(N / 8, N / 8, N / 8), dim3(8, 8, 8)>>>(rg.toKernel());
        rg.flush<smax_<0>>(ctx, FLUSH_ON_DEVICE);
        remove_even<<<dim3(N / 8, N / 8, N / 8), dim3(8, 8, 8)>>>(rg.toKernel());
        std::vector<int32_t> oc;
        std::vector<float> ov;
        size_t odd = 0;
        for (int z = 0; z < N; ++z)
            for (int y = 0; y < N; ++y)
                for (int x = 0; x < N; ++x)
                    if (in_shape(x, y, z) && (x + y + z) % 2 == 1) {
                        oc.insert(oc.end(), {x, y, z});
                        ov.push_back(val_a(x, y, z));
                        ++odd;
                    }
        int32_t* dc;
        float* dv;
        cudaMalloc(&dc, oc.size() * 4);
        cudaMalloc(&dv, ov.size() * 4);
        cudaMemcpy(dc, oc.data(), oc.size() * 4, cudaMemcpyHostToDevice);
        cudaMemcpy(dv, ov.data(), ov.size() * 4, cudaMemcpyHostToDevice);
        const void* vals[6] = {dv, nullptr, nullptr, nullptr, nullptr, nullptr};
        check(sgb_insert(og.handle(), (int64_t)odd, dc, vals, nullptr), "sgb_insert");
        int ops[6] = {SGB_OP_MAX, SGB_OP_NONE, SGB_OP_NONE, SGB_OP_NONE, SGB_OP_NONE, SGB_OP_NONE};
        check(sgb_flush(og.handle(), ops, nullptr), "sgb_flush");
        cudaDeviceSynchronize();
        cudaFree(dc);
        cudaFree(dv);
        const bool cnt_ok = rg.countExistingElements() == odd && og.countExistingElements() == odd;
        rg.tagBoundaries<NNStar<3>>(ctx);
        og.tagBoundaries<NNStar<3>>(ctx);
        rg.applyStencils<HeatStencil<3, 0, 1>>(rg.getBox(), STENCIL_MODE_INPLACE, 0.1f);
        og.applyStencils<HeatStencil<3, 0, 1>>(og.getBox(), STENCIL_MODE_INPLACE, 0.1f);
        cudaDeviceSynchronize();
        rg.deviceToHost<0, 1>();
        og.deviceToHost<0, 1>();
        bool eq = cnt_ok && rg.countBoundaryElements() == og.countBoundaryElements();
        for (int z = 0; z < N && eq; ++z)
            for (int y = 0; y < N; ++y)
                for (int x = 0; x < N; ++x) {
                    const grid_key_dx<3, int> k({x, y, z});
                    const float a = rg.get<1>(k), b = og.get<1>(k);
                    eq = eq && std::memcmp(&a, &b, 4) == 0;
                }
        CHECK(eq, "device_remove_then_heat");
    }

    // ---------------------------------------------------------------- SparseGridGpu_z (Morton chunk ids)
    {
        Grid6 sg(sz);
        SparseGridGpu_z<3, Agg6, 8> zg(sz);
        sg.setBackgroundValue<0>(0.0f);
        zg.setBackgroundValue<0>(0.0f);
        sg.setGPUInsertBuffer(dim3(N / 8, N / 8, N / 8), dim3(1024, 1, 1));
        zg.setGPUInsertBuffer(dim3(N / 8, N / 8, N / 8), dim3(1024, 1, 1));
        insert_shape<0><<<dim3(N / 8, N / 8, N / 8), dim3(8, 8, 8)>>>(sg.toKernel());
        insert_shape<0><<<dim3(N / 8, N / 8, N / 8), dim3(8, 8, 8)>>>(zg.toKernel());
        sg.flush<smax_<0>>(ctx, FLUSH_ON_DEVICE);
        zg.flush<smax_<0>>(ctx, FLUSH_ON_DEVICE);
        sg.tagBoundaries<NNStar<3>>(ctx);
        zg.tagBoundaries<NNStar<3>>(ctx);
        sg.applyStencils<HeatStencil<3, 0, 1>>(sg.getBox(), STENCIL_MODE_INPLACE, 0.1f);
        zg.applyStencils<HeatStencil<3, 0, 1>>(zg.getBox(), STENCIL_MODE_INPLACE, 0.1f);
        cudaDeviceSynchronize();
        sg.deviceToHost<0, 1>();
        zg.deviceToHost<0, 1>();
        bool eq = zg.countExistingElements() == npts && sg.nchunks() == zg.nchunks();
        for (int z = 0; z < N && eq; ++z)
            for (int y = 0; y < N; ++y)
                for (int x = 0; x < N; ++x) {
                    const grid_key_dx<3, int> k({x, y, z});
                    const float a0 = sg.get<0>(k), b0 = zg.get<0>(k), a1 = sg.get<1>(k), b1 = zg.get<1>(k);
                    eq = eq && std::memcmp(&a0, &b0, 4) == 0 && std::memcmp(&a1, &b1, 4) == 0 &&
                         sg.getFlag(k) == zg.getFlag(k);
                }
        // the chunk ids differ: Morton codes, sorted
        std::vector<int64_t> zk(zg.nchunks());
        cudaMemcpy(zk.data(), zg.private_get_index_array(), zk.size() * 8, cudaMemcpyDeviceToHost);
        bool morton = true;
        for (size_t i = 1; i < zk.size(); ++i) morton = morton && zk[i] > zk[i - 1];
        CHECK(eq && morton, "sparsegridgpu_z_insert_tag_heat");
        // write(): a VTK file of every point whose mask byte is not 0
        const std::string vtk = "/tmp/sgb_dropin_" + std::to_string((long)getpid()) + ".vtk";
        bool wrote = zg.write(vtk);
        std::ifstream in(vtk, std::ios::binary);
        std::string head;
        std::getline(in, head);
        std::string all((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
        wrote = wrote && head == "# vtk DataFile Version 3.0" &&
                all.find("POINTS " + std::to_string(npts) + " float") != std::string::npos;
        std::remove(vtk.c_str());
        CHECK(wrote, "write_vtk");
    }

    // ---------------------------------------------------------------- insertBlock (chunk slots)
    {
        // the sphere shell of insertSphere3D written through insertBlock, against the same points
        // through the staged C ABI insert
        Grid6 bg(sz), rg(sz);
        bg.setBackgroundValue<0>(0.0f);
        rg.setBackgroundValue<0>(0.0f);
        const dim3 gsz(N / 8, N / 8, N / 8);
        bg.setGPUInsertBuffer(gsz, dim3(1, 1, 1));
        insert_sphere_blocks<0><<<gsz, 512>>>(bg.toKernel(), grid_key_dx<3, int>({0, 0, 0}), 28.0f, 12.0f, 0.5f);
        bg.flush<smax_<0>>(ctx, FLUSH_ON_DEVICE);
        std::vector<int32_t> sc;
        std::vector<float> sv;
        for (int bz = 0; bz < N / 8; ++bz)
            for (int by = 0; by < N / 8; ++by)
                for (int bx = 0; bx < N / 8; ++bx)
                    for (int o = 0; o < 512; ++o) {
                        const long x = bx * 8 + o % 8, y = by * 8 + (o / 8) % 8, z = bz * 8 + o / 64;
                        const long dx = x - N / 2, dy = y - N / 2, dz = z - N / 2;
                        const float r = sqrtf((float)(dx * dx + dy * dy + dz * dz));
                        if (r < 28.0f && r >= 12.0f) {
                            sc.insert(sc.end(), {(int32_t)x, (int32_t)y, (int32_t)z});
                            sv.push_back(0.5f + (float)(x + 3 * y));
                        }
                    }
        int32_t* dc;
        float* dv;
        cudaMalloc(&dc, sc.size() * 4);
        cudaMalloc(&dv, sv.size() * 4);
        cudaMemcpy(dc, sc.data(), sc.size() * 4, cudaMemcpyHostToDevice);
        cudaMemcpy(dv, sv.data(), sv.size() * 4, cudaMemcpyHostToDevice);
        const void* vals[6] = {dv, nullptr, nullptr, nullptr, nullptr, nullptr};
        check(sgb_insert(rg.handle(), (int64_t)sv.size(), dc, vals, nullptr), "sgb_insert");
        int ops[6] = {SGB_OP_MAX, SGB_OP_NONE, SGB_OP_NONE, SGB_OP_NONE, SGB_OP_NONE, SGB_OP_NONE};
        check(sgb_flush(rg.handle(), ops, nullptr), "sgb_flush");
        cudaDeviceSynchronize();
        cudaFree(dc);
        cudaFree(dv);
        HostMap A = download(bg.handle(), 6), B = download(rg.handle(), 6);
        CHECK(!A.keys.empty() && A.keys == B.keys && A.mask == B.mask && same(A, 0, B, 0, existing) &&
                  bg.countExistingElements() == sv.size(),
              "insertBlock_sphere_shell");

        // insertConstantValue2: two properties through one chunk slot per CTA, twice (the second
        // flush merges into the existing chunks with smax_)
        Grid6 cg(sz);
        cg.setGPUInsertBuffer(gsz, dim3(1, 1, 1));
        insert_constant_blocks<0, 2><<<gsz, dim3(8, 8, 8)>>>(cg.toKernel(), 3.0f);
        cg.flush<smax_<0>, smax_<2>>(ctx, FLUSH_ON_DEVICE);
        insert_constant_blocks<0, 2><<<gsz, dim3(8, 8, 8)>>>(cg.toKernel(), 2.0f);
        cg.flush<smax_<0>, smax_<2>>(ctx, FLUSH_ON_DEVICE);
        cg.deviceToHost<0, 2>();
        bool all3 = cg.countExistingElements() == (size_t)N * N * N;
        for (int z = 0; z < N && all3; z += 3)
            for (int y = 0; y < N; y += 5)
                for (int x = 0; x < N; ++x) {
                    const grid_key_dx<3, int> k({x, y, z});
                    all3 = all3 && cg.get<0>(k) == 3.0f && cg.get<2>(k) == 3.0f;
                }
        CHECK(all3, "insertBlock_constant_two_properties");
    }

    // ---------------------------------------------------------------- conv lambdas on int / double / float
    {
        // the shell of in_shape with integer values in int, double and float properties: the 7-point sums
        // are exact in every type, so each typed result must equal the host's sum (points that do not
        // exist, and absent chunks, read the background 0)
        typedef SparseGridGpu<3, aggregate<int, double, float, int, double, float>, 8> GridM;
        GridM mg(sz);
        mg.setBackgroundValue<0>(0);
        mg.setBackgroundValue<1>(0.0);
        mg.setBackgroundValue<2>(0.0f);
        mg.setBackgroundValue<3>(0);
        mg.setBackgroundValue<4>(0.0);
        mg.setBackgroundValue<5>(0.0f);
        auto iv = [](int x, int y, int z) { return (x * 7 + y * 13 + z * 29) % 97; };
        std::vector<int64_t> mk;
        for (int bz = 0; bz < N / 8; ++bz)
            for (int by = 0; by < N / 8; ++by)
                for (int bx = 0; bx < N / 8; ++bx) {
                    bool any = false;
                    for (int o = 0; o < 512 && !any; ++o) any = in_shape(bx * 8 + o % 8, by * 8 + (o / 8) % 8, bz * 8 + o / 64);
                    if (any) mk.push_back(bx + (N / 8) * (by + (N / 8) * (int64_t)bz));
                }
        const int64_t mn = (int64_t)mk.size();
        std::vector<int> mi((mn + 1) * 512, 0);
        std::vector<double> md((mn + 1) * 512, 0.0);
        std::vector<float> mf((mn + 1) * 512, 0.0f);
        std::vector<uint8_t> mm((mn + 1) * 512, 0);
        auto coord = [&](int64_t c, int o, int& x, int& y, int& z) {
            x = (int)(mk[c] % (N / 8)) * 8 + o % 8;
            y = (int)((mk[c] / (N / 8)) % (N / 8)) * 8 + (o / 8) % 8;
            z = (int)(mk[c] / (N / 8 * N / 8)) * 8 + o / 64;
        };
        for (int64_t c = 0; c < mn; ++c)
            for (int o = 0; o < 512; ++o) {
                int x, y, z;
                coord(c, o, x, y, z);
                if (!in_shape(x, y, z)) continue;
                mi[c * 512 + o] = iv(x, y, z);
                md[c * 512 + o] = iv(x, y, z);
                mf[c * 512 + o] = (float)iv(x, y, z);
                mm[c * 512 + o] = 1;
            }
        auto load = [&] {
            const void* d[6] = {mi.data(), md.data(), mf.data(), mi.data(), md.data(), mf.data()};
            check(sgb_load_map(mg.handle(), mn, mk.data(), d, mm.data(), nullptr), "load_map");
        };
        // results at the existing points: the host's sum, in each typed property 3, 4, 5
        auto verify = [&] {
            std::vector<int64_t> k(mn);
            std::vector<int> ri((mn + 1) * 512), di((mn + 1) * 512);
            std::vector<double> rd((mn + 1) * 512), dd((mn + 1) * 512);
            std::vector<float> rf((mn + 1) * 512), df((mn + 1) * 512);
            std::vector<uint8_t> m((mn + 1) * 512);
            void* ptrs[6] = {di.data(), dd.data(), df.data(), ri.data(), rd.data(), rf.data()};
            check(sgb_download_map(mg.handle(), k.data(), ptrs, m.data(), nullptr), "download");
            auto at = [&](int x, int y, int z) {
                return (x >= 0 && y >= 0 && z >= 0 && x < N && y < N && z < N && in_shape(x, y, z)) ? iv(x, y, z) : 0;
            };
            bool ok = k == mk;
            size_t cnt = 0;
            for (int64_t c = 0; c < mn && ok; ++c)
                for (int o = 0; o < 512; ++o) {
                    if (m[c * 512 + o] != 1) continue;
                    int x, y, z;
                    coord(c, o, x, y, z);
                    const int e = at(x, y, z) + at(x - 1, y, z) + at(x + 1, y, z) + at(x, y - 1, z) + at(x, y + 1, z) +
                                  at(x, y, z - 1) + at(x, y, z + 1);
                    const int64_t i = c * 512 + o;
                    ok = ok && ri[i] == e && rd[i] == (double)e && rf[i] == (float)e;
                    ++cnt;
                }
            return ok && cnt > 0;
        };
        const grid_key_dx<3> mlo({0, 0, 0}), mhi({N - 1, N - 1, N - 1});
        load();
        mg.conv<0, 3, 1>(mlo, mhi, [] __device__(cp_block<int, 8>& u, int i, int j, int k) {
            return u(i, j, k) + u(i - 1, j, k) + u(i + 1, j, k) + u(i, j - 1, k) + u(i, j + 1, k) + u(i, j, k - 1) +
                   u(i, j, k + 1);
        });
        mg.conv<1, 4, 1>(mlo, mhi, [] __device__(cp_block<double, 8>& u, int i, int j, int k) {
            return u(i, j, k) + u(i - 1, j, k) + u(i + 1, j, k) + u(i, j - 1, k) + u(i, j + 1, k) + u(i, j, k - 1) +
                   u(i, j, k + 1);
        });
        mg.conv<2, 5, 1>(mlo, mhi, [] __device__(cp_block<float, 8>& u, int i, int j, int k) {
            return u(i, j, k) + u(i - 1, j, k) + u(i + 1, j, k) + u(i, j - 1, k) + u(i, j + 1, k) + u(i, j, k - 1) +
                   u(i, j, k + 1);
        });
        cudaDeviceSynchronize();
        CHECK(verify(), "conv_int_double_float");
        load();  // properties 3, 4, 5 back to the inputs, which differ from the sums
        mg.conv3_b<0, 1, 2, 3, 4, 5, 1>(
            mlo, mhi,
            [] __device__(int& a, double& b, float& c, cp_block<int, 8>& u, cp_block<double, 8>& v,
                          cp_block<float, 8>& w, data_block<8>&, int, int i, int j, int k) {
                a = u(i, j, k) + u(i - 1, j, k) + u(i + 1, j, k) + u(i, j - 1, k) + u(i, j + 1, k) + u(i, j, k - 1) +
                    u(i, j, k + 1);
                b = v(i, j, k) + v(i - 1, j, k) + v(i + 1, j, k) + v(i, j - 1, k) + v(i, j + 1, k) + v(i, j, k - 1) +
                    v(i, j, k + 1);
                c = w(i, j, k) + w(i - 1, j, k) + w(i + 1, j, k) + w(i, j - 1, k) + w(i, j + 1, k) + w(i, j, k - 1) +
                    w(i, j, k + 1);
            });
        cudaDeviceSynchronize();
        CHECK(verify(), "conv3_b_int_double_float");
    }
    {
        // the same sums on 4^3 chunks (64 points a chunk, fewer than a CTA's threads)
        typedef SparseGridGpu<3, aggregate<float, float, float, float, float, float>, 4> Grid4e;
        Grid4e eg(sz);
        eg.setBackgroundValue<0>(0.0f);
        eg.setBackgroundValue<1>(0.0f);
        eg.setBackgroundValue<2>(0.0f);
        eg.setBackgroundValue<3>(0.0f);
        eg.setBackgroundValue<4>(0.0f);
        eg.setBackgroundValue<5>(0.0f);
        auto iv = [](int x, int y, int z) { return (x * 7 + y * 13 + z * 29) % 97; };
        constexpr int B = N / 4;
        std::vector<int64_t> ek;
        for (int bz = 0; bz < B; ++bz)
            for (int by = 0; by < B; ++by)
                for (int bx = 0; bx < B; ++bx) {
                    bool any = false;
                    for (int o = 0; o < 64 && !any; ++o) any = in_shape(bx * 4 + o % 4, by * 4 + (o / 4) % 4, bz * 4 + o / 16);
                    if (any) ek.push_back(bx + B * (by + B * (int64_t)bz));
                }
        const int64_t en = (int64_t)ek.size();
        std::vector<float> ev((en + 1) * 64, 0.0f);
        std::vector<uint8_t> em((en + 1) * 64, 0);
        auto coord = [&](int64_t c, int o, int& x, int& y, int& z) {
            x = (int)(ek[c] % B) * 4 + o % 4;
            y = (int)((ek[c] / B) % B) * 4 + (o / 4) % 4;
            z = (int)(ek[c] / (B * B)) * 4 + o / 16;
        };
        for (int64_t c = 0; c < en; ++c)
            for (int o = 0; o < 64; ++o) {
                int x, y, z;
                coord(c, o, x, y, z);
                if (!in_shape(x, y, z)) continue;
                ev[c * 64 + o] = (float)iv(x, y, z);
                em[c * 64 + o] = 1;
            }
        const void* d[6] = {ev.data(), ev.data(), ev.data(), ev.data(), ev.data(), ev.data()};
        check(sgb_load_map(eg.handle(), en, ek.data(), d, em.data(), nullptr), "load_map");
        const grid_key_dx<3> elo({0, 0, 0}), ehi({N - 1, N - 1, N - 1});
        auto at = [&](int x, int y, int z) {
            return (x >= 0 && y >= 0 && z >= 0 && x < N && y < N && z < N && in_shape(x, y, z)) ? iv(x, y, z) : 0;
        };
        // every existing point's results in properties 3, 4, 5 against expected(x, y, z, p)
        auto verify = [&](auto expected) {
            std::vector<int64_t> k2(en);
            std::vector<std::vector<float>> r(6, std::vector<float>((en + 1) * 64));
            std::vector<uint8_t> m2((en + 1) * 64);
            void* ptrs[6] = {r[0].data(), r[1].data(), r[2].data(), r[3].data(), r[4].data(), r[5].data()};
            check(sgb_download_map(eg.handle(), k2.data(), ptrs, m2.data(), nullptr), "download");
            bool ok = k2 == ek;
            size_t cnt = 0;
            for (int64_t c = 0; c < en && ok; ++c)
                for (int o = 0; o < 64; ++o) {
                    if (m2[c * 64 + o] != 1) continue;
                    int x, y, z;
                    coord(c, o, x, y, z);
                    for (int p = 3; p < 6; ++p) ok = ok && r[p][c * 64 + o] == (float)expected(x, y, z, p);
                    ++cnt;
                }
            return ok && cnt > 0;
        };
        // conv3_b: three different reads of the three (equal) source fields
        eg.conv3_b<0, 1, 2, 3, 4, 5, 1>(
            elo, ehi,
            [] __device__(float& a, float& b, float& c, cp_block<float, 4>& u, cp_block<float, 4>& v,
                          cp_block<float, 4>& w, data_block<8>&, int, int i, int j, int k) {
                a = u(i + 1, j, k) + u(i, j + 1, k) + u(i, j, k + 1);
                b = v(i - 1, j, k) + v(i, j - 1, k) + v(i, j, k - 1);
                c = w(i, j, k);
            });
        cudaDeviceSynchronize();
        const bool ok3 = verify([&](int x, int y, int z, int p) {
            return p == 3 ? at(x + 1, y, z) + at(x, y + 1, z) + at(x, y, z + 1)
                 : p == 4 ? at(x - 1, y, z) + at(x, y - 1, z) + at(x, y, z - 1)
                          : at(x, y, z);
        });
        // conv: the 7-point sum into property 3, the others unchanged
        eg.conv<0, 3, 1>(elo, ehi, [] __device__(cp_block<float, 4>& u, int i, int j, int k) {
            return u(i, j, k) + u(i - 1, j, k) + u(i + 1, j, k) + u(i, j - 1, k) + u(i, j + 1, k) + u(i, j, k - 1) +
                   u(i, j, k + 1);
        });
        cudaDeviceSynchronize();
        const bool ok1 = verify([&](int x, int y, int z, int p) {
            return p == 3 ? at(x, y, z) + at(x - 1, y, z) + at(x + 1, y, z) + at(x, y - 1, z) + at(x, y + 1, z) +
                                at(x, y, z - 1) + at(x, y, z + 1)
                 : p == 4 ? at(x - 1, y, z) + at(x, y - 1, z) + at(x, y, z - 1)
                          : at(x, y, z);
        });
        CHECK(ok3 && ok1, "conv_and_conv3_b_on_4x4x4_chunks");
    }

    // ---------------------------------------------------------------- user stencil functors
    {
        // testStencilHeat (SparseGridGpu_tests.cu:472-518) in 3-D: a 16^3 grid of 2^3 chunks, padding
        // points set to 10 x / 15 by a boundary functor, then 1000 pairs of heat steps of the
        // reference's HeatStencil written as user code: the interior relaxes to the linear profile
        typedef SparseGridGpu<3, aggregate<float, float>, 8> Grid2;
        const size_t s16[3] = {16, 16, 16};
        Grid2 hg(s16), fg(s16);
        for (Grid2* g : {&hg, &fg}) {
            g->setBackgroundValue<0>(0.0f);
            g->setGPUInsertBuffer(dim3(2, 2, 2), dim3(1, 1, 1));
            insert_constant_blocks<0, 1><<<dim3(2, 2, 2), dim3(8, 8, 8)>>>(g->toKernel(), 0.0f);
            g->flush<smax_<0>, smax_<1>>(ctx, FLUSH_ON_DEVICE);
            g->findNeighbours();
            g->tagBoundaries(ctx);
            g->applyStencils<UserBoundarySetXRescaled<3, 0, 0>>(g->getBox(), STENCIL_MODE_INPLACE, 0.0, 16, 0.0, 10.0);
        }
        {
            // which rounding does nvcc give the reference's HeatStencil?  One step of the functor on a
            // twin grid, against the two candidate roundings of the first Laplacian term computed
            // here: -6 cur rounded, then + (xm + xp) rounded; or both in one fused multiply-add
            Grid2 dg(s16);
            dg.setBackgroundValue<0>(0.0f);
            dg.setGPUInsertBuffer(dim3(2, 2, 2), dim3(1, 1, 1));
            insert_constant_blocks<0, 1><<<dim3(2, 2, 2), dim3(8, 8, 8)>>>(dg.toKernel(), 0.0f);
            dg.flush<smax_<0>, smax_<1>>(ctx, FLUSH_ON_DEVICE);
            dg.tagBoundaries(ctx);
            dg.applyStencils<UserBoundarySetXRescaled<3, 0, 0>>(dg.getBox(), STENCIL_MODE_INPLACE, 0.0, 16, 0.0, 10.0);
            for (int k = 0; k < 6; ++k) {  // some structure in the interior first
                dg.applyStencils<HeatStencil<3, 0, 1>>(dg.getBox(), STENCIL_MODE_INPLACE, 0.1f);
                dg.applyStencils<HeatStencil<3, 1, 0>>(dg.getBox(), STENCIL_MODE_INPLACE, 0.1f);
            }
            HostMap pre = download(dg.handle(), 2);
            dg.applyStencils<UserHeatStencil<3, 0, 1>>(dg.getBox(), STENCIL_MODE_INPLACE, 0.1f);
            HostMap post = download(dg.handle(), 2);
            auto at = [&](int x, int y, int z) -> float {
                if (x < 0 || y < 0 || z < 0 || x >= 16 || y >= 16 || z >= 16) return 0.0f;
                const long key = (x / 8) + 2 * ((y / 8) + 2 * (long)(z / 8));
                for (size_t i = 0; i < pre.keys.size(); ++i)
                    if (pre.keys[i] == key) {
                        const size_t o = i * 512 + (x % 8) + 8 * ((y % 8) + 8 * (z % 8));
                        return pre.mask[o] ? pre.data[0][o] : 0.0f;
                    }
                return 0.0f;
            };
            size_t nact = 0, sep_ok = 0, fused_ok = 0;
            for (size_t c = 0; c < pre.keys.size(); ++c) {
                const int bx = (int)(pre.keys[c] % 2), by = (int)((pre.keys[c] / 2) % 2), bz = (int)(pre.keys[c] / 4);
                for (int o = 0; o < 512; ++o) {
                    if ((pre.mask[c * 512 + o] & 3) != 1) continue;
                    const int x = bx * 8 + o % 8, y = by * 8 + (o / 8) % 8, z = bz * 8 + o / 64;
                    const float cur = at(x, y, z);
                    const float sx = at(x - 1, y, z) + at(x + 1, y, z), sy = at(x, y - 1, z) + at(x, y + 1, z),
                                sz = at(x, y, z - 1) + at(x, y, z + 1);
                    volatile float m6 = (float)(-6.0 * (double)cur);
                    float lsep = m6 + sx;
                    lsep = lsep + sy;
                    lsep = lsep + sz;
                    float lfus = std::fmaf(-6.0f, cur, sx);
                    lfus = lfus + sy;
                    lfus = lfus + sz;
                    const float rsep = std::fmaf(0.1f, lsep, cur), rfus = std::fmaf(0.1f, lfus, cur);
                    const float got = post.data[1][c * 512 + o];
                    ++nact;
                    sep_ok += std::memcmp(&got, &rsep, 4) == 0;
                    fused_ok += std::memcmp(&got, &rfus, 4) == 0;
                }
            }
            std::printf("  reference HeatStencil compiled here: %zu active points, %zu match the separate rounding, "
                        "%zu the fused multiply-add\n",
                        nact, sep_ok, fused_ok);
            // the library's HeatStencil (and the oracle) use the rounding nvcc gives the reference's source
            CHECK(nact > 0 && fused_ok == nact, "HeatStencil_rounding_is_the_fused_multiply_add");
        }
        for (int it = 0; it < 1000; ++it) {
            hg.applyStencils<UserHeatStencil<3, 0, 1>>(hg.getBox(), STENCIL_MODE_INPLACE, 0.1f);
            hg.applyStencils<UserHeatStencil<3, 1, 0>>(hg.getBox(), STENCIL_MODE_INPLACE, 0.01f);
            if (it < 50) {  // the library's fixed-function HeatStencil on the twin grid
                fg.applyStencils<HeatStencil<3, 0, 1>>(fg.getBox(), STENCIL_MODE_INPLACE, 0.1f);
                fg.applyStencils<HeatStencil<3, 1, 0>>(fg.getBox(), STENCIL_MODE_INPLACE, 0.01f);
            }
            if (it == 49) {
                HostMap a = download(hg.handle(), 2), b = download(fg.handle(), 2);
                for (int p = 0; p < 2; ++p)
                    for (size_t i = 0; i < a.keys.size() * 512; ++i)
                        if (existing(a.mask[i]) && std::memcmp(&a.data[p][i], &b.data[p][i], 4) != 0) {
                            std::printf("  first difference: property %d point %zu mask %d user %.9g fixed %.9g\n", p, i,
                                        (int)a.mask[i], a.data[p][i], b.data[p][i]);
                            break;
                        }
                CHECK(same(a, 0, b, 0, existing) && same(a, 1, b, 1, existing), "user_HeatStencil_equals_fixed_50");
            }
        }
        hg.deviceToHost<0, 1>();
        bool prof = hg.countExistingElements() == 4096;
        for (int z = 0; z < 16; ++z)
            for (int y = 0; y < 16; ++y)
                for (int x = 0; x < 16; ++x) {
                    const float expect = 10.0f * x / 15.0f;
                    prof = prof && std::fabs(hg.get<1>(grid_key_dx<3, int>({x, y, z})) - expect) < 1e-2f;
                }
        CHECK(prof, "testStencilHeat_3d_user_functor_linear_profile");

        // testStencil_lap_simplified (SparseGridGpu_tests.cu:520-566) in 3-D with conv_cross lambdas
        Grid2 lg(s16);
        lg.setBackgroundValue<0>(0.0f);
        lg.setGPUInsertBuffer(dim3(2, 2, 2), dim3(1, 1, 1));
        insert_constant_blocks<0, 1><<<dim3(2, 2, 2), dim3(8, 8, 8)>>>(lg.toKernel(), 0.0f);
        lg.flush<smax_<0>, smax_<1>>(ctx, FLUSH_ON_DEVICE);
        lg.findNeighbours();
        lg.tagBoundaries(ctx);
        lg.applyStencils<UserBoundarySetXRescaled<3, 0, 0>>(lg.getBox(), STENCIL_MODE_INPLACE, 0.0, 16, 0.0, 10.0);
        for (int it = 0; it < 1000; ++it) {
            lg.conv_cross<0, 1, 1>({0, 0, 0}, {16, 16, 16}, [] __device__(float& u, cross_stencil<3, float>& cs) {
                return u + (cs.xm[0] + cs.xp[0] + cs.xm[1] + cs.xp[1] + cs.xm[2] + cs.xp[2] - 6.0f * u) * 0.1f;
            });
            lg.conv_cross<1, 0, 1>({0, 0, 0}, {16, 16, 16}, [] __device__(float& u, cross_stencil<3, float>& cs) {
                return u + (cs.xm[0] + cs.xp[0] + cs.xm[1] + cs.xp[1] + cs.xm[2] + cs.xp[2] - 6.0f * u) * 0.1f;
            });
        }
        lg.deviceToHost<0, 1>();
        bool lap = true;
        for (int z = 0; z < 16; ++z)
            for (int y = 0; y < 16; ++y)
                for (int x = 0; x < 16; ++x)
                    lap = lap && std::fabs(lg.get<1>(grid_key_dx<3, int>({x, y, z})) - 10.0f * x / 15.0f) < 1e-2f;
        CHECK(lap, "testStencil_lap_simplified_3d_conv_cross");

        // Conv3x3x3 and Conv3x3x3_noshared as user functors against the library's kernels, on the
        // shell grid (holes, absent neighbour chunks), bit for bit at the active points
        Grid6 cg(sz);
        cg.setBackgroundValue<0>(0.0f);
        cg.setGPUInsertBuffer(dim3(N / 8, N / 8, N / 8), dim3(1024, 1, 1));
        insert_shape<0><<<dim3(N / 8, N / 8, N / 8), dim3(8, 8, 8)>>>(cg.toKernel());
        cg.flush<smax_<0>>(ctx, FLUSH_ON_DEVICE);
        cg.setNNType<NNFull<3>>();
        cg.tagBoundaries<NNFull<3>>(ctx, No_check(), tag_boundaries::CALCULATE_EXISTING_POINTS);
        conv_coeff cc;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                for (int k = 0; k < 3; ++k) cc.coeff[i][j][k] = 0.01f * (float)(1 + i + 3 * j + 9 * k);
        cg.applyStencils<UserConv3x3x3<3, 0, 1>>(cg.getBox(), STENCIL_MODE_INPLACE, cc);
        cg.applyStencils<Conv3x3x3<3, 0, 2>>(cg.getBox(), STENCIL_MODE_INPLACE, cc);
        cg.applyStencils<UserConv3x3x3NoShared<3, 0, 3>>(cg.getBox(), STENCIL_MODE_INPLACE_NO_SHARED, cc);
        cg.applyStencils<Conv3x3x3_noshared<3, 0, 4>>(cg.getBox(), STENCIL_MODE_INPLACE_NO_SHARED, cc);
        cudaDeviceSynchronize();
        HostMap C = download(cg.handle(), 6);
        size_t nact = 0;
        for (uint8_t m : C.mask) nact += active(m);
        CHECK(nact > 1000 && same(C, 1, C, 2, active), "user_Conv3x3x3_equals_fixed");
        CHECK(same(C, 3, C, 4, active), "user_Conv3x3x3_noshared_equals_fixed");

        // loadGhostBlock with a mask tile on NNStar: the edge / corner halo cells come from neighbour 0
        // (the -x chunk) at the wrapped coordinate, as the reference's ghost-layer map gives them
        cg.setNNType<NNStar<3>>();
        cg.applyStencils<UserCountTile<0, 5>>(cg.getBox(), STENCIL_MODE_INPLACE);
        cudaDeviceSynchronize();
        HostMap T = download(cg.handle(), 6);
        const int bz8 = N / 8;
        auto pos_of = [&](int bx, int by, int bz) -> long {
            if (bx < 0 || by < 0 || bz < 0 || bx >= bz8 || by >= bz8 || bz >= bz8) return -1;
            const long key = bx + bz8 * (by + (long)bz8 * bz);
            for (size_t i = 0; i < T.keys.size(); ++i)
                if (T.keys[i] == key) return (long)i;
            return -1;
        };
        bool rule = true;
        for (size_t c = 0; c < T.keys.size() && rule; ++c) {
            const int bx = (int)(T.keys[c] % bz8), by = (int)((T.keys[c] / bz8) % bz8), bz = (int)(T.keys[c] / (bz8 * bz8));
            for (int o = 0; o < 512; ++o) {
                if (!(T.mask[c * 512 + o] & 1)) continue;
                const int lx = o % 8, ly = (o / 8) % 8, lz = o / 64;
                float acc = 0;
                for (int dz = -1; dz <= 1; ++dz)
                    for (int dy = -1; dy <= 1; ++dy)
                        for (int dx = -1; dx <= 1; ++dx) {
                            const int tx = lx + dx, ty = ly + dy, tz = lz + dz;
                            const int ox = tx < 0 ? -1 : (tx > 7 ? 1 : 0), oy = ty < 0 ? -1 : (ty > 7 ? 1 : 0),
                                      oz = tz < 0 ? -1 : (tz > 7 ? 1 : 0);
                            const int nout = (ox != 0) + (oy != 0) + (oz != 0);
                            long src = (long)c;
                            if (nout == 1) src = pos_of(bx + ox, by + oy, bz + oz);
                            else if (nout > 1) src = pos_of(bx - 1, by, bz);
                            const int w = ((tx + 8) % 8) + 8 * (((ty + 8) % 8) + 8 * ((tz + 8) % 8));
                            acc += (src >= 0 && (T.mask[src * 512 + w] & 1)) ? T.data[0][src * 512 + w] : 0.0f;
                        }
                if (std::memcmp(&acc, &T.data[5][c * 512 + o], 4) != 0) rule = false;
            }
        }
        CHECK(rule, "loadGhostBlock_nnstar_edge_corner_rule");
    }

    int st = sgb_check_device_errors(grid.handle(), nullptr);
    CHECK(st == SGB_OK, "device_error_word_clear");
    std::printf("%s: %d failure(s)\n", g_fail ? "FAILED" : "PASSED", g_fail);
    return g_fail ? 1 : 0;
}
