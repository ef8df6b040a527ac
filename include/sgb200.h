/*
 * sgb200.h -- C ABI of the B200-native SparseGridGpu hot path.
 *
 * A drop-in for openfpm_data's sparse block grid pipeline (insert -> flush into
 * the block map -> findNeighbours / tagBoundaries -> applyStencils over chunks
 * with one-point halos).  Every entry point takes plain pointers and sizes,
 * returns an sgb_status, and runs on the CUDA stream it is given (NULL = the
 * legacy default stream).  Device pointers are marked "dev", host pointers
 * "host".  Handles are not thread safe; one handle is used by one host thread
 * at a time.
 *
 * Devices: a grid lives on the device it was created for.  The entry points
 * that take a device or only free or look up memory (sgb_create,
 * sgb_destroy, sgb_release_scratch, sgb_batch_create, sgb_batch_destroy,
 * sgb_existing_offsets_noalloc, sgb_probe_bounded_waits) switch to that
 * device themselves and give the caller's current device back before they
 * return; every other entry point runs on the calling thread's current
 * device, which must be the grid's (as every call of the reference runs on
 * the current device).
 *
 * Block-map layout (identical to the reference's memory_traits_inte layout):
 *   index[n]                int64 chunk ids, sorted ascending
 *   data_p[(n+1) * bs]      one array per property, chunk major; position n
 *                           holds the background chunk
 *   mask[(n+1) * bs]        uint8 per point: bit0 EXIST, bit1 PADDING
 * with bs = edge^dim points per chunk and the point at local coordinates
 * (x,y,z) of a chunk at offset x + edge*(y + edge*z).
 *
 * Citations name the reference interface each entry point replaces (paths
 * inside the openfpm_data project).
 */
#ifndef SGB200_H
#define SGB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct sgb_grid sgb_grid;
typedef struct sgb_batch sgb_batch;
typedef void* sgb_stream; /* cudaStream_t */

typedef enum {
    SGB_OK = 0,
    SGB_EINVAL = 1,   /* bad argument */
    SGB_ECUDA = 2,    /* CUDA runtime error (see sgb_last_error_string) */
    SGB_ENOMEM = 3,   /* device allocation failed */
    SGB_ERANGE = 4,   /* a point lies outside the grid domain */
    SGB_ESTATE = 5,   /* call not valid in the current state */
    SGB_ETIMEOUT = 6, /* a device-side bounded wait gave up */
    SGB_ENOTSUP = 7   /* configuration not supported by this build */
} sgb_status;

typedef enum { SGB_F32 = 0, SGB_I32 = 1, SGB_F64 = 2, SGB_U8 = 3 } sgb_type;

/* Flush reduction operators: sRight_, sLeft_, sadd_, smax_, smin_,
 * sBitwiseOr_ (src/Vector/cuda/map_vector_sparse_cuda_kernels.cuh:51-352).
 * SGB_OP_NONE leaves the property out of the flush. */
typedef enum {
    SGB_OP_NONE = 0,
    SGB_OP_RIGHT = 1,
    SGB_OP_LEFT = 2,
    SGB_OP_ADD = 3,
    SGB_OP_MAX = 4,
    SGB_OP_MIN = 5,
    SGB_OP_OR = 6
} sgb_op;

/* Neighbourhoods: NNStar (faces) and NNFull (3^dim box)
 * (src/SparseGridGpu/SparseGridGpu_ker_util.hpp:86-167,
 *  src/SparseGridGpu/SparseGridGpu.hpp:261-360). */
typedef enum { SGB_NN_STAR = 0, SGB_NN_FULL = 1 } sgb_nn;

/* Fixed-function stencils.
 *  SGB_HEAT7 : HeatStencil<3,src,dst> (src/SparseGridGpu/tests/utils/
 *              SparseGridGpu_util_test.cuh:201-345); params {dt}; writes the
 *              whole destination chunk.
 *  SGB_GS7   : Gray-Scott written as a conv2_b user function
 *              (src/SparseGridGpu/SparseGridGpu.hpp:2627-2645); src {u,v},
 *              dst {u',v'}, params {Du, Dv, F, k, dt}; writes active points.
 *  SGB_BOX27 : Conv3x3x3<3,src,dst> (src/SparseGridGpu/tests/
 *              SparseGridGpu_tests.cu:887-952); params = 27 coefficients
 *              c[i][j][k], i along x; writes active points; NNFull halo.
 *  SGB_BOX27_NS : Conv3x3x3_noshared<3,src,dst> applied in
 *              STENCIL_MODE_INPLACE_NO_SHARED (SparseGridGpu_tests.cu:955-1010,
 *              SparseGridGpu.hpp:1051-1075): one thread per existing point
 *              of the existing-point list, neighbours read point by point
 *              through the NNFull table; params = 27 coefficients c[i][j][k],
 *              i along z; writes active points. */
typedef enum { SGB_HEAT7 = 0, SGB_GS7 = 1, SGB_BOX27 = 2, SGB_BOX27_NS = 3 } sgb_stencil;

const char* sgb_status_string(int status);
const char* sgb_last_error_string(void);
int sgb_version(void);

/* ---------------------------------------------------------------- grids */

/* SparseGridGpu(const size_t (&res)[dim], stencilSupportRadius = 1)
 * (src/SparseGridGpu/SparseGridGpu.hpp:1694-1698).  dim == 3, edge 4 or 8,
 * at most 8 properties. */
int sgb_create(sgb_grid** out, int dim, int edge, const int64_t* size, int nprop, const int* prop_types,
               int device);
int sgb_destroy(sgb_grid* g);

/* Chunk-id linearizer: SGB_LIN_SMB, grid_smb (block x fastest, the
 * default), or SGB_LIN_ZMB, grid_zmb (3-D Morton code of the block
 * coordinate, SparseGridGpu_z, src/Grid/Geometry/grid_zmb.hpp:25-104,
 * src/SparseGridGpu/SparseGridGpu.hpp:3948-3960); offsets inside a chunk
 * are x fastest for both.  Chosen while the grid is empty; SGB_LIN_ZMB needs
 * 3-D and at most 2^21 blocks per dimension.  Stencils on Morton grids run
 * the one-chunk-per-CTA kernel; batches and the scene builder take
 * SGB_LIN_SMB grids only. */
typedef enum { SGB_LIN_SMB = 0, SGB_LIN_ZMB = 1 } sgb_linearizer;
int sgb_set_linearizer(sgb_grid* g, int kind);

/* removeUnusedBuffers (SparseGridGpu.hpp:3739-3742): free the grid's
 * temporary device buffers (flush and scan scratch, the second buffer set,
 * existence bitmaps, the existing-point list; the staged inserts when none
 * are pending).  They are allocated again when needed.  Synchronises the
 * device. */
int sgb_release_scratch(sgb_grid* g);

/* Self-check of failure detection (no reference counterpart): runs the
 * library's two kinds of bounded wait -- on an mbarrier phase and on an
 * arrival counter -- on conditions nothing satisfies, with a limit of
 * limit_ns (at most 1 s).  Returns SGB_ETIMEOUT when both gave up as they
 * should, with the device still usable. */
int sgb_probe_bounded_waits(int64_t limit_ns, int device, sgb_stream s);

/* Tell the grid that a user kernel may have changed which points exist
 * (device-side remove through the view): the cached existence bitmaps and
 * existing-point list are rebuilt when next needed.  A kernel that clears a
 * mask byte must also store the properties' backgrounds at that point (the
 * C++ header's device remove does). */
int sgb_existence_changed(sgb_grid* g);

/* setBackgroundValue<p> (SparseGridGpu.hpp:2878-2884); value host. */
int sgb_set_background(sgb_grid* g, int prop, const void* value_host);

/* Device-side insert<p>(coord) for a batch of points
 * (src/SparseGridGpu/SparseGridGpu_ker.cuh:446-450 ->
 *  src/Vector/cuda/map_vector_sparse_cuda_ker.cuh:309-318).
 * coords dev int32 [n][3]; values[p] dev, one array of n elements per
 * property (NULL entries leave that property out).  Points are staged in
 * insertion order until sgb_flush. */
int sgb_insert(sgb_grid* g, int64_t n, const int32_t* coords_dev, const void* const* values_dev, sgb_stream s);

/* The same with linearised point ids (grid_smb::LinId,
 * src/Grid/Geometry/grid_smb.hpp:176-190): BlockMapGpu::insert<p>(linId)
 * (src/SparseGridGpu/BlockMapGpu.hpp:137-150). */
int sgb_insert_lin(sgb_grid* g, int64_t n, const int64_t* lin_dev, const void* const* values_dev, sgb_stream s);

/* Stage the contents of per-CTA insert pools written by a user kernel
 * (setGPUInsertBuffer(nBlock, nSlot) + insert<p> + flush_block_insert,
 * src/Vector/map_vector_sparse.hpp:1883-1890,
 * src/Vector/cuda/map_vector_sparse_cuda_ker.cuh:309-318, 424-439; compacted
 * pool after pool like make_continuos, map_vector_sparse.hpp:880-946).
 * counts_dev int32[npools]; lin_dev int64[npools*nslot] linearised point
 * ids; values_dev[p] [npools*nslot] per property (NULL: background).  A
 * count above nslot (a pool that overflowed) makes the next sgb_flush fail
 * with SGB_ERANGE and drop the staged points. */
int sgb_insert_pools(sgb_grid* g, int64_t npools, int64_t nslot, const int32_t* counts_dev, const int64_t* lin_dev,
                     const void* const* values_dev, sgb_stream s);

/* Stage the chunk slots written by a user kernel through insertBlock
 * (src/SparseGridGpu/BlockMapGpu_ker.cuh:199-227: each call takes one whole
 * chunk slot of its CTA's insert buffer and the CTA writes any of its points,
 * setting their EXIST mask bits).  npools pools of nslot chunk slots:
 * counts_dev[b] = slots used by pool b; keys_dev[b*nslot+k] = the slot's chunk
 * id; values_dev[p] = [npools*nslot*bs] elements of property p (NULL entries
 * leave the property out); masks_dev = [npools*nslot*bs] mask bytes.  Every
 * slot point whose mask has EXIST set is staged as an insert, in (pool, slot,
 * offset) order, until sgb_flush, which reduces duplicates in that order as
 * the reference reduces its chunk slots.  A count above nslot makes the next
 * sgb_flush fail with SGB_ERANGE. */
int sgb_insert_blocks(sgb_grid* g, int64_t npools, int64_t nslot, const int32_t* counts_dev, const int64_t* keys_dev,
                      const void* const* values_dev, const uint8_t* masks_dev, sgb_stream s);

/* Device view of a grid for user kernels (SparseGridGpu::toKernelNN,
 * SparseGridGpu.hpp:1749-1789): block map pointers and the neighbour table
 * of nn_kind (int32, -1 absent), valid until the next flush or map upload.
 * Points whose mask byte is 0 hold the background value. */
typedef struct {
    int64_t n;
    int edge, bs, nprop, nn_kind;
    int64_t size[3], bsz[3];
    const int64_t* keys;
    void* data[8];
    const uint8_t* mask;
    const int32_t* nn;
    int zorder; /* chunk ids: 0 grid_smb (x fastest), 1 grid_zmb (Morton) */
} sgb_view;
int sgb_get_view(sgb_grid* g, int nn_kind, sgb_view* out, sgb_stream s);

/* flush<v_reduce...>(ctx, FLUSH_ON_DEVICE) (SparseGridGpu.hpp:772-779,
 * BlockMapGpu.hpp:289-299, src/Vector/map_vector_sparse.hpp:1784-1795).
 * ops[nprop]: one sgb_op per property.  Duplicates of one point are reduced
 * in insertion order, A = first, A = op(A, next); a point that already
 * exists is then reduced as op(A, old); masks are OR-ed. */
int sgb_flush(sgb_grid* g, const int* ops_host, sgb_stream s);

/* findNeighbours<NN>() (SparseGridGpu.hpp:2396-2420). */
int sgb_find_neighbours(sgb_grid* g, int nn, sgb_stream s);

/* Neighbour table in the reference's nn_blocks format (host int64
 * [n][nNN], nNN = 8 for NNStar, 27 for NNFull): data position of the
 * neighbour chunk, n when it is absent, -1 in the unused NNStar slots. */
int sgb_neighbour_table(sgb_grid* g, int nn, int64_t* out_host, sgb_stream s);

/* tagBoundaries<NN>(ctx) (SparseGridGpu.hpp:2290-2394). */
int sgb_tag_boundaries(sgb_grid* g, int nn, sgb_stream s);

/* applyStencils<S>(box, STENCIL_MODE_INPLACE, args...)
 * (SparseGridGpu.hpp:2704-2734, 954-1048).  src/dst host arrays of property
 * ids (1 entry for HEAT7/BOX27, 2 for GS7); params host floats; box host
 * int64 {lo[3], hi[3]} inclusive, or NULL for the whole grid. */
int sgb_apply_stencil(sgb_grid* g, int kind, const int* src, const int* dst, const float* params, int nparams,
                      const int64_t* box, sgb_stream s);

/* nsteps stencil applications alternating src->dst and dst->src (the
 * reference's ping-pong loop, src/SparseGridGpu/tests/
 * SparseGridGpu_tests.cu:499-503), launched as one captured CUDA graph.
 * On return *final_is_dst is 1 when the last step wrote the dst properties. */
int sgb_run_steps(sgb_grid* g, int kind, const int* src, const int* dst, const float* params, int nparams,
                  int nsteps, int use_graph, int* final_is_dst, sgb_stream s);

/* Number of chunks (private_get_index_array().size()). */
int sgb_nchunks(const sgb_grid* g, int64_t* n);

/* Non-owning device views (private_get_index_array / private_get_data_array,
 * SparseGridGpu.hpp:1959-1990).  Invalidated by sgb_flush. */
int sgb_index_buffer(sgb_grid* g, const int64_t** dev);
int sgb_data_buffer(sgb_grid* g, int prop, void** dev);
int sgb_mask_buffer(sgb_grid* g, uint8_t** dev);

/* Build the block map directly from host arrays (hostToDevice of a map laid
 * out as above, without the background chunk), replacing the current one.
 * A NULL data_host[p] fills property p with its background value. */
int sgb_load_map(sgb_grid* g, int64_t n, const int64_t* keys_host, const void* const* data_host,
                 const uint8_t* mask_host, sgb_stream s);

/* The same from device arrays. */
int sgb_load_map_dev(sgb_grid* g, int64_t n, const int64_t* keys_dev, const void* const* data_dev,
                     const uint8_t* mask_dev, sgb_stream s);

/* deviceToHost: copy keys[n], data_p[(n+1)*bs] and mask[(n+1)*bs] to host
 * (any pointer may be NULL to skip it). */
int sgb_download_map(sgb_grid* g, int64_t* keys_host, void* const* data_host, uint8_t* mask_host, sgb_stream s);

/* remove(box) for each box, then removePoints (SparseGridGpu.hpp:3417-3489,
 * 3528-3531): every existing point inside one of the boxes loses its mask
 * byte (EXIST and PADDING); chunks are kept.  boxes_host: nboxes x {lo[3],
 * hi[3]}, inclusive, tested as unsigned int like the reference's
 * Box<dim, unsigned int> (a negative lower corner matches nothing).  3-D
 * grids; synchronises the stream. */
int sgb_remove_boxes(sgb_grid* g, int64_t nboxes, const int64_t* boxes_host, sgb_stream s);

/* The coordinates of the existing points, in (chunk position, offset in the
 * chunk) order: the points the reference's getIterator() / sub-iterator
 * (src/SparseGridGpu/Iterators/SparseGridGpu_iterator.hpp:17-304) visit.
 * box_host: NULL or {lo[3], hi[3]} inclusive.  *count receives the number of
 * points; coords_dev (int32 [3 * capacity]) is written when capacity >=
 * *count, so a first call with capacity 0 sizes the buffer.  3-D grids. */
int sgb_existing_points(sgb_grid* g, const int64_t* box_host, int32_t* coords_dev, int64_t capacity,
                        int64_t* count, sgb_stream s);

/* Packing of sub-boxes for ghost exchange, in the reference's packed-box
 * format (packRequest + packCalculate, pack + packFinalize, unpack:
 * SparseGridGpu.hpp:3041-3210, 3244-3370, 1420-1615, 3665-3750).  One packed
 * box, every section padded to 8 bytes:
 *   uint64 n_cnk; int32 start[3] (box lower corner); int32 size[3] (grid size);
 *   int64 chunk_id[n_cnk]; uint32 scan[n_cnk + 1] (scan[n_cnk] = n_pnt);
 *   per packed property in the given order: n_pnt elements of its type;
 *   int16 offset[n_pnt] (offset in the chunk); uint8 mask[n_pnt].
 * A reference property of array type T[N] is N consecutive properties here,
 * whose blocks sit back to back like the reference's component-major block.
 * Packed points are the existing points inside the inclusive box, chunks in
 * index order; inside a chunk the points are in offset order (the reference
 * writes them in atomic-counter order, any order).  3-D grids; each call
 * synchronises the stream.
 *
 * sgb_pack_request: bytes_host[k] = size of box k packed with props. */
int sgb_pack_request(sgb_grid* g, int64_t nboxes, const int64_t* boxes_host, int nprops, const int* props,
                     int64_t* bytes_host, sgb_stream s);

/* Pack the boxes back to back into out_dev (8-byte aligned, capacity bytes;
 * SGB_ERANGE if smaller than the summed request).  Padding bytes are zero. */
int sgb_pack(sgb_grid* g, int64_t nboxes, const int64_t* boxes_host, int nprops, const int* props, void* out_dev,
             int64_t capacity, int64_t* bytes_written, sgb_stream s);

/* unpack of ONE packed box at buf_dev (8-byte aligned, nbytes readable):
 * stages its points as inserts at packed coordinate - packed start +
 * start_host (start_host NULL: at the packed coordinate), with the packed
 * values for props (the properties the box was packed with, same order) and
 * the background for the others.  *consumed = the box's size, the offset of
 * the next box.  The packing grid must have this grid's chunk edge.  Points
 * that land outside the domain fail the next flush like out-of-domain
 * inserts.  removeAddUnpackFinalize<prp...> is sgb_flush with SGB_OP_RIGHT
 * for the unpacked properties and SGB_OP_NONE for the others; sgb_remove_boxes
 * before the unpacks plays the queued remove(box). */
int sgb_unpack(sgb_grid* g, const void* buf_dev, int64_t nbytes, int nprops, const int* props,
               const int64_t* start_host, int64_t* consumed, sgb_stream s);

/* sgb_unpack of nboxes consecutive packed boxes in one call (no reference
 * counterpart: the reference unpacks box by box, reading each header on the
 * host).  The headers are walked on the device, so the call synchronises
 * the stream once instead of twice per box.  starts_host: nboxes x 3
 * destination corners, or NULL (points at their packed coordinates).
 * *consumed = bytes of the nboxes boxes. */
int sgb_unpack_boxes(sgb_grid* g, const void* buf_dev, int64_t nbytes, int nprops, const int* props, int64_t nboxes,
                     const int64_t* starts_host, int64_t* consumed, sgb_stream s);

/* The existing-point list of tagBoundaries(..., CALCULATE_EXISTING_POINTS)
 * (SparseGridGpu.hpp:2354-2387): every existing point as uint32 chunk
 * position * chunk size + offset, in (chunk position, offset) order (the
 * reference's order inside a chunk is arbitrary).  Built on demand and kept
 * until existence changes; SGB_BOX27_NS builds it itself.  Grids of at most
 * 2^32 chunk points.  *count may be NULL. */
int sgb_calc_existing_points(sgb_grid* g, int64_t* count, sgb_stream s);

/* The same list's device array (valid until existence changes) and length. */
int sgb_existing_point_list(sgb_grid* g, const uint32_t** ids_dev, int64_t* count, sgb_stream s);

/* Links between the levels of a multi-resolution hierarchy
 * (construct_link_dw / construct_link_up, SparseGridGpu.hpp:2113-2262;
 * kernels SparseGridGpu_kernels.cuh:775-1000).  The padding points (mask
 * bit 1) of g inside the inclusive box {lo[3], hi[3]} are listed in (chunk
 * position, offset) order; a padding point at p links
 *   down: to the existing points of grid_dw at 2p + p_dw + (j & 1,
 *         (j >> 1) & 1, (j >> 2) & 1), j = 0 .. 5 (the reference's loop
 *         bound 2*dim: the children (0,1,1) and (1,1,1) are not visited);
 *   up:   to the existing point of grid_up at (p - p_up) / 2, truncating.
 * The other grid is addressed as the reference's device get does
 * (grid_smb::LinId without bounds checks, cast to unsigned int).  Both
 * grids share the chunk edge and the device; each call replaces g's links of
 * that direction and synchronises the stream. */
int sgb_construct_link_dw(sgb_grid* g, const sgb_grid* grid_dw, const int64_t* box_host, const int64_t* p_dw_host,
                          sgb_stream s);
int sgb_construct_link_up(sgb_grid* g, const sgb_grid* grid_up, const int64_t* box_host, const int64_t* p_up_host,
                          sgb_stream s);

/* The links of one direction (up = 0 down, 1 up): getDownLinks /
 * getDownLinksOffsets / getUpLinks / getUpLinksOffsets.  Device arrays valid
 * until the next construct call: the padding points (pad_pos chunk
 * position, pad_off offset), offsets[npad + 1] (first link of each padding
 * point, nlinks last) and the links (link_pos chunk position in the other
 * grid, link_off offset; only existing points are linked). */
typedef struct {
    int64_t npad;
    const int32_t* pad_pos;
    const int16_t* pad_off;
    const uint32_t* offsets;
    int64_t nlinks;
    const int32_t* link_pos;
    const int16_t* link_off;
} sgb_links;
int sgb_get_links(sgb_grid* g, int up, sgb_links* out);

/* countExistingElements / countBoundaryElements (SparseGridGpu.hpp:2422-2474). */
int sgb_count_existing(sgb_grid* g, int64_t* existing, int64_t* padding, sgb_stream s);

/* Per-chunk offsets of the existing points: offsets_dev[i] = number of EXIST
 * points in chunks 0..i-1, offsets_dev[n] = total (int64, n + 1 entries).
 * The calc_exist_points + scan step of tagBoundaries(...,
 * CALCULATE_EXISTING_POINTS) (SparseGridGpu.hpp:2355-2387,
 * SparseGridGpu_kernels.cuh:1194-1225).  Grids of 2^32 or more chunk points
 * (chunks x edge^3) are rejected with SGB_ERANGE: the counts are scanned in
 * 32-bit words. */
int sgb_existing_offsets(sgb_grid* g, int64_t* offsets_dev, sgb_stream s);

/* The same offsets without allocating device memory (no counterpart in the
 * reference).  For callers that may not allocate: applications whose device
 * memory belongs to their own pool allocator, and loops that may not call
 * cudaMalloc because it can synchronise the device.  The scan scratch is a
 * fixed file-scope device array (4 KiB, kept by every GPU that loads the
 * library until exit), so grids of more than 1,048,576 chunks are rejected
 * with SGB_ERANGE.  The first call on a device looks up that array's device
 * address; make that first call before any stream capture.  All calls share
 * the array: calls that overlap on the GPU race on it. */
int sgb_existing_offsets_noalloc(const sgb_grid* g, int64_t* offsets_dev, sgb_stream s);

/* get<p>(coord) for a batch of points (SparseGridGpu_ker.cuh:409-413):
 * value if the point exists, background otherwise.  coords dev int32 [n][3],
 * out dev n elements of the property's type. */
int sgb_get(sgb_grid* g, int64_t n, const int32_t* coords_dev, int prop, void* out_dev, sgb_stream s);

/* Scene builder (no reference counterpart; reference users insert points
 * from their own kernels): replace the block map by the union of nballs
 * balls (host float [nballs][4] = cx, cy, cz, r; a point exists when
 * |p - c|^2 <= r^2), and fill the listed properties (host ids):
 *   init 0 (SGB_INIT_UNIFORM):    props[0] = U[0,1) from a hash of (seed, point id)
 *   init 1 (SGB_INIT_GRAY_SCOTT): props[0] = u = 1, props[1] = v = 0, except
 *        in the 6^3 cube [floor(c)-3, floor(c)+3) of every ball centre:
 *        u = 0.5(1 + 0.01a), v = 0.25(1 + 0.01b), a, b ~ U[-1,1)
 * Every other property is set to its background.  At most 64 balls. */
int sgb_build_balls(sgb_grid* g, int nballs, const float* balls_host, int init, uint64_t seed, const int* props,
                    sgb_stream s);

/* Device-side error word of the last kernels (bounded waits that gave up,
 * out-of-domain inserts).  Synchronises the stream; clears the word. */
int sgb_check_device_errors(sgb_grid* g, sgb_stream s);

/* Bytes of device memory held by the grid. */
int sgb_device_bytes(const sgb_grid* g, int64_t* bytes);

/* Stencil launch configuration of the 8^3 kernel: CTAs per SM (1..16, two
 * warps each, every warp its own pipeline; -1 for the automatic choice per
 * stencil kind, the default) and the staging ring depth per warp (3..16
 * chunks, at most what fits in one CTA's shared memory, or -1 for the
 * automatic depth: the deepest ring, up to 8, with which the CTAs per SM stay
 * resident; the default); 0 keeps the current value. */
int sgb_set_launch_config(sgb_grid* g, int ctas_per_sm, int stages);

/* ---------------------------------------------------------------- batches
 * Many independent grids advanced by one persistent launch per step over
 * their concatenated block maps (no reference counterpart: the reference
 * launches one applyStencils per grid).  All member grids share dim, edge,
 * property types and stencil kind; each keeps its own parameters and
 * background values. */
int sgb_batch_create(sgb_batch** out, int device);
int sgb_batch_destroy(sgb_batch* b);
/* Copy a grid's block map and its src/dst properties into the batch; the
 * grid will take part in the next `nsteps` batch steps (ping-pong src->dst,
 * dst->src, ...) and then stay idle.  params as for sgb_apply_stencil
 * (HEAT7 or GS7, no box).  Returns the slot id. */
int sgb_batch_add(sgb_batch* b, sgb_grid* g, int kind, const int* src, const int* dst, const float* params,
                  int nparams, int64_t nsteps, int* slot, sgb_stream s);
/* Drop a slot; its chunks are compacted away before the next step. */
int sgb_batch_remove(sgb_batch* b, int slot, sgb_stream s);
/* Advance the batch by nsteps global steps: one persistent launch per step
 * over all chunks, captured as one CUDA graph when use_graph != 0.  The batch
 * keeps the instantiated graph and updates it in place on the next call with
 * the same nsteps.  The call returns without waiting for the GPU: the steps
 * run on stream s in order with the batch's other calls on that stream. */
int sgb_batch_step(sgb_batch* b, int nsteps, int use_graph, sgb_stream s);
/* Steps a slot has done so far (<= its nsteps). */
int sgb_batch_slot_steps(const sgb_batch* b, int slot, int64_t* done);
/* Copy a slot's fields back into g's src/dst properties (g must have the
 * block map the slot was added from); *final_is_dst as in sgb_run_steps. */
int sgb_batch_extract(sgb_batch* b, int slot, sgb_grid* g, int* final_is_dst, sgb_stream s);
/* Copy a slot's block map and current fields to host memory (any pointer may
 * be NULL): keys[n], mask[n*bs], fields[j][n*bs] for the np source fields,
 * holding the state after the steps the slot has done. */
int sgb_batch_read(sgb_batch* b, int slot, int64_t* keys_host, uint8_t* mask_host, float* const* fields_host,
                   int64_t* nchunks, sgb_stream s);
/* sgb_batch_read without the host wait (no reference counterpart; for a
 * serving loop that keeps the GPU busy): the copies are queued on stream s,
 * in order with the batch's steps; the host buffers (pinned for an
 * asynchronous copy) hold the slot's state once the stream has reached them.
 * A removed slot's data stays in place until a later call compacts the batch
 * on the same stream, so a read queued before that compaction is safe. */
int sgb_batch_read_async(sgb_batch* b, int slot, int64_t* keys_host, uint8_t* mask_host, float* const* fields_host,
                         int64_t* nchunks, sgb_stream s);
int sgb_batch_info(const sgb_batch* b, int* ngrids, int64_t* nchunks, int64_t* bytes);
/* Launch configuration of the batched kernels (as sgb_set_launch_config). */
int sgb_batch_set_launch_config(sgb_batch* b, int ctas_per_sm, int stages);

#ifdef __cplusplus
}
#endif

#endif /* SGB200_H */
