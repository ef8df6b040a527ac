// Stencil arithmetic and launch description shared by the single-grid and
// the batched entry points.
#pragma once

#include <cuda_runtime.h>

#include "common.cuh"
#include "internal.h"

namespace sgb {

__device__ __forceinline__ bool in_box(const StencilParams& prm, int64_t cx, int64_t cy, int64_t cz) {
    return cx >= prm.box_lo[0] && cx <= prm.box_hi[0] && cy >= prm.box_lo[1] && cy <= prm.box_hi[1] &&
           cz >= prm.box_lo[2] && cz <= prm.box_hi[2];
}

// HeatStencil's Laplacian (src/SparseGridGpu/tests/utils/SparseGridGpu_util_test.cuh:256-274) as
// nvcc compiles that source:
//   ScalarT laplacian = -2.0 * dim * cur;           // a double product, narrowed to float
//   laplacian += neighbourMinus + neighbourPlus;    // per dimension, x first
//   res = cur + dt * laplacian;
// -6 * cur is exact in double, so its narrowing equals a float multiply, which nvcc's default FMA
// contraction fuses with the first add: lap = fma(-6, cur, xm + xp), then + (ym + yp), + (zm + zp),
// and res = fma(dt, lap, cur).  (The drop-in test compiles the reference's functor and checks this
// rounding point by point.)
__device__ __forceinline__ float lap7_heat(float c, float xm, float xp, float ym, float yp, float zm, float zp) {
    float lap = __fmaf_rn(-6.0f, c, __fadd_rn(xm, xp));
    lap = __fadd_rn(lap, __fadd_rn(ym, yp));
    return __fadd_rn(lap, __fadd_rn(zm, zp));
}

__device__ __forceinline__ float heat_update(float cur, float xm, float xp, float ym, float yp, float zm, float zp,
                                             float dt) {
    return __fmaf_rn(dt, lap7_heat(cur, xm, xp, ym, yp, zm, zp), cur);
}

// 7-point Laplacian of the Gray-Scott update (the oracle's conv2_b definition): -6 c rounded on its own,
// then the neighbour pairs in HeatStencil's order.
__device__ __forceinline__ float lap7(float c, float xm, float xp, float ym, float yp, float zm, float zp) {
    float lap = __fmul_rn(-6.0f, c);
    lap = __fadd_rn(lap, __fadd_rn(xm, xp));
    lap = __fadd_rn(lap, __fadd_rn(ym, yp));
    return __fadd_rn(lap, __fadd_rn(zm, zp));
}

template <int KIND>
__device__ __forceinline__ float lap7k(float c, float xm, float xp, float ym, float yp, float zm, float zp) {
    return KIND == SGB_HEAT7 ? lap7_heat(c, xm, xp, ym, yp, zm, zp) : lap7(c, xm, xp, ym, yp, zm, zp);
}

// Gray-Scott as a conv2_b user function:
//   uvv = (u*v)*v
//   u' = u + dt*fma(F, 1-u, fma(Du, lu, -uvv))
//   v' = v + dt*fma(-(F+k), v, fma(Dv, lv, uvv))
__device__ __forceinline__ void gs_update(float u, float v, float lu, float lv, const GridInfo& p, float& un,
                                          float& vn) {
    const float uvv = __fmul_rn(__fmul_rn(u, v), v);
    float du = __fmaf_rn(p.Du, lu, -uvv);
    du = __fmaf_rn(p.F, __fsub_rn(1.0f, u), du);
    float dv = __fmaf_rn(p.Dv, lv, uvv);
    dv = __fmaf_rn(p.nFK, v, dv);
    un = __fmaf_rn(p.dt, du, u);
    vn = __fmaf_rn(p.dt, dv, v);
}

// CTAs per SM of the pipelined 8^3 kernel when the caller leaves it automatic
// (measured on the 512^3 grids: Gray-Scott runs best with 6 two-warp CTAs
// and 3-deep rings resident, heat with 8).
inline int auto_ctas_per_sm(int kind) { return kind == SGB_GS7 ? 6 : 8; }

// Everything one stencil launch needs.
struct LaunchDesc {
    int kind, edge, use_tile, stages, num_sms;
    unsigned ctas;
    FieldSet fs;
    const uint8_t* mask;
    const int32_t* nn;
    const int64_t* keys;
    const int32_t* gid;      // per chunk grid id (NULL: single grid g0)
    const GridInfo* grids;   // per grid entries (NULL: single grid g0)
    GridInfo g0;
    int64_t n;
    int64_t arr_chunks;      // chunks held by the field arrays (n + background chunk for grids)
    Geometry geo;
    StencilParams prm;
    int64_t t;
    unsigned* err;
};

int launch_fields(const LaunchDesc& L, cudaStream_t s);
int launch_e8(const LaunchDesc& L, cudaStream_t s);  // pipelined 8^3 kernel (stencil8.cu)
GridInfo grid_info_of(const StencilParams& prm);

// Capture `body(stream)` into a CUDA graph, launch it on `s`, wait for it.
template <typename F>
int run_graph(F body, cudaStream_t s) {
    cudaStream_t cap;
    SGB_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int st = SGB_OK;
    cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        st = body(cap);
        cudaError_t e2 = cudaStreamEndCapture(cap, &graph);
        if (st == SGB_OK && e2 != cudaSuccess) st = cuda_status(e2, "cudaStreamEndCapture");
    } else {
        st = cuda_status(e, "cudaStreamBeginCapture");
    }
    if (st == SGB_OK) {
        e = cudaGraphInstantiate(&exec, graph, 0);
        if (e != cudaSuccess) st = cuda_status(e, "cudaGraphInstantiate");
    }
    if (st == SGB_OK) {
        e = cudaGraphLaunch(exec, s);
        if (e != cudaSuccess) st = cuda_status(e, "cudaGraphLaunch");
    }
    if (st == SGB_OK) {
        e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) st = cuda_status(e, "cudaStreamSynchronize");
    }
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    cudaStreamDestroy(cap);
    return st;
}

}  // namespace sgb
