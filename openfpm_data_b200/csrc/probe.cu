// Self-check of the bounded waits (failure detection without a GPU fault).
//
// Every wait in the library's kernels is bounded: on an mbarrier phase
// (mbar_wait_bounded) and on the grid barrier of the one-launch multi-step
// kernel (an arrival counter watched against the global timer).  When the
// limit passes, the kernel raises kErrWaitTimeout in the grid's error word
// and returns, and the host reports SGB_ETIMEOUT with the context intact.
// This entry point runs both kinds of wait on conditions that nothing ever
// satisfies (an mbarrier phase with no arrivals, a counter nobody
// increments), each with a short limit, so a test can see that path work.
#include "common.cuh"
#include "internal.h"

namespace sgb {

__global__ void k_probe_waits(uint64_t limit_ns, unsigned* err, unsigned* counter) {
    __shared__ uint64_t bar;
    if (threadIdx.x != 0) return;
    mbar_init(&bar, 1);
    mbar_fence_init();
    // phase 0 never completes: nobody arrives
    mbar_wait_bounded(&bar, 0, err, limit_ns);
    // the counter stays 0: nobody increments it
    const uint64_t t0 = global_timer_ns();
    for (uint32_t it = 0;; ++it) {
        if (*reinterpret_cast<volatile unsigned*>(counter) >= 1u) break;
        if ((it & 63u) == 63u && global_timer_ns() - t0 > limit_ns) {
            atomicOr(err, kErrWaitTimeout);
            break;
        }
    }
}

}  // namespace sgb

using namespace sgb;

extern "C" int sgb_probe_bounded_waits(int64_t limit_ns, int device, sgb_stream stream) {
    if (limit_ns <= 0 || limit_ns > 1000000000ll) return SGB_EINVAL;
    DeviceGuard dg(device);
    SGB_CUDA(dg.status);
    cudaStream_t s = (cudaStream_t)stream;
    unsigned* d = nullptr;
    SGB_CUDA(cudaMalloc(&d, 8));
    unsigned h[2] = {0, 0};
    cudaError_t e = cudaMemsetAsync(d, 0, 8, s);
    if (e == cudaSuccess) {
        k_probe_waits<<<1, 32, 0, s>>>((uint64_t)limit_ns, d, d + 1);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, d, 8, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(d);
    if (e != cudaSuccess) return cuda_status(e, "sgb_probe_bounded_waits");
    if (h[0] & kErrWaitTimeout) {
        set_error("a bounded wait gave up (as this probe intends)");
        return SGB_ETIMEOUT;
    }
    return SGB_OK;
}
