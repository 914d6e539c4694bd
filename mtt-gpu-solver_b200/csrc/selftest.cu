// selftest.cu — a self-check of the bounded device waits.
//
// Every kernel that waits on an mbarrier (the terminal groups, the table
// staging of the evaluator, the GEMM pipelines) gives up after a poll limit or
// a wall-time limit, records an error word and returns, and the host turns the
// word into MTT_ERR_TIMEOUT.  This entry point exercises that path on its own:
// one CTA waits on an mbarrier that no copy targets.  When `arrive` is zero
// nothing arrives on it, so the wait runs out after `limit_us` microseconds;
// when it is non-zero one thread arrives first and the wait completes.  No
// copy is ever in flight, so a wait that gives up leaves nothing behind and the
// context stays usable.
#include "mtt_bulk.cuh"
#include "mtt_common.h"

namespace mtt {

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// The bounded wait of mtt_bulk.cuh with the wall-time limit as an argument.
__device__ __forceinline__ bool mbar_wait_limited(uint64_t* bar, uint32_t parity, uint64_t limit_ns) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = globaltimer_ns();
    for (uint32_t i = 0; i < MTT_WAIT_LIMIT; ++i) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((i & 63u) == 63u && globaltimer_ns() - t0 > limit_ns) return false;
    }
    return false;
}

__global__ void k_selftest_wait(int arrive, uint64_t limit_ns, int* err) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        mbar_fence_init();
    }
    __syncthreads();
    if (arrive && threadIdx.x == 0) mbar_arrive(&bar);
    const bool ok = mbar_wait_limited(&bar, 0u, limit_ns);
    if (__syncthreads_or(!ok) && threadIdx.x == 0) atomicOr(err, 1);
}

}  // namespace mtt

using namespace mtt;

extern "C" int mtt_selftest_bounded_wait(int32_t arrive, int32_t limit_us, void* stream) {
    if (limit_us < 1 || limit_us > 2000000) return MTT_ERR_INVALID;
    cudaStream_t st = as_stream(stream);
    int* d_err = nullptr;
    MTT_TRY_CUDA(cudaMallocAsync(&d_err, sizeof(int), st));
    int s = cuda_status(cudaMemsetAsync(d_err, 0, sizeof(int), st));
    if (!s) {
        k_selftest_wait<<<1, 32, 0, st>>>(arrive ? 1 : 0, 1000ull * (uint64_t)limit_us, d_err);
        s = cuda_status(cudaGetLastError());
    }
    int h_err = 0;
    if (!s) s = cuda_status(cudaMemcpyAsync(&h_err, d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    if (!s) s = cuda_status(cudaStreamSynchronize(st));
    cudaFreeAsync(d_err, st);
    if (!s && h_err) s = MTT_ERR_TIMEOUT;
    return s;
}
