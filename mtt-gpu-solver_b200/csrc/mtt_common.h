// mtt_common.h — host-side status handling shared by the C ABI sources.
#pragma once
#include <cuda_runtime.h>
#include "../../include/mtt_b200.h"

namespace mtt {

// cudaError_t of the last failing CUDA call made by this host thread.
extern thread_local int g_last_cuda_error;

inline int cuda_status(cudaError_t e) {
    if (e == cudaSuccess) return MTT_OK;
    g_last_cuda_error = (int)e;
    return e == cudaErrorMemoryAllocation ? MTT_ERR_NOMEM : MTT_ERR_CUDA;
}

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

inline int ceil_div(int a, int b) { return (a + b - 1) / b; }
inline long long ceil_div_ll(long long a, long long b) { return (a + b - 1) / b; }

}  // namespace mtt

#define MTT_TRY_CUDA(call)                                            \
    do {                                                              \
        int _mtt_s = ::mtt::cuda_status(call);                        \
        if (_mtt_s != MTT_OK) return _mtt_s;                          \
    } while (0)

#define MTT_TRY(call)                                                 \
    do {                                                              \
        int _mtt_s = (call);                                          \
        if (_mtt_s != MTT_OK) return _mtt_s;                          \
    } while (0)

// A launch's own error (bad configuration) surfaces right away.
#define MTT_CHECK_LAUNCH() MTT_TRY_CUDA(cudaGetLastError())
