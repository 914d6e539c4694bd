// capi.cpp — status strings, version and the per-thread CUDA error slot.
#include "mtt_common.h"

namespace mtt {
thread_local int g_last_cuda_error = 0;
}

extern "C" const char* mtt_status_string(int status) {
    switch (status) {
        case MTT_OK: return "ok";
        case MTT_ERR_INVALID: return "invalid argument";
        case MTT_ERR_CUDA: return "CUDA error";
        case MTT_ERR_NOMEM: return "out of memory";
        case MTT_ERR_TIMEOUT: return "bounded device wait timed out";
        case MTT_ERR_IO: return "file missing, short or malformed";
        case MTT_ERR_UNSUPPORTED: return "unsupported size or feature";
        default: return "unknown status";
    }
}

extern "C" int mtt_last_cuda_error(void) { return mtt::g_last_cuda_error; }

extern "C" const char* mtt_version(void) { return "mtt-b200 0.1.0 (sm_100a)"; }
