// CUDA error bookkeeping of the C ABI: every PE_ERR_CUDA return records the cudaError_t behind it, per
// host thread, so that pe_last_cuda_error() can name it.
#pragma once
#include <cuda_runtime.h>

namespace pe {

// Records e as this thread's last CUDA error and returns PE_ERR_CUDA.
int cuda_fail(cudaError_t e);

// Status of the launches just queued on this thread: PE_OK, or PE_ERR_CUDA with the error recorded.
inline int launch_status() {
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : cuda_fail(e);
}

}  // namespace pe

// Returns from the enclosing function with PE_ERR_CUDA (error recorded) when `call` fails.
#define PE_CUDA_TRY(call)                                            \
    do {                                                             \
        const cudaError_t pe_err_ = (call);                          \
        if (pe_err_ != cudaSuccess) return ::pe::cuda_fail(pe_err_); \
    } while (0)
