// Internal helpers shared by the CUDA entry points and the host engine.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace alk {
int cuda_fail(cudaError_t e);
void set_last_cuda_error(cudaError_t e);
const char* last_cuda_error();
// sm_100a kernel launches issued by this library since load (statistics).
extern uint64_t g_kernel_launches;
}  // namespace alk
