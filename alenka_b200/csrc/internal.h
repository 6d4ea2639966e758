// Internal helpers shared by the CUDA entry points and the host engine.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "alenka_b200.h"

#include <vector>

namespace alk {
int cuda_fail(cudaError_t e);
void set_last_cuda_error(cudaError_t e);
const char* last_cuda_error();
// sm_100a kernel launches issued by this library since load (statistics).
extern uint64_t g_kernel_launches;

// Source pointer for a host-to-device upload of `bytes` from `host`: the caller's buffer,
// or, while the stream is being captured into a CUDA graph, a pinned copy that must live
// as long as the graph. Such copies are listed in capture_host_buffers() (this thread);
// whoever ends the capture takes them over and frees them (cudaFreeHost) with the graph.
const void* upload_source(const void* host, size_t bytes, cudaStream_t s, cudaError_t* err);
std::vector<void*>& capture_host_buffers();

// A filter program as a conjunction of single-column tests `value * mul OP k` (OP one of
// the comparison opcodes); false when the program has another form. An empty program is
// the empty conjunction.
struct CardConj {
  int64_t mul, k;
  uint32_t slot, op;
};
bool program_conjuncts(const alk_program& p, std::vector<CardConj>& out);
}  // namespace alk
