// Library runtime helpers (see runtime.cu).
#pragma once
#include "heff_common.cuh"

namespace heff {
// Scratch buffer private to (current device, stream); grows on demand (growth synchronises
// the stream and allocates, so it must not happen inside a stream capture).
int stream_workspace(cudaStream_t stream, size_t bytes, void **out);
int release_workspaces();
// Process-wide count of the kernels the FP64 matvec path has launched (heff_matvec_launches): its launch sites add
// what they enqueue, so a caller can count exactly the launches of a timed region.
void count_launches(int64_t n);
}  // namespace heff
