// Library runtime helpers (see runtime.cu).
#pragma once
#include "heff_common.cuh"

namespace heff {
// Scratch buffer private to (current device, stream); grows on demand (growth synchronises
// the stream and allocates, so it must not happen inside a stream capture).
int stream_workspace(cudaStream_t stream, size_t bytes, void **out);
int release_workspaces();
}  // namespace heff
