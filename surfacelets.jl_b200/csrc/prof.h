// Launch-level timing of the library's own kernels with CUDA events, for the
// benchmark: when enabled, every kernel launch is bracketed by two events on
// its stream and filed under the kernel's tag.
#pragma once

#include <cuda_runtime.h>

namespace sfl {

bool prof_on();
// Returns a token for prof_end (-1 when profiling is off).
int prof_begin(const char* tag, cudaStream_t st);
void prof_end(int token, cudaStream_t st);
// Adds a launch's algorithmic bytes (inputs read once, outputs written once)
// to its tag's total; no-op when profiling is off.
void prof_bytes(const char* tag, double bytes);

}  // namespace sfl
