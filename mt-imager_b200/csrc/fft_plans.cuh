#pragma once
#include <cufft.h>
#include "mtb_internal.cuh"

namespace mtb {
// Cached 2-D batched plan (batch planes of ny x nx, contiguous); `work` is the
// work-area size the plan needs.
int fft_plan(cufftType type, int ny, int nx, int batch, cufftHandle *plan, size_t *work);
// Executes the cached plan on `stream` with `work` as its work area.
int fft_exec(cufftType type, int ny, int nx, int batch, void *in, void *out, int direction,
             void *work, size_t work_bytes, cudaStream_t stream);
void fft_release_all();
}  // namespace mtb
