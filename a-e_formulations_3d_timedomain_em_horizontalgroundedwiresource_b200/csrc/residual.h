// Device residual norms of a block of solutions (tdem_residual_norms).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace tdem {

constexpr int kResBlocks = 296;   // CTAs of the first pass (2 per SM)
constexpr int kResMaxCols = 64;   // most columns per call
// scratch of the two passes: kResBlocks x kResMaxCols x 2 partial sums
constexpr size_t kResScratchBytes = sizeof(double) * kResBlocks * kResMaxCols * 2;

// Returns a message for invalid arguments, nullptr when they are usable.
const char* check_residual_args(int64_t n, const int64_t* rowptr, const int* col, const double* val,
                                const double* x, const double* b, int64_t ld, int ncols, const double* norms);

// Launches both passes on stream s; `scratch` holds kResScratchBytes.  Every
// scratch entry the second pass reads is written by the first one, so scratch
// needs no initialisation.
cudaError_t launch_residual_norms(int64_t n, const int64_t* rowptr, const int* col, const double* val,
                                  const double* x, const double* b, int64_t ld, int ncols, double* norms,
                                  double* scratch, cudaStream_t s);

}  // namespace tdem
