// Tensor-core (tcgen05, 3xTF32) trailing update of the FP32 factorization.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

namespace tdem {

// Sets the kernel's shared-memory limit; call once per device before launching.
std::string tc_update_setup();

// F[J1:m, J1:m] -= X X^T with X = F[J1:m, J0:J1] for the fronts of one task list
// (128 x 128 lower-triangle tiles, ctas in total; j0 names the inner panel that
// ends the outer panel [J0, J1)).  err[2] is set if a wait inside the kernel gave
// up.
void launch_syrk_tc(float* L, float* U, const int64_t* l_off, const int64_t* u_off, const int* m, const int* k,
                    const int* fronts, const int64_t* prefix, int count, int64_t ctas, int j0, int* err,
                    cudaStream_t s);

}  // namespace tdem
