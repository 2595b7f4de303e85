// FP64 trailing update of the multifrontal factorization on the integer tensor
// pipe (tcgen05 kind::i8), exact to FP64 level by digit splitting (the Ozaki
// scheme): every row of the outer panel X is scaled by a power of two and split
// into kOzSlices signed 7-bit digits, the products of digit slices are exact
// integer sums, and the tile F -= X X^T is put back together in FP64.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

namespace tdem {

// Device buffers and tensor maps of the digit slices (one set per factorization
// engine; factorizations using it must not overlap).
struct OzakiBuffers {
  int8_t* slices = nullptr;  // [kOzSlices][rows][kOzK] digits
  int* exps = nullptr;       // [rows] row exponents
  int64_t rows = 0;
  int sms = 0;               // SMs of the device: CTAs of the persistent update
  alignas(64) unsigned char map_a[128] = {};  // CUtensorMap of 128-row operand boxes
  alignas(64) unsigned char map_b[128] = {};  // CUtensorMap of 64-row operand boxes
};

// Creates the tensor maps over slices/exps already allocated for `rows` rows and
// sets the kernels' shared-memory limits (current device).
std::string ozaki_setup(OzakiBuffers& ob);

// Splits the outer-panel rows [J1, m) of every front of a task list into digits
// (64 rows per CTA; aux[i] = the i-th front's first row in the buffer).
void launch_ozaki_slice(const double* L, const int64_t* l_off, const int* m, const int* k, const int* fronts,
                        const int64_t* prefix, const int64_t* aux, int count, int64_t ctas, int j0,
                        const OzakiBuffers& ob, cudaStream_t s);

// F[J1:m, J1:m] -= X X^T for the same fronts, in the 128 x 128 lower-triangle tiles
// of the syrk_big task list (two CTAs per tile, one per 64-column half); err[2]
// is set when a wait inside the kernel gave up.
void launch_ozaki_update(double* L, double* U, const int64_t* l_off, const int64_t* u_off, const int* m,
                         const int* k, const int* fronts, const int64_t* prefix, const int64_t* aux, int count,
                         int64_t ctas, int j0, const OzakiBuffers& ob, int* err, cudaStream_t s);

}  // namespace tdem
