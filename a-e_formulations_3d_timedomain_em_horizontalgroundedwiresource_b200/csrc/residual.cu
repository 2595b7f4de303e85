// Residual norms of a block of solutions of a sparse system, on the device:
//   norms[2j] = ||b_j - A x_j||_2,  norms[2j + 1] = ||b_j||_2   for j < ncols.
//
// Two deterministic passes.  Pass 1 (kResBlocks CTAs of 256 threads): one warp per
// CSR row, lanes over the row's entries and a shuffle reduction per column; each
// CTA writes its partial sums of squares to scratch[cta][j][2].  Pass 2 (one CTA):
// thread j adds the kResBlocks partials of column j in CTA order.  The row -> warp
// assignment and every summation order are fixed, so repeated calls on the same
// data give bit-identical norms.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/tdem.h"
#include "residual.h"

namespace tdem {
namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;

__global__ void __launch_bounds__(kThreads)
k_residual_partial(int64_t n, const int64_t* __restrict__ rowptr, const int* __restrict__ col,
                   const double* __restrict__ val, const double* __restrict__ x, const double* __restrict__ b,
                   int64_t ld, int ncols, double* __restrict__ partial) {
  __shared__ double red[kWarps][kResMaxCols][2];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // lane l accumulates columns l and l + 32
  double rr[2] = {0.0, 0.0}, bb[2] = {0.0, 0.0};
  const int64_t gw = (int64_t)blockIdx.x * kWarps + warp, nw = (int64_t)gridDim.x * kWarps;
  for (int64_t i = gw; i < n; i += nw) {
    const int64_t p0 = rowptr[i], p1 = rowptr[i + 1];
    for (int j = 0; j < ncols; ++j) {
      const double* xj = x + (int64_t)j * ld;
      double s = 0.0;
      for (int64_t p = p0 + lane; p < p1; p += 32) s = fma(val[p], xj[col[p]], s);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      if (lane == (j & 31)) {
        const double bi = b[i + (int64_t)j * ld];
        const double r = bi - s;
        rr[j >> 5] = fma(r, r, rr[j >> 5]);
        bb[j >> 5] = fma(bi, bi, bb[j >> 5]);
      }
    }
  }
  for (int h = 0; h < 2; ++h) {
    const int j = lane + 32 * h;
    if (j < ncols) {
      red[warp][j][0] = rr[h];
      red[warp][j][1] = bb[h];
    }
  }
  __syncthreads();
  for (int q = threadIdx.x; q < 2 * ncols; q += kThreads) {
    const int j = q >> 1, c = q & 1;
    double s = 0.0;
    for (int w = 0; w < kWarps; ++w) s += red[w][j][c];
    partial[((int64_t)blockIdx.x * kResMaxCols + j) * 2 + c] = s;
  }
}

__global__ void k_residual_final(int ncols, const double* __restrict__ partial, double* __restrict__ norms) {
  const int q = threadIdx.x;
  if (q >= 2 * ncols) return;
  const int j = q >> 1, c = q & 1;
  double s = 0.0;
  for (int blk = 0; blk < kResBlocks; ++blk) s += partial[((int64_t)blk * kResMaxCols + j) * 2 + c];
  norms[2 * j + c] = sqrt(s);
}

}  // namespace

const char* check_residual_args(int64_t n, const int64_t* rowptr, const int* col, const double* val,
                                const double* x, const double* b, int64_t ld, int ncols, const double* norms) {
  if (n < 0) return "n must be non-negative";
  if (ncols < 1 || ncols > kResMaxCols) return "ncols must be in [1, 64]";
  if (ld < n) return "ld must be at least n";
  if (!rowptr || !norms || (n > 0 && (!col || !val || !x || !b))) return "null pointer";
  return nullptr;
}

cudaError_t launch_residual_norms(int64_t n, const int64_t* rowptr, const int* col, const double* val,
                                  const double* x, const double* b, int64_t ld, int ncols, double* norms,
                                  double* scratch, cudaStream_t s) {
  k_residual_partial<<<kResBlocks, kThreads, 0, s>>>(n, rowptr, col, val, x, b, ld, ncols, scratch);
  k_residual_final<<<1, 2 * kResMaxCols, 0, s>>>(ncols, scratch, norms);
  return cudaGetLastError();
}

}  // namespace tdem

namespace {

// Makes `device` current for the lifetime of the guard and restores the caller's.
struct DeviceGuard {
  int prev = -1;
  cudaError_t err = cudaSuccess;
  explicit DeviceGuard(int device) {
    err = cudaGetDevice(&prev);
    if (err == cudaSuccess && prev != device) err = cudaSetDevice(device);
  }
  ~DeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

}  // namespace

extern "C" tdem_status tdem_residual_norms(int device, int64_t n, const int64_t* rowptr, const int* col,
                                           const double* val, const double* x, const double* b, int64_t ld,
                                           int ncols, double* norms, void* stream) {
  if (tdem::check_residual_args(n, rowptr, col, val, x, b, ld, ncols, norms)) return TDEM_ERR_ARGUMENT;
  DeviceGuard g(device);
  if (g.err != cudaSuccess) return TDEM_ERR_CUDA;
  cudaStream_t s = (cudaStream_t)stream;
  double* scratch = nullptr;
  if (cudaMallocAsync((void**)&scratch, tdem::kResScratchBytes, s) != cudaSuccess) return TDEM_ERR_CUDA;
  const cudaError_t e = tdem::launch_residual_norms(n, rowptr, col, val, x, b, ld, ncols, norms, scratch, s);
  const cudaError_t f = cudaFreeAsync(scratch, s);
  return (e == cudaSuccess && f == cudaSuccess) ? TDEM_OK : TDEM_ERR_CUDA;
}

// ---------------------------------------------------------------------------
// Allocation-free variant: the scratch is a file-scope device array of fixed
// size (kResScratchBytes = 303,104 bytes: 296 CTAs x 64 columns x 2 sums), so a
// call makes no device allocation.  Its device address is looked up on every
// call (cudaGetSymbolAddress, with the call's device current): cheap once the
// module is loaded, and never stale, also after a caller's cudaDeviceReset.  The
// first call on a device may load the module and should happen before any stream
// capture.  The scratch needs no initial value (pass 1 writes every entry pass 2
// reads).  Calls whose executions overlap on one device share the scratch and
// race: order them on one stream or synchronise between them.
// ---------------------------------------------------------------------------
namespace {

__device__ __align__(256) double g_res_scratch[tdem::kResBlocks * tdem::kResMaxCols * 2];

constexpr int kMaxDevices = 64;

// Device address of g_res_scratch on the current device (nullptr on failure).
double* scratch_address() {
  void* p = nullptr;
  if (cudaGetSymbolAddress(&p, g_res_scratch) != cudaSuccess) return nullptr;
  return static_cast<double*>(p);
}

}  // namespace

extern "C" tdem_status tdem_residual_norms_noalloc(int device, int64_t n, const int64_t* rowptr, const int* col,
                                                   const double* val, const double* x, const double* b, int64_t ld,
                                                   int ncols, double* norms, void* stream) {
  if (tdem::check_residual_args(n, rowptr, col, val, x, b, ld, ncols, norms)) return TDEM_ERR_ARGUMENT;
  if (device < 0 || device >= kMaxDevices) return TDEM_ERR_ARGUMENT;
  DeviceGuard g(device);
  if (g.err != cudaSuccess) return TDEM_ERR_CUDA;
  double* scratch = scratch_address();
  if (!scratch) return TDEM_ERR_CUDA;
  const cudaError_t e =
      tdem::launch_residual_norms(n, rowptr, col, val, x, b, ld, ncols, norms, scratch, (cudaStream_t)stream);
  return e == cudaSuccess ? TDEM_OK : TDEM_ERR_CUDA;
}
