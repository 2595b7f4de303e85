// GPU multifrontal Cholesky: batched dense front kernels driven level by level
// and panel by panel from the host plan in symbolic.h.  Kernels are templated on
// the factor's value type (FP64, or FP32 for the mixed-precision path); the
// caller's right-hand sides and solutions are always FP64.
//
// Layout in HBM
//   L   persistent factor; front s owns an m x k column-major block (ld = m) at l_off[s]
//   U   update workspace; front s owns an r x r block (ld = r, r = m - k) at u_off[s]
//       while it waits for its parent (offsets planned on the host, first fit)
//   W   solve front vectors, m x nrhs per front at w_off[s] * nrhs (ld = m)
// Every kernel receives a task list (fronts + CTA prefix sums) and finds its
// front by binary search over the prefix, so one launch covers every front of a
// level that takes part in the current panel.
//
// Factorization per level: zero the update blocks, extend-add the children,
// then for each 64-wide inner panel [j0, j1): Cholesky of the diagonal block,
// triangular solve of the rows below, rank-64 update of the rest of the 256-wide
// outer panel [J0, J1); at the end of each outer panel one rank-(J1 - J0) update
// of the whole trailing matrix on 128 x 128 register-blocked tiles.
#include "gpu_cholesky.h"

#include <algorithm>
#include <cstdio>
#include <type_traits>

#include "tc_update.h"

namespace tdem {
namespace {

constexpr int P = kPanel;  // 64

__device__ __forceinline__ int find_task(const int64_t* __restrict__ prefix, int count, int64_t b) {
  int lo = 0, hi = count - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (prefix[mid] <= b) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

struct Fronts {
  const int64_t* l_off;
  const int64_t* u_off;
  const int* m;
  const int* k;
};

// Element (i, c), i >= c, of a split front.
template <class T>
__device__ __forceinline__ T* felem(T* L, T* U, int64_t lo, int64_t uo, int m, int k, int i, int c) {
  return (c < k) ? L + lo + i + (int64_t)c * m : U + uo + (i - k) + (int64_t)(c - k) * (m - k);
}

__device__ __forceinline__ double tsqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float tsqrt(float x) { return sqrtf(x); }

// ---------------------------------------------------------------------------
// factorization kernels
// ---------------------------------------------------------------------------
template <class T>
__global__ void k_scatter_entries(T* __restrict__ L, const int64_t* __restrict__ dst,
                                  const double* __restrict__ val, int64_t nnz) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nnz;
       q += (int64_t)gridDim.x * blockDim.x)
    L[dst[q]] = (T)val[q];
}

template <class T>
__global__ void k_zero_u(T* __restrict__ U, Fronts f, const int* __restrict__ fronts,
                         const int64_t* __restrict__ prefix, int count) {
  const int idx = find_task(prefix, count, blockIdx.x);
  const int s = fronts[idx];
  const int m = f.m[s], k = f.k[s], r = m - k;
  const int64_t t = blockIdx.x - prefix[idx];
  const int c0 = (int)t * kSolveRows, c1 = min(r, c0 + kSolveRows);
  T* u = U + f.u_off[s];
  for (int c = c0; c < c1; ++c)
    for (int i = threadIdx.x; i < r; i += blockDim.x) u[i + (int64_t)c * r] = (T)0;
}

// Extend-add of the children's update blocks into their parents (one child per
// parent per launch, so no two CTAs write the same parent element).  One warp
// per child column, 8 columns per CTA.
template <class T>
__global__ void k_extend_add(T* __restrict__ L, T* __restrict__ U, Fronts f, const int* __restrict__ parent,
                             const int64_t* __restrict__ rel_off, const int* __restrict__ rel,
                             const int* __restrict__ kids, const int64_t* __restrict__ prefix, int count) {
  const int idx = find_task(prefix, count, blockIdx.x);
  const int c = kids[idx];
  const int p = parent[c];
  const int mc = f.m[c], kc = f.k[c], rc = mc - kc;
  const int mp = f.m[p], kp = f.k[p];
  const int64_t lo = f.l_off[p], uo = f.u_off[p];
  const int* rl = rel + rel_off[c];
  const T* uc = U + f.u_off[c];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int b = (int)(blockIdx.x - prefix[idx]) * 8 + warp;
  if (b >= rc) return;
  const int pc = rl[b];
  for (int a = b + lane; a < rc; a += 32) *felem(L, U, lo, uo, mp, kp, rl[a], pc) += uc[a + (int64_t)b * rc];
}

// Cholesky of the w x w diagonal block of panel [j0, j0 + w) (one CTA per front).
template <class T>
__global__ void k_potrf(T* __restrict__ L, Fronts f, const int* __restrict__ fronts, int j0,
                        int* __restrict__ err, const int* __restrict__ c0_of) {
  __shared__ T A[P][P + 1];
  const int s = fronts[blockIdx.x];
  const int m = f.m[s], k = f.k[s];
  const int w = min(P, k - j0);
  T* F = L + f.l_off[s];
  for (int idx = threadIdx.x; idx < w * w; idx += blockDim.x) {
    const int i = idx % w, j = idx / w;
    A[i][j] = (i >= j) ? F[(j0 + i) + (int64_t)(j0 + j) * m] : (T)0;
  }
  __syncthreads();
  for (int j = 0; j < w; ++j) {
    if (threadIdx.x == 0) {
      T d = A[j][j];
      if (!(d > (T)0)) {
        atomicCAS(err, 0, c0_of[s] + j0 + j + 1);
        d = (T)1;
      }
      A[j][j] = tsqrt(d);
    }
    __syncthreads();
    const T inv = (T)1 / A[j][j];
    for (int i = j + 1 + threadIdx.x; i < w; i += blockDim.x) A[i][j] *= inv;
    __syncthreads();
    const int t = w - j - 1;
    for (int idx = threadIdx.x; idx < t * t; idx += blockDim.x) {
      const int i = j + 1 + idx / t, c = j + 1 + idx % t;
      if (c <= i) A[i][c] -= A[i][j] * A[c][j];
    }
    __syncthreads();
  }
  for (int idx = threadIdx.x; idx < w * w; idx += blockDim.x) {
    const int i = idx % w, j = idx / w;
    if (i >= j) F[(j0 + i) + (int64_t)(j0 + j) * m] = A[i][j];
  }
}

// Panel triangular solve: rows [j1, m) of the panel columns times L_dd^-T.
// kTrsmRows rows per CTA, one thread per row.
template <class T>
__global__ void __launch_bounds__(kTrsmRows) k_trsm(T* __restrict__ L, Fronts f, const int* __restrict__ fronts,
                                                    const int64_t* __restrict__ prefix, int count, int j0) {
  extern __shared__ __align__(16) unsigned char sm_raw[];
  T(*Ld)[P + 1] = reinterpret_cast<T(*)[P + 1]>(sm_raw);
  T(*X)[P + 1] = reinterpret_cast<T(*)[P + 1]>(sm_raw + sizeof(T) * P * (P + 1));
  const int idx = find_task(prefix, count, blockIdx.x);
  const int s = fronts[idx];
  const int m = f.m[s], k = f.k[s];
  const int w = min(P, k - j0), j1 = j0 + w;
  T* F = L + f.l_off[s];
  const int r0 = j1 + (int)(blockIdx.x - prefix[idx]) * kTrsmRows;
  for (int q = threadIdx.x; q < w * w; q += blockDim.x) {
    const int i = q % w, j = q / w;
    Ld[i][j] = (i >= j) ? F[(j0 + i) + (int64_t)(j0 + j) * m] : (T)0;
  }
  for (int q = threadIdx.x; q < kTrsmRows * w; q += blockDim.x) {
    const int i = q % kTrsmRows, j = q / kTrsmRows;
    const int row = r0 + i;
    X[i][j] = (row < m) ? F[row + (int64_t)(j0 + j) * m] : (T)0;
  }
  __syncthreads();
  const int t = threadIdx.x;
  for (int c = 0; c < w; ++c) {
    T v = X[t][c];
    for (int cc = 0; cc < c; ++cc) v -= X[t][cc] * Ld[c][cc];
    X[t][c] = v / Ld[c][c];
  }
  __syncthreads();
  for (int q = threadIdx.x; q < kTrsmRows * w; q += blockDim.x) {
    const int i = q % kTrsmRows, j = q / kTrsmRows;
    const int row = r0 + i;
    if (row < m) F[row + (int64_t)(j0 + j) * m] = X[i][j];
  }
}

// Update of the rest of the outer panel by the inner panel [j0, j1):
// F[r, c] -= sum_p X[r, p] X[c, p] for c in [j1, J1), r >= c.  64 x 64 tiles,
// 256 threads with 4 x 4 outputs each.
template <class T>
__global__ void __launch_bounds__(256) k_syrk_panel(T* __restrict__ L, Fronts f, const int* __restrict__ fronts,
                                                    const int64_t* __restrict__ prefix, int count, int j0) {
  constexpr int TS = kTileSyrk;
  extern __shared__ __align__(16) unsigned char sm_raw[];
  T(*As)[P + 1] = reinterpret_cast<T(*)[P + 1]>(sm_raw);
  T(*Bs)[P + 1] = reinterpret_cast<T(*)[P + 1]>(sm_raw + sizeof(T) * TS * (P + 1));
  const int idx = find_task(prefix, count, blockIdx.x);
  const int s = fronts[idx];
  const int m = f.m[s], k = f.k[s];
  const int w = min(P, k - j0), j1 = j0 + w;
  const int J0 = (j0 / kOuter) * kOuter, J1 = min(k, J0 + kOuter);
  T* F = L + f.l_off[s];
  const int nr = (m - j1 + TS - 1) / TS;
  int t = (int)(blockIdx.x - prefix[idx]);
  int bj = 0;
  while (t >= nr - bj) {
    t -= nr - bj;
    ++bj;
  }
  const int bi = bj + t;
  const int r0 = j1 + bi * TS, c0 = j1 + bj * TS;
  for (int q = threadIdx.x; q < TS * w; q += blockDim.x) {
    const int i = q % TS, p = q / TS;
    As[i][p] = (r0 + i < m) ? F[(r0 + i) + (int64_t)(j0 + p) * m] : (T)0;
    Bs[i][p] = (c0 + i < J1) ? F[(c0 + i) + (int64_t)(j0 + p) * m] : (T)0;
  }
  __syncthreads();
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  T acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = (T)0;
  for (int p = 0; p < w; ++p) {
    T av[4], bv[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) av[a] = As[tx + 16 * a][p];
#pragma unroll
    for (int b = 0; b < 4; ++b) bv[b] = Bs[ty + 16 * b][p];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) acc[a][b] = fma(av[a], bv[b], acc[a][b]);
  }
  T old[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int r = r0 + tx + 16 * a, c = c0 + ty + 16 * b;
      old[a][b] = (r < m && c < J1 && c <= r) ? F[r + (int64_t)c * m] : (T)0;
    }
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int r = r0 + tx + 16 * a, c = c0 + ty + 16 * b;
      if (r < m && c < J1 && c <= r) F[r + (int64_t)c * m] = old[a][b] - acc[a][b];
    }
}

// Trailing update at the end of an outer panel: F[J1:m, J1:m] -= X X^T with X the
// outer panel rows [J1, m), columns [J0, J1).  128 x 128 tiles, 256 threads with
// 8 x 8 outputs each, K consumed in chunks of 32.
constexpr int KC = 32;
template <class T>
__global__ void __launch_bounds__(256) k_syrk_big(T* __restrict__ L, T* __restrict__ U, Fronts f,
                                                  const int* __restrict__ fronts,
                                                  const int64_t* __restrict__ prefix, int count, int j0) {
  constexpr int TB = kTileBig;
  extern __shared__ __align__(16) unsigned char sm_raw[];
  T(*As)[TB + 1] = reinterpret_cast<T(*)[TB + 1]>(sm_raw);
  T(*Bs)[TB + 1] = reinterpret_cast<T(*)[TB + 1]>(sm_raw + sizeof(T) * KC * (TB + 1));
  const int idx = find_task(prefix, count, blockIdx.x);
  const int s = fronts[idx];
  const int m = f.m[s], k = f.k[s];
  const int J0 = (j0 / kOuter) * kOuter, J1 = min(k, J0 + kOuter);
  const int64_t lo = f.l_off[s], uo = f.u_off[s];
  const T* F = L + lo;
  const int64_t t = blockIdx.x - prefix[idx];
  int bi = (int)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
  while ((int64_t)(bi + 1) * (bi + 2) / 2 <= t) ++bi;
  while ((int64_t)bi * (bi + 1) / 2 > t) --bi;
  const int bj = (int)(t - (int64_t)bi * (bi + 1) / 2);
  const int r0 = J1 + bi * TB, c0 = J1 + bj * TB;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  T acc[8][8];
#pragma unroll
  for (int a = 0; a < 8; ++a)
#pragma unroll
    for (int b = 0; b < 8; ++b) acc[a][b] = (T)0;
  const int K = J1 - J0;
  for (int k0 = 0; k0 < K; k0 += KC) {
    const int kc = min(KC, K - k0);
    for (int q = threadIdx.x; q < TB * KC; q += blockDim.x) {
      const int i = q % TB, p = q / TB;
      const bool okp = p < kc;
      const int64_t col = (int64_t)(J0 + k0 + p) * m;
      As[p][i] = (okp && r0 + i < m) ? F[(r0 + i) + col] : (T)0;
      Bs[p][i] = (okp && c0 + i < m) ? F[(c0 + i) + col] : (T)0;
    }
    __syncthreads();
#pragma unroll 4
    for (int p = 0; p < kc; ++p) {
      T av[8], bv[8];
#pragma unroll
      for (int a = 0; a < 8; ++a) av[a] = As[p][tx + 16 * a];
#pragma unroll
      for (int b = 0; b < 8; ++b) bv[b] = Bs[p][ty + 16 * b];
#pragma unroll
      for (int a = 0; a < 8; ++a)
#pragma unroll
        for (int b = 0; b < 8; ++b) acc[a][b] = fma(av[a], bv[b], acc[a][b]);
    }
    __syncthreads();
  }
  // per output row: the 8 loads first, then the 8 stores (the element pointers may
  // alias as far as the compiler knows, which would serialise load-store pairs)
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    const int r = r0 + tx + 16 * a;
    if (r >= m) continue;
    T old[8];
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      const int c = c0 + ty + 16 * b;
      old[b] = (c < m && c <= r) ? *felem(L, U, lo, uo, m, k, r, c) : (T)0;
    }
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      const int c = c0 + ty + 16 * b;
      if (c < m && c <= r) *felem(L, U, lo, uo, m, k, r, c) = old[b] - acc[a][b];
    }
  }
}

// ---------------------------------------------------------------------------
// solve kernels (front vectors W: m x nrhs per front, ld = m)
// ---------------------------------------------------------------------------
struct SolveArgs {
  const int64_t* l_off;
  const int64_t* w_off;
  const int* m;
  const int* k;
  const int64_t* rows_off;
  const int* rows;  // caller vector position of each front row
  int nrhs;
  int64_t ld;
};

template <class T>
__global__ void k_fwd_init(T* __restrict__ W, const double* __restrict__ b, SolveArgs a,
                           const int* __restrict__ fronts, const int64_t* __restrict__ prefix, int count) {
  const int idx = find_task(prefix, count, blockIdx.x);
  const int s = fronts[idx];
  const int m = a.m[s], k = a.k[s];
  const int i = (int)(blockIdx.x - prefix[idx]) * kSolveRows + threadIdx.x;
  if (i >= m) return;
  T* w = W + a.w_off[s] * a.nrhs;
  const int pos = (i < k) ? a.rows[a.rows_off[s] + i] : -1;
  for (int r = 0; r < a.nrhs; ++r) w[i + (int64_t)r * m] = (i < k) ? (T)b[pos + r * a.ld] : (T)0;
}

template <class T>
__global__ void k_fwd_extend(T* __restrict__ W, SolveArgs a, const int* __restrict__ parent,
                             const int64_t* __restrict__ rel_off, const int* __restrict__ rel,
                             const int* __restrict__ kids, const int64_t* __restrict__ prefix, int count) {
  const int idx = find_task(prefix, count, blockIdx.x);
  const int c = kids[idx], p = parent[c];
  const int mc = a.m[c], kc = a.k[c], rc = mc - kc, mp = a.m[p];
  const int i = (int)(blockIdx.x - prefix[idx]) * kSolveRows + threadIdx.x;
  if (i >= rc) return;
  const T* wc = W + a.w_off[c] * a.nrhs;
  T* wp = W + a.w_off[p] * a.nrhs;
  const int pr = rel[rel_off[c] + i];
  for (int r = 0; r < a.nrhs; ++r) wp[pr + (int64_t)r * mp] += wc[kc + i + (int64_t)r * mc];
}

// Forward diagonal-block solve of panel [j0, j0 + w) (one CTA per front).
template <class T>
__global__ void k_fwd_diag(const T* __restrict__ L, T* __restrict__ W, SolveArgs a,
                           const int* __restrict__ fronts, int j0) {
  __shared__ T Ld[P][P + 1];
  extern __shared__ __align__(16) unsigned char sm_raw[];
  T* Y = reinterpret_cast<T*>(sm_raw);  // P x nrhs
  const int s = fronts[blockIdx.x];
  const int m = a.m[s], k = a.k[s];
  const int w = min(P, k - j0);
  const T* F = L + a.l_off[s];
  T* wv = W + a.w_off[s] * a.nrhs;
  const int nr = a.nrhs;
  for (int q = threadIdx.x; q < w * w; q += blockDim.x) {
    const int i = q % w, j = q / w;
    Ld[i][j] = (i >= j) ? F[(j0 + i) + (int64_t)(j0 + j) * m] : (T)0;
  }
  for (int q = threadIdx.x; q < w * nr; q += blockDim.x) {
    const int i = q % w, r = q / w;
    Y[i + r * P] = wv[j0 + i + (int64_t)r * m];
  }
  __syncthreads();
  for (int c = 0; c < w; ++c) {
    for (int r = threadIdx.x; r < nr; r += blockDim.x) Y[c + r * P] /= Ld[c][c];
    __syncthreads();
    for (int q = threadIdx.x; q < (w - c - 1) * nr; q += blockDim.x) {
      const int i = c + 1 + q % (w - c - 1), r = q / (w - c - 1);
      Y[i + r * P] -= Ld[i][c] * Y[c + r * P];
    }
    __syncthreads();
  }
  for (int q = threadIdx.x; q < w * nr; q += blockDim.x) {
    const int i = q % w, r = q / w;
    wv[j0 + i + (int64_t)r * m] = Y[i + r * P];
  }
}

// W[j1:m] -= L[j1:m, panel] * Y (one row per thread).
template <class T>
__global__ void __launch_bounds__(kSolveRows) k_fwd_update(const T* __restrict__ L, T* __restrict__ W, SolveArgs a,
                                                           const int* __restrict__ fronts,
                                                           const int64_t* __restrict__ prefix, int count, int j0) {
  extern __shared__ __align__(16) unsigned char sm_raw[];
  T* Y = reinterpret_cast<T*>(sm_raw);  // P x nrhs
  const int idx = find_task(prefix, count, blockIdx.x);
  const int s = fronts[idx];
  const int m = a.m[s], k = a.k[s];
  const int w = min(P, k - j0), j1 = j0 + w;
  const T* F = L + a.l_off[s];
  T* wv = W + a.w_off[s] * a.nrhs;
  const int nr = a.nrhs;
  for (int q = threadIdx.x; q < w * nr; q += blockDim.x) {
    const int i = q % w, r = q / w;
    Y[i + r * P] = wv[j0 + i + (int64_t)r * m];
  }
  __syncthreads();
  const int row = j1 + (int)(blockIdx.x - prefix[idx]) * kSolveRows + threadIdx.x;
  if (row >= m) return;
  for (int r = 0; r < nr; ++r) {
    T acc = (T)0;
    for (int c = 0; c < w; ++c) acc = fma(F[row + (int64_t)(j0 + c) * m], Y[c + r * P], acc);
    wv[row + (int64_t)r * m] -= acc;
  }
}

template <class T>
__global__ void k_bwd_init(T* __restrict__ W, const double* __restrict__ x, SolveArgs a,
                           const int* __restrict__ fronts, const int64_t* __restrict__ prefix, int count) {
  const int idx = find_task(prefix, count, blockIdx.x);
  const int s = fronts[idx];
  const int m = a.m[s], k = a.k[s];
  const int i = (int)(blockIdx.x - prefix[idx]) * kSolveRows + threadIdx.x;
  if (i < k || i >= m) return;
  T* w = W + a.w_off[s] * a.nrhs;
  const int pos = a.rows[a.rows_off[s] + i];
  for (int r = 0; r < a.nrhs; ++r) w[i + (int64_t)r * m] = (T)x[pos + r * a.ld];
}

// Partial sums of L[j1:m, panel]^T W[j1:m] over one row chunk.
template <class T>
__global__ void __launch_bounds__(kSolveRows) k_bwd_partial(const T* __restrict__ L, const T* __restrict__ W,
                                                            SolveArgs a, T* __restrict__ part,
                                                            const int* __restrict__ fronts,
                                                            const int64_t* __restrict__ prefix, int count, int j0) {
  __shared__ T red[kSolveRows / 32][P];
  const int idx = find_task(prefix, count, blockIdx.x);
  const int s = fronts[idx];
  const int m = a.m[s], k = a.k[s];
  const int w = min(P, k - j0), j1 = j0 + w;
  const T* F = L + a.l_off[s];
  const T* wv = W + a.w_off[s] * a.nrhs;
  const int row = j1 + (int)(blockIdx.x - prefix[idx]) * kSolveRows + threadIdx.x;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int r = 0; r < a.nrhs; ++r) {
    const T xv = (row < m) ? wv[row + (int64_t)r * m] : (T)0;
    for (int c = 0; c < w; ++c) {
      T v = (row < m) ? F[row + (int64_t)(j0 + c) * m] * xv : (T)0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      if (lane == 0) red[warp][c] = v;
    }
    __syncthreads();
    if (threadIdx.x < w) {
      T v = (T)0;
      for (int q = 0; q < kSolveRows / 32; ++q) v += red[q][threadIdx.x];
      part[((int64_t)blockIdx.x * a.nrhs + r) * P + threadIdx.x] = v;
    }
    __syncthreads();
  }
}

// Backward diagonal-block solve of panel [j0, j0 + w) after subtracting the partials.
template <class T>
__global__ void k_bwd_diag(const T* __restrict__ L, T* __restrict__ W, SolveArgs a, const T* __restrict__ part,
                           const int* __restrict__ fronts, const int64_t* __restrict__ prefix, int j0) {
  __shared__ T Ld[P][P + 1];
  extern __shared__ __align__(16) unsigned char sm_raw[];
  T* Y = reinterpret_cast<T*>(sm_raw);
  const int s = fronts[blockIdx.x];
  const int m = a.m[s], k = a.k[s];
  const int w = min(P, k - j0);
  const T* F = L + a.l_off[s];
  T* wv = W + a.w_off[s] * a.nrhs;
  const int nr = a.nrhs;
  const int64_t b0 = prefix[blockIdx.x], b1 = prefix[blockIdx.x + 1];
  for (int q = threadIdx.x; q < w * w; q += blockDim.x) {
    const int i = q % w, j = q / w;
    Ld[i][j] = (i >= j) ? F[(j0 + i) + (int64_t)(j0 + j) * m] : (T)0;
  }
  for (int q = threadIdx.x; q < w * nr; q += blockDim.x) {
    const int i = q % w, r = q / w;
    T v = wv[j0 + i + (int64_t)r * m];
    for (int64_t b = b0; b < b1; ++b) v -= part[(b * nr + r) * P + i];
    Y[i + r * P] = v;
  }
  __syncthreads();
  for (int c = w - 1; c >= 0; --c) {
    for (int r = threadIdx.x; r < nr; r += blockDim.x) Y[c + r * P] /= Ld[c][c];
    __syncthreads();
    for (int q = threadIdx.x; q < c * nr; q += blockDim.x) {
      const int i = q % c, r = q / c;
      Y[i + r * P] -= Ld[c][i] * Y[c + r * P];
    }
    __syncthreads();
  }
  for (int q = threadIdx.x; q < w * nr; q += blockDim.x) {
    const int i = q % w, r = q / w;
    wv[j0 + i + (int64_t)r * m] = Y[i + r * P];
  }
}

template <class T>
__global__ void k_bwd_store(const T* __restrict__ W, double* __restrict__ x, SolveArgs a,
                            const int* __restrict__ fronts, const int64_t* __restrict__ prefix, int count) {
  const int idx = find_task(prefix, count, blockIdx.x);
  const int s = fronts[idx];
  const int k = a.k[s], m = a.m[s];
  const int i = (int)(blockIdx.x - prefix[idx]) * kSolveRows + threadIdx.x;
  if (i >= k) return;
  const T* w = W + a.w_off[s] * a.nrhs;
  const int pos = a.rows[a.rows_off[s] + i];
  for (int r = 0; r < a.nrhs; ++r) x[pos + r * a.ld] = (double)w[i + (int64_t)r * m];
}

// ---------------------------------------------------------------------------
// fused level solves
//
// One launch per assembly-tree level and direction.  Every CTA owns one 64-row
// block of one front; it takes a ticket (atomicAdd) that names its item, so the
// items start in list order.  A block waits only for pivot blocks of its own
// front that come earlier in the list (flag per pivot block, set with release
// semantics after the block's values are stored), hence every block it waits for
// is already running or finished.  Waits are bounded: after kSpinLimit polls the
// CTA records err[1] and goes on (the results are then wrong and the host reports
// the error; the kernel still ends).
//
// Diagonal blocks are applied through their inverses (Dinv, computed once per
// factorization), so the dependency chain costs one 64 x 64 block product per
// pivot block instead of a 64-step substitution.
// ---------------------------------------------------------------------------
constexpr int SB = kPanel;  // 64 rows per solve block
constexpr unsigned kSpinLimit = 1u << 21;

__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
// Publishes the values the whole CTA stored before its last __syncthreads: the
// acq_rel fence at GPU scope orders those stores (cumulatively, they were observed
// through the barrier) before the relaxed flag store / counter increment.
__device__ __forceinline__ void publish_flag(int* p) {
  asm volatile("fence.acq_rel.gpu;\n\tst.relaxed.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(1) : "memory");
}
__device__ __forceinline__ void publish_add(int* p) {
  asm volatile("fence.acq_rel.gpu;\n\tred.relaxed.gpu.global.add.s32 [%0], %1;" ::"l"(p), "r"(1) : "memory");
}

// Called by one thread.  Gives up after kSpinLimit polls (or at once when an
// earlier wait of this solve gave up) and records the failure in *err.
__device__ void wait_flag(const int* flag, int* err) {
  if (*(volatile int*)err != 0) return;
  for (unsigned it = 0; it < kSpinLimit; ++it) {
    if (ld_acquire(flag) != 0) return;
    __nanosleep(64);
  }
  atomicExch(err, 1);
}

// Waits until *c reaches target (one thread; bounded like wait_flag).
__device__ void wait_count(const int* c, int target, int* err) {
  if (*(volatile int*)err != 0) return;
  for (unsigned it = 0; it < kSpinLimit; ++it) {
    if (ld_acquire(c) >= target) return;
    __nanosleep(64);
  }
  atomicExch(err, 1);
}

struct FusedArgs {
  const int* units;        // units of this launch (8 ints each, Symbolic::solve_units)
  int* ticket;             // launch-order counter (zeroed before the solve)
  int* flags;              // one per pivot block (zeroed before the solve)
  int* counters;           // finished chunk units per row (zeroed before the solve)
  const int64_t* flag_off; // per front: first flag
  const int64_t* dinv_off; // per front: first inverted diagonal block
  int* err;                // err[1]: a wait gave up
};

// A chunk unit hands its partial sums (thread t: entries (t % 64, t / 64 + 4 j))
// to the final unit of its row: store, then publish with a counter increment.
template <class T, int RPT>
__device__ __forceinline__ void publish_partial(T* part, const T (&acc)[RPT], int nr_rhs, int* counter) {
  const int i = threadIdx.x & 63, g = threadIdx.x >> 6;
#pragma unroll
  for (int j = 0; j < RPT; ++j) {
    const int r = g + 4 * j;
    if (r < nr_rhs) part[i + SB * r] = acc[j];
  }
  __syncthreads();
  if (threadIdx.x == 0) publish_add(counter);
}

// The final unit of a row: acc = (p_0 + p_1) + ... in a fixed order (left as is
// when the row has no chunk units).
template <class T, int RPT>
__device__ __forceinline__ void gather_partials(const T* part, int nparts, int nr_rhs, const int* counter, int* err,
                                                T (&acc)[RPT]) {
  if (nparts == 0) return;
  if (threadIdx.x == 0) wait_count(counter, nparts, err);
  __syncthreads();
  const int i = threadIdx.x & 63, g = threadIdx.x >> 6;
#pragma unroll
  for (int j = 0; j < RPT; ++j) {
    const int r = g + 4 * j;
    if (r >= nr_rhs) continue;
    T tot = __ldcg(part + i + SB * r);
    for (int c = 1; c < nparts; ++c) tot += __ldcg(part + (int64_t)c * SB * nr_rhs + i + SB * r);
    acc[j] = tot;
  }
}

// 64 x 64 block of a front (rows [r0, r0 + nr), columns [c0, c0 + nc), zero
// outside) into 16 registers per thread: element (i, c) goes to thread
// (i + 64 c) mod 256, slot (i + 64 c) / 256.
template <class T>
__device__ __forceinline__ void load_block(T (&pre)[16], const T* __restrict__ F, int64_t ld, int r0, int nr, int c0,
                                           int nc) {
#pragma unroll
  for (int e = 0; e < 16; ++e) {
    const int q = threadIdx.x + 256 * e;
    const int i = q & 63, c = q >> 6;
    pre[e] = (i < nr && c < nc) ? F[(r0 + i) + (int64_t)(c0 + c) * ld] : (T)0;
  }
}
// registers -> Ls[c][i]
template <class T>
__device__ __forceinline__ void store_block(T (*Ls)[SB + 1], const T (&pre)[16]) {
#pragma unroll
  for (int e = 0; e < 16; ++e) {
    const int q = threadIdx.x + 256 * e;
    Ls[q >> 6][q & 63] = pre[e];
  }
}

// Forward unit: row block R of front s (R < pb: pivot rows [64R, ..); else update
// rows [k + 64 (R - pb), ..)), accumulating L_Rq y_q for the pivot blocks q in
// [lo, hi).  Chunk units publish partial sums; the final unit (q = the last one
// the row needs) adds them, then a pivot row solves y_R = Dinv_R (w_R - sum) and
// raises its flag, an update row stores w_R - sum for the parent.
// Thread t: row i = t % 64 of the block, right-hand sides r = t / 64 + 4 j.
template <class T, int RPT>
__global__ void __launch_bounds__(256, 2) k_fwd_level(const T* __restrict__ L, const T* __restrict__ Dinv, T* W, T* part,
                                                   SolveArgs a, FusedArgs fa) {
  __shared__ T Ls[SB][SB + 1];
  __shared__ int s_item;
  extern __shared__ __align__(16) unsigned char sm_raw[];
  T* Ys = reinterpret_cast<T*>(sm_raw);  // SB x nrhs, [c * nrhs + r]
  const int t = threadIdx.x, i = t & 63, g = t >> 6;
  if (t == 0) s_item = atomicAdd(fa.ticket, 1);
  __syncthreads();
  const int* u = fa.units + 8 * s_item;
  const int s = u[0], R = u[1], lo = u[2], hi = u[3], slot = u[4], cnt = u[5], nparts = u[6], fin = u[7];
  const int m = a.m[s], k = a.k[s], nr_rhs = a.nrhs;
  const int pb = (k + SB - 1) / SB;
  const bool piv = R < pb;
  const int r0 = piv ? SB * R : k + SB * (R - pb);
  const int nr = min(SB, (piv ? k : m) - r0);
  const T* F = L + a.l_off[s];
  T* w = W + a.w_off[s] * nr_rhs;
  const int* flags = fa.flags + fa.flag_off[s];
  T acc[RPT];
#pragma unroll
  for (int j = 0; j < RPT; ++j) acc[j] = (T)0;
  // final pivot unit: its inverted diagonal block and its own rows of W do not
  // depend on this launch, so they are read before any wait
  // (with many right-hand sides the registers go to the accumulators instead and
  // the inverse is read after the last block)
  constexpr bool kPreD = RPT <= 2;
  const T* D = Dinv + fa.dinv_off[s] + (int64_t)R * SB * SB;
  T dpre[kPreD ? 16 : 1], wrow[RPT];
  if (fin && piv) {
    if (kPreD) {
#pragma unroll
      for (int e = 0; e < 16; ++e) {
        const int q = t + 256 * e, ii = q & 63, c = q >> 6;
        dpre[e] = (ii < nr && c < nr) ? D[ii + c * nr] : (T)0;
      }
    }
#pragma unroll
    for (int j = 0; j < RPT; ++j) {
      const int r = g + 4 * j;
      wrow[j] = (r < nr_rhs && i < nr) ? w[r0 + i + (int64_t)r * m] : (T)0;
    }
  }
  T* my_part = part + (int64_t)slot * SB * nr_rhs;
  T tot[RPT];
#pragma unroll
  for (int j = 0; j < RPT; ++j) tot[j] = (T)0;
  // the chunk partials of this row are ready long before the last block's flag
  if (fin) gather_partials<T, RPT>(my_part, nparts, nr_rhs, fa.counters + cnt, fa.err, tot);
  T pre[16];
  if (lo < hi) load_block(pre, F, m, r0, nr, SB * lo, min(SB, k - SB * lo));
  for (int q = lo; q < hi; ++q) {
    const int wq = min(SB, k - SB * q);
    if (t == 0) wait_flag(flags + q, fa.err);
    __syncthreads();
    store_block(Ls, pre);
    for (int e = t; e < SB * nr_rhs; e += 256) {
      const int c = e % SB, r = e / SB;
      Ys[c * nr_rhs + r] = (c < wq) ? __ldcg(w + SB * q + c + (int64_t)r * m) : (T)0;
    }
    __syncthreads();
    if (q + 1 < hi) load_block(pre, F, m, r0, nr, SB * (q + 1), min(SB, k - SB * (q + 1)));
#pragma unroll 8
    for (int c = 0; c < SB; ++c) {
      const T l = Ls[c][i];
#pragma unroll
      for (int j = 0; j < RPT; ++j) {
        const int r = g + 4 * j;
        if (r < nr_rhs) acc[j] = fma(l, Ys[c * nr_rhs + r], acc[j]);
      }
    }
  }
  if (!fin) {
    publish_partial<T, RPT>(my_part, acc, nr_rhs, fa.counters + cnt);
    return;
  }
#pragma unroll
  for (int j = 0; j < RPT; ++j) acc[j] = tot[j] + acc[j];
  if (!piv) {
    if (i < nr) {
#pragma unroll
      for (int j = 0; j < RPT; ++j) {
        const int r = g + 4 * j;
        if (r < nr_rhs) w[r0 + i + (int64_t)r * m] -= acc[j];
      }
    }
    return;
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < RPT; ++j) {
    const int r = g + 4 * j;
    if (r < nr_rhs) Ys[i * nr_rhs + r] = (i < nr) ? wrow[j] - acc[j] : (T)0;
  }
  if constexpr (kPreD) {
    store_block(Ls, dpre);
  } else {
    for (int e = t; e < SB * SB; e += 256) {
      const int ii = e & 63, c = e >> 6;
      Ls[c][ii] = (ii < nr && c < nr) ? D[ii + c * nr] : (T)0;
    }
  }
  __syncthreads();
  T y[RPT];
#pragma unroll
  for (int j = 0; j < RPT; ++j) y[j] = (T)0;
#pragma unroll 8
  for (int c = 0; c < SB; ++c) {
    const T l = Ls[c][i];
#pragma unroll
    for (int j = 0; j < RPT; ++j) {
      const int r = g + 4 * j;
      if (r < nr_rhs) y[j] = fma(l, Ys[c * nr_rhs + r], y[j]);
    }
  }
  if (i < nr) {
#pragma unroll
    for (int j = 0; j < RPT; ++j) {
      const int r = g + 4 * j;
      if (r < nr_rhs) w[r0 + i + (int64_t)r * m] = y[j];
    }
  }
  __syncthreads();
  if (t == 0) {
    publish_flag(fa.flags + fa.flag_off[s] + R);
  }
}

// Backward unit: column block p of front s, accumulating L_Rp^T x_R over the row
// blocks R in [lo, hi) (R < pb: pivot rows, waited for; else update rows, whose x
// come from ancestors and were staged in W by k_bwd_init).  The final unit (row
// block p + 1) adds the chunk partials and solves x_p = Dinv_p^T (y_p - sum),
// written to W and to the caller's vector, then raises the column's flag.
// Thread t: column c = t % 64 of the block, right-hand sides r = t / 64 + 4 j.
template <class T, int RPT>
__global__ void __launch_bounds__(256, 2) k_bwd_level(const T* __restrict__ L, const T* __restrict__ Dinv, T* W, T* part,
                                                   double* __restrict__ x, SolveArgs a, FusedArgs fa) {
  __shared__ T Ls[SB][SB + 1];
  __shared__ int s_item;
  extern __shared__ __align__(16) unsigned char sm_raw[];
  T* Ws = reinterpret_cast<T*>(sm_raw);  // SB x nrhs, [row * nrhs + r]
  const int t = threadIdx.x, c = t & 63, g = t >> 6;
  if (t == 0) s_item = atomicAdd(fa.ticket, 1);
  __syncthreads();
  const int* u = fa.units + 8 * s_item;
  const int s = u[0], p = u[1], lo = u[2], hi = u[3], slot = u[4], cnt = u[5], nparts = u[6], fin = u[7];
  const int m = a.m[s], k = a.k[s], nr_rhs = a.nrhs;
  const int pb = (k + SB - 1) / SB;
  const int c0 = SB * p, wc = min(SB, k - c0);
  const T* F = L + a.l_off[s];
  T* w = W + a.w_off[s] * nr_rhs;
  const int* flags = fa.flags + fa.flag_off[s];
  T acc[RPT];
#pragma unroll
  for (int j = 0; j < RPT; ++j) acc[j] = (T)0;
  constexpr bool kPreD = RPT <= 2;
  const T* D = Dinv + fa.dinv_off[s] + (int64_t)p * SB * SB;
  T dpre[kPreD ? 16 : 1], wrow[RPT];
  if (fin) {
    if (kPreD) {
#pragma unroll
      for (int e = 0; e < 16; ++e) {
        const int q = t + 256 * e, ii = q & 63, cc = q >> 6;
        dpre[e] = (ii < wc && cc < wc) ? D[ii + cc * wc] : (T)0;
      }
    }
#pragma unroll
    for (int j = 0; j < RPT; ++j) {
      const int r = g + 4 * j;
      wrow[j] = (r < nr_rhs && c < wc) ? w[c0 + c + (int64_t)r * m] : (T)0;
    }
  }
  T* my_part = part + (int64_t)slot * SB * nr_rhs;
  T tot[RPT];
#pragma unroll
  for (int j = 0; j < RPT; ++j) tot[j] = (T)0;
  if (fin) gather_partials<T, RPT>(my_part, nparts, nr_rhs, fa.counters + cnt, fa.err, tot);
  auto rows_of = [&](int R, int& r0, int& nr) {
    r0 = (R < pb) ? SB * R : k + SB * (R - pb);
    nr = min(SB, (R < pb ? k : m) - r0);
  };
  // rows farthest from the diagonal first: their x are known earliest (update rows
  // from the ancestors, pivot blocks solved longest ago), the newest last
  T pre[16];
  if (lo < hi) {
    int r0, nr;
    rows_of(hi - 1, r0, nr);
    load_block(pre, F, m, r0, nr, c0, wc);
  }
  for (int R = hi - 1; R >= lo; --R) {
    int r0, nr;
    rows_of(R, r0, nr);
    if (R < pb && t == 0) wait_flag(flags + R, fa.err);
    __syncthreads();
    store_block(Ls, pre);
    for (int e = t; e < SB * nr_rhs; e += 256) {
      const int ii = e % SB, r = e / SB;
      Ws[ii * nr_rhs + r] = (ii < nr) ? __ldcg(w + r0 + ii + (int64_t)r * m) : (T)0;
    }
    __syncthreads();
    if (R - 1 >= lo) {
      int r1, n1;
      rows_of(R - 1, r1, n1);
      load_block(pre, F, m, r1, n1, c0, wc);
    }
#pragma unroll 8
    for (int ii = 0; ii < SB; ++ii) {
      const T l = Ls[c][ii];
#pragma unroll
      for (int j = 0; j < RPT; ++j) {
        const int r = g + 4 * j;
        if (r < nr_rhs) acc[j] = fma(l, Ws[ii * nr_rhs + r], acc[j]);
      }
    }
  }
  if (!fin) {
    publish_partial<T, RPT>(my_part, acc, nr_rhs, fa.counters + cnt);
    return;
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < RPT; ++j) {
    const int r = g + 4 * j;
    if (r < nr_rhs) Ws[c * nr_rhs + r] = (c < wc) ? wrow[j] - (tot[j] + acc[j]) : (T)0;
  }
  if constexpr (kPreD) {
    store_block(Ls, dpre);
  } else {
    for (int e = t; e < SB * SB; e += 256) {
      const int ii = e & 63, cc = e >> 6;
      Ls[cc][ii] = (ii < wc && cc < wc) ? D[ii + cc * wc] : (T)0;
    }
  }
  __syncthreads();
  T xv[RPT];
#pragma unroll
  for (int j = 0; j < RPT; ++j) xv[j] = (T)0;
#pragma unroll 8
  for (int ii = 0; ii < SB; ++ii) {
    const T l = Ls[c][ii];
#pragma unroll
    for (int j = 0; j < RPT; ++j) {
      const int r = g + 4 * j;
      if (r < nr_rhs) xv[j] = fma(l, Ws[ii * nr_rhs + r], xv[j]);
    }
  }
  if (c < wc) {
    const int pos = a.rows[a.rows_off[s] + c0 + c];
#pragma unroll
    for (int j = 0; j < RPT; ++j) {
      const int r = g + 4 * j;
      if (r < nr_rhs) {
        w[c0 + c + (int64_t)r * m] = xv[j];
        x[pos + (int64_t)r * a.ld] = (double)xv[j];
      }
    }
  }
  __syncthreads();
  if (t == 0) {
    publish_flag(fa.flags + fa.flag_off[s] + p);
  }
}

// Inverse of the lower-triangular diagonal block p of front s (w x w, w <= 64),
// stored column-major with leading dimension w at dinv_off[s] + 64 * 64 * p.
// Computed in FP64: four threads per column j run the substitution
// X[i][j] = -(sum_{j <= l < i} A[i][l] X[l][j]) / A[i][i] down the column.
template <class T>
__global__ void __launch_bounds__(256) k_diag_inverse(const T* __restrict__ L, T* __restrict__ Dinv, Fronts f,
                                                      const int64_t* __restrict__ dinv_off,
                                                      const int* __restrict__ items) {
  extern __shared__ __align__(16) unsigned char sm_raw[];
  double(*A)[SB + 1] = reinterpret_cast<double(*)[SB + 1]>(sm_raw);
  double(*X)[SB + 1] = reinterpret_cast<double(*)[SB + 1]>(sm_raw + sizeof(double) * SB * (SB + 1));
  const int s = items[2 * blockIdx.x], p = items[2 * blockIdx.x + 1];
  const int m = f.m[s], k = f.k[s];
  const int c0 = SB * p, w = min(SB, k - c0);
  const T* F = L + f.l_off[s];
  for (int q = threadIdx.x; q < SB * SB; q += blockDim.x) {
    const int i = q & 63, j = q >> 6;
    A[i][j] = (i < w && j < w && i >= j) ? (double)F[(c0 + i) + (int64_t)(c0 + j) * m] : 0.0;
  }
  __syncthreads();
  const int j = threadIdx.x >> 2, part = threadIdx.x & 3;
  const unsigned mask = 0xFu << ((threadIdx.x & 31) & ~3);
  if (j < w) {
    if (part == 0) X[j][j] = 1.0 / A[j][j];
    __syncwarp(mask);
    for (int i = j + 1; i < w; ++i) {
      double sum = 0.0;
      for (int l = j + part; l < i; l += 4) sum = fma(A[i][l], X[l][j], sum);
      sum += __shfl_xor_sync(mask, sum, 1);
      sum += __shfl_xor_sync(mask, sum, 2);
      if (part == 0) X[i][j] = -sum / A[i][i];
      __syncwarp(mask);
    }
  }
  __syncthreads();
  T* D = Dinv + dinv_off[s] + (int64_t)p * SB * SB;
  for (int q = threadIdx.x; q < w * w; q += blockDim.x) {
    const int i = q % w, jj = q / w;
    D[q] = (i >= jj) ? (T)X[i][jj] : (T)0;
  }
}

#define TDEM_CUDA_TRY(x)                                                          \
  do {                                                                             \
    cudaError_t e_ = (x);                                                          \
    if (e_ != cudaSuccess) return std::string(#x ": ") + cudaGetErrorString(e_);   \
  } while (0)

inline unsigned grid_of(int64_t ctas) { return (unsigned)ctas; }
template <class T>
constexpr size_t trsm_smem() { return sizeof(T) * (P + kTrsmRows) * (P + 1); }
template <class T>
constexpr size_t syrk_smem() { return sizeof(T) * 2 * kTileSyrk * (P + 1); }
template <class T>
constexpr size_t big_smem() { return sizeof(T) * 2 * KC * (kTileBig + 1); }

template <class T>
std::string set_attributes() {
  TDEM_CUDA_TRY(cudaFuncSetAttribute(k_trsm<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)trsm_smem<T>()));
  TDEM_CUDA_TRY(cudaFuncSetAttribute(k_syrk_panel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)syrk_smem<T>()));
  TDEM_CUDA_TRY(cudaFuncSetAttribute(k_syrk_big<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)big_smem<T>()));
  TDEM_CUDA_TRY(cudaFuncSetAttribute(k_fwd_diag<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024));
  TDEM_CUDA_TRY(cudaFuncSetAttribute(k_bwd_diag<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024));
  TDEM_CUDA_TRY(cudaFuncSetAttribute(k_fwd_update<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024));
  return "";
}

template <class T>
int launch_factor(const Symbolic& sy, T* L, T* U, const double* vals, const int64_t* entry, Fronts fr,
                  const int* parent, const int64_t* rel_off, const int* rel, const int* tasks,
                  const int64_t* prefix, int* err, const int* c0, bool use_tc, cudaStream_t s) {
  int launches = 0;
  cudaMemsetAsync(L, 0, sizeof(T) * sy.nnz_l, s);
  {
    const int64_t nnz = sy.nnz_lower;
    const unsigned g = (unsigned)std::min<int64_t>((nnz + 255) / 256, 148 * 32);
    if (nnz > 0) {
      k_scatter_entries<T><<<g, 256, 0, s>>>(L, entry, vals, nnz);
      ++launches;
    }
  }
  for (const LevelPlan& lp : sy.levels) {
    if (lp.assemble.ctas > 0) {
      k_zero_u<T><<<grid_of(lp.assemble.ctas), 256, 0, s>>>(U, fr, tasks + lp.assemble.off, prefix + lp.assemble.pre,
                                                           lp.assemble.count);
      ++launches;
    }
    for (const TaskList& tl : lp.extend_slots) {
      if (tl.ctas == 0) continue;
      k_extend_add<T><<<grid_of(tl.ctas), 256, 0, s>>>(L, U, fr, parent, rel_off, rel, tasks + tl.off,
                                                       prefix + tl.pre, tl.count);
      ++launches;
    }
    for (const PanelStep& ps : lp.panels) {
      k_potrf<T><<<ps.potrf.count, 256, 0, s>>>(L, fr, tasks + ps.potrf.off, ps.j0, err, c0);
      ++launches;
      if (ps.trsm.ctas > 0) {
        k_trsm<T><<<grid_of(ps.trsm.ctas), kTrsmRows, trsm_smem<T>(), s>>>(L, fr, tasks + ps.trsm.off,
                                                                           prefix + ps.trsm.pre, ps.trsm.count, ps.j0);
        ++launches;
      }
      if (ps.syrk.ctas > 0) {
        k_syrk_panel<T><<<grid_of(ps.syrk.ctas), 256, syrk_smem<T>(), s>>>(L, fr, tasks + ps.syrk.off,
                                                                           prefix + ps.syrk.pre, ps.syrk.count, ps.j0);
        ++launches;
      }
      if (ps.syrk_big.ctas > 0) {
        if (std::is_same<T, float>::value && use_tc)
          launch_syrk_tc((float*)L, (float*)U, fr.l_off, fr.u_off, fr.m, fr.k, tasks + ps.syrk_big.off,
                         prefix + ps.syrk_big.pre, ps.syrk_big.count, ps.syrk_big.ctas, ps.j0, err, s);
        else
          k_syrk_big<T><<<grid_of(ps.syrk_big.ctas), 256, big_smem<T>(), s>>>(
              L, U, fr, tasks + ps.syrk_big.off, prefix + ps.syrk_big.pre, ps.syrk_big.count, ps.j0);
        ++launches;
      }
    }
  }
  return launches;
}

template <class T>
int launch_solve(const Symbolic& sy, const T* L, T* W, T* part, const double* b, double* x, SolveArgs a,
                 const int* parent, const int64_t* rel_off, const int* rel, const int* tasks, const int64_t* prefix,
                 cudaStream_t s) {
  int launches = 0;
  const size_t ysm = sizeof(T) * P * a.nrhs;
  for (const LevelPlan& lp : sy.levels) {
    k_fwd_init<T><<<grid_of(lp.assemble.ctas), kSolveRows, 0, s>>>(W, b, a, tasks + lp.assemble.off,
                                                                   prefix + lp.assemble.pre, lp.assemble.count);
    ++launches;
    for (const TaskList& tl : lp.extend_vec) {
      if (tl.ctas == 0) continue;
      k_fwd_extend<T><<<grid_of(tl.ctas), kSolveRows, 0, s>>>(W, a, parent, rel_off, rel, tasks + tl.off,
                                                              prefix + tl.pre, tl.count);
      ++launches;
    }
    for (const PanelStep& ps : lp.panels) {
      k_fwd_diag<T><<<ps.potrf.count, 256, ysm, s>>>(L, W, a, tasks + ps.potrf.off, ps.j0);
      ++launches;
      if (ps.solve_upd.ctas > 0) {
        k_fwd_update<T><<<grid_of(ps.solve_upd.ctas), kSolveRows, ysm, s>>>(
            L, W, a, tasks + ps.solve_upd.off, prefix + ps.solve_upd.pre, ps.solve_upd.count, ps.j0);
        ++launches;
      }
    }
  }
  for (int l = (int)sy.levels.size() - 1; l >= 0; --l) {
    const LevelPlan& lp = sy.levels[l];
    k_bwd_init<T><<<grid_of(lp.assemble.ctas), kSolveRows, 0, s>>>(W, x, a, tasks + lp.assemble.off,
                                                                   prefix + lp.assemble.pre, lp.assemble.count);
    ++launches;
    for (int p = (int)lp.panels.size() - 1; p >= 0; --p) {
      const PanelStep& ps = lp.panels[p];
      if (ps.solve_upd.ctas > 0) {
        k_bwd_partial<T><<<grid_of(ps.solve_upd.ctas), kSolveRows, 0, s>>>(
            L, W, a, part, tasks + ps.solve_upd.off, prefix + ps.solve_upd.pre, ps.solve_upd.count, ps.j0);
        ++launches;
      }
      k_bwd_diag<T><<<ps.potrf.count, 256, ysm, s>>>(L, W, a, part, tasks + ps.solve_upd.off,
                                                      prefix + ps.solve_upd.pre, ps.j0);
      ++launches;
    }
    k_bwd_store<T><<<grid_of(lp.assemble.ctas), kSolveRows, 0, s>>>(W, x, a, tasks + lp.assemble.off,
                                                                    prefix + lp.assemble.pre, lp.assemble.count);
    ++launches;
  }
  return launches;
}

template <class T, int RPT>
void launch_level_solves(const Symbolic& sy, const T* L, const T* Dinv, T* W, T* part, const double* b, double* x,
                         SolveArgs a, const int* parent, const int64_t* rel_off, const int* rel, const int* tasks,
                         const int64_t* prefix, FusedArgs fa, int* sync, int& launches, cudaStream_t s) {
  const int nlev = (int)sy.levels.size();
  int* tickets = sync;
  int* fflags = sync + 2 * nlev;
  int* bflags = fflags + sy.n_flags;
  fa.counters = bflags + sy.n_flags;
  cudaMemsetAsync(sync, 0, sizeof(int) * (2 * nlev + 2 * sy.n_flags + sy.n_counters), s);
  const size_t ysm = sizeof(T) * SB * a.nrhs;
  for (int l = 0; l < nlev; ++l) {
    const LevelPlan& lp = sy.levels[l];
    k_fwd_init<T><<<grid_of(lp.assemble.ctas), kSolveRows, 0, s>>>(W, b, a, tasks + lp.assemble.off,
                                                                   prefix + lp.assemble.pre, lp.assemble.count);
    ++launches;
    for (const TaskList& tl : lp.extend_vec) {
      if (tl.ctas == 0) continue;
      k_fwd_extend<T><<<grid_of(tl.ctas), kSolveRows, 0, s>>>(W, a, parent, rel_off, rel, tasks + tl.off,
                                                              prefix + tl.pre, tl.count);
      ++launches;
    }
    FusedArgs f = fa;
    f.units = fa.units + 8 * lp.fwd_off;
    f.ticket = tickets + 2 * l;
    f.flags = fflags;
    k_fwd_level<T, RPT><<<grid_of(lp.fwd_count), 256, ysm, s>>>(L, Dinv, W, part, a, f);
    ++launches;
  }
  for (int l = nlev - 1; l >= 0; --l) {
    const LevelPlan& lp = sy.levels[l];
    k_bwd_init<T><<<grid_of(lp.assemble.ctas), kSolveRows, 0, s>>>(W, x, a, tasks + lp.assemble.off,
                                                                   prefix + lp.assemble.pre, lp.assemble.count);
    ++launches;
    FusedArgs f = fa;
    f.units = fa.units + 8 * lp.bwd_off;
    f.ticket = tickets + 2 * l + 1;
    f.flags = bflags;
    k_bwd_level<T, RPT><<<grid_of(lp.bwd_count), 256, ysm, s>>>(L, Dinv, W, part, x, a, f);
    ++launches;
  }
}

template <class T>
int launch_solve_fused(const Symbolic& sy, const T* L, const T* Dinv, T* W, T* part, const double* b, double* x,
                       SolveArgs a, const int* parent, const int64_t* rel_off, const int* rel, const int* tasks,
                       const int64_t* prefix, FusedArgs fa, int* sync, cudaStream_t s) {
  int launches = 0;
  if (a.nrhs <= 4)
    launch_level_solves<T, 1>(sy, L, Dinv, W, part, b, x, a, parent, rel_off, rel, tasks, prefix, fa, sync, launches, s);
  else if (a.nrhs <= 8)
    launch_level_solves<T, 2>(sy, L, Dinv, W, part, b, x, a, parent, rel_off, rel, tasks, prefix, fa, sync, launches, s);
  else if (a.nrhs <= 16)
    launch_level_solves<T, 4>(sy, L, Dinv, W, part, b, x, a, parent, rel_off, rel, tasks, prefix, fa, sync, launches, s);
  else if (a.nrhs <= 32)
    launch_level_solves<T, 8>(sy, L, Dinv, W, part, b, x, a, parent, rel_off, rel, tasks, prefix, fa, sync, launches, s);
  else
    launch_level_solves<T, 16>(sy, L, Dinv, W, part, b, x, a, parent, rel_off, rel, tasks, prefix, fa, sync, launches,
                               s);
  return launches;
}

template <class T>
std::string set_fused_attributes() {
  const int ysm = (int)(sizeof(T) * SB * kMaxRhs);
  TDEM_CUDA_TRY(cudaFuncSetAttribute(k_fwd_level<T, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, ysm));
  TDEM_CUDA_TRY(cudaFuncSetAttribute(k_fwd_level<T, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, ysm));
  TDEM_CUDA_TRY(cudaFuncSetAttribute(k_fwd_level<T, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, ysm));
  TDEM_CUDA_TRY(cudaFuncSetAttribute(k_fwd_level<T, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, ysm));
  TDEM_CUDA_TRY(cudaFuncSetAttribute(k_fwd_level<T, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, ysm));
  TDEM_CUDA_TRY(cudaFuncSetAttribute(k_bwd_level<T, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, ysm));
  TDEM_CUDA_TRY(cudaFuncSetAttribute(k_bwd_level<T, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, ysm));
  TDEM_CUDA_TRY(cudaFuncSetAttribute(k_bwd_level<T, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, ysm));
  TDEM_CUDA_TRY(cudaFuncSetAttribute(k_bwd_level<T, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, ysm));
  TDEM_CUDA_TRY(cudaFuncSetAttribute(k_bwd_level<T, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, ysm));
  TDEM_CUDA_TRY(cudaFuncSetAttribute(k_diag_inverse<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)(2 * sizeof(double) * SB * (SB + 1))));
  return "";
}

}  // namespace

GpuCholesky::~GpuCholesky() {
  if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
  for (void* p : allocs_) cudaFree(p);
}

std::string GpuCholesky::alloc(void** p, size_t bytes) {
  *p = nullptr;
  if (bytes == 0) bytes = 16;
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) return std::string("cudaMalloc: ") + cudaGetErrorString(e);
  allocs_.push_back(*p);
  bytes_ += bytes;
  return "";
}

template <class T>
std::string GpuCholesky::upload(T** dst, const std::vector<T>& src, cudaStream_t s) {
  std::string e = alloc((void**)dst, src.size() * sizeof(T));
  if (!e.empty()) return e;
  if (!src.empty())
    TDEM_CUDA_TRY(cudaMemcpyAsync(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice, s));
  return "";
}

int64_t GpuCholesky::bytes_needed(const Symbolic& sy, int nrhs_max, int precision_bytes) {
  const int64_t el = (precision_bytes == 4) ? 4 : 8, nr = std::max(1, nrhs_max);
  int64_t b = el * (sy.nnz_l + sy.u_elems + sy.wvec_elems * nr + sy.solve_partials * nr + sy.dinv_elems +
                    sy.solve_slots * kPanel * nr);
  b += 8 * (int64_t)(sy.l_off.size() + sy.u_off.size() + sy.wvec_off.size() + sy.entry_dst.size() +
                     sy.rel_off.size() + sy.rows_off.size() + sy.task_prefix.size() + sy.flag_off.size() +
                     sy.dinv_off.size());
  b += 4 * (int64_t)(sy.front_m.size() + sy.front_k.size() + sy.rel.size() + sy.rows_all.size() + sy.tasks.size() +
                     sy.front_parent.size() + sy.front_c0.size() + sy.solve_items.size() + sy.solve_units.size() +
                     2 * sy.levels.size() + 2 * sy.n_flags + sy.n_counters + 4);
  return b;
}

std::string GpuCholesky::setup(Symbolic&& sy, const std::vector<int>& perm_to_vec, int nrhs_max,
                               cudaStream_t s, int precision_bytes) {
  sy_ = std::move(sy);
  nrhs_max_ = std::max(1, nrhs_max);
  elem_ = (precision_bytes == 4) ? 4 : 8;
  if ((int)perm_to_vec.size() != sy_.n) return "perm_to_vec size mismatch";
  if (nrhs_max_ > kMaxRhs) return "too many right-hand sides";
  std::string e;
  if (!(e = alloc(&d_L_, elem_ * std::max<int64_t>(1, sy_.nnz_l))).empty()) return e;
  if (!(e = alloc(&d_U_, elem_ * std::max<int64_t>(1, sy_.u_elems))).empty()) return e;
  if (!(e = alloc(&d_W_, elem_ * std::max<int64_t>(1, sy_.wvec_elems) * nrhs_max_)).empty()) return e;
  if (!(e = alloc(&d_part_, elem_ * std::max<int64_t>(1, sy_.solve_partials) * nrhs_max_)).empty()) return e;
  if (!(e = upload(&d_l_off_, sy_.l_off, s)).empty()) return e;
  if (!(e = upload(&d_u_off_, sy_.u_off, s)).empty()) return e;
  if (!(e = upload(&d_w_off_, sy_.wvec_off, s)).empty()) return e;
  if (!(e = upload(&d_m_, sy_.front_m, s)).empty()) return e;
  if (!(e = upload(&d_k_, sy_.front_k, s)).empty()) return e;
  if (!(e = upload(&d_entry_, sy_.entry_dst, s)).empty()) return e;
  if (!(e = upload(&d_rel_off_, sy_.rel_off, s)).empty()) return e;
  if (!(e = upload(&d_rel_, sy_.rel, s)).empty()) return e;
  if (!(e = upload(&d_rows_off_, sy_.rows_off, s)).empty()) return e;
  {
    std::vector<int> rows(sy_.rows_all.size());
    for (size_t i = 0; i < rows.size(); ++i) rows[i] = perm_to_vec[sy_.rows_all[i]];
    if (!(e = upload(&d_rows_, rows, s)).empty()) return e;
  }
  if (!(e = upload(&d_tasks_, sy_.tasks, s)).empty()) return e;
  if (!(e = upload(&d_prefix_, sy_.task_prefix, s)).empty()) return e;
  if (!(e = upload(&d_parent_, sy_.front_parent, s)).empty()) return e;
  if (!(e = upload(&d_c0_, sy_.front_c0, s)).empty()) return e;
  if (!(e = upload(&d_items_, sy_.solve_items, s)).empty()) return e;
  if (!(e = upload(&d_flag_off_, sy_.flag_off, s)).empty()) return e;
  if (!(e = upload(&d_dinv_off_, sy_.dinv_off, s)).empty()) return e;
  if (!(e = alloc(&d_dinv_, elem_ * std::max<int64_t>(1, sy_.dinv_elems))).empty()) return e;
  if (!(e = upload(&d_units_, sy_.solve_units, s)).empty()) return e;
  if (!(e = alloc(&d_spart_, elem_ * std::max<int64_t>(1, sy_.solve_slots) * kPanel * nrhs_max_)).empty()) return e;
  if (!(e = alloc((void**)&d_sync_,
                  sizeof(int) * (2 * sy_.levels.size() + 2 * sy_.n_flags + sy_.n_counters + 1))).empty())
    return e;
  if (!(e = alloc((void**)&d_err_, 3 * sizeof(int))).empty()) return e;
  TDEM_CUDA_TRY(cudaMemsetAsync(d_err_, 0, 3 * sizeof(int), s));
  if (elem_ == 4 && tc_update_ && !(e = tc_update_setup()).empty()) return e;
  if (!(e = (elem_ == 4 ? set_attributes<float>() : set_attributes<double>())).empty()) return e;
  if (!(e = (elem_ == 4 ? set_fused_attributes<float>() : set_fused_attributes<double>())).empty()) return e;
  TDEM_CUDA_TRY(cudaStreamSynchronize(s));
  return "";
}

void GpuCholesky::factor(const double* d_vals, cudaStream_t s) {
  Fronts fr{d_l_off_, d_u_off_, d_m_, d_k_};
  const unsigned ni = (unsigned)sy_.inv_count;
  const size_t ism = 2 * sizeof(double) * SB * (SB + 1);
  if (elem_ == 4) {
    launches_factor_ = launch_factor<float>(sy_, (float*)d_L_, (float*)d_U_, d_vals, d_entry_, fr, d_parent_,
                                            d_rel_off_, d_rel_, d_tasks_, d_prefix_, d_err_, d_c0_, tc_update_, s);
    if (ni) k_diag_inverse<float><<<ni, 256, ism, s>>>((const float*)d_L_, (float*)d_dinv_, fr, d_dinv_off_,
                                                       d_items_ + 2 * sy_.inv_off);
  } else {
    launches_factor_ = launch_factor<double>(sy_, (double*)d_L_, (double*)d_U_, d_vals, d_entry_, fr, d_parent_,
                                             d_rel_off_, d_rel_, d_tasks_, d_prefix_, d_err_, d_c0_, false, s);
    if (ni) k_diag_inverse<double><<<ni, 256, ism, s>>>((const double*)d_L_, (double*)d_dinv_, fr, d_dinv_off_,
                                                        d_items_ + 2 * sy_.inv_off);
  }
  if (ni) ++launches_factor_;
}

void GpuCholesky::solve(const double* d_b, double* d_x, int64_t ld, int nrhs, cudaStream_t s) {
  SolveArgs a{d_l_off_, d_w_off_, d_m_, d_k_, d_rows_off_, d_rows_, nrhs, ld};
  if (!panel_solve_) {
    FusedArgs fa{d_units_, nullptr, nullptr, nullptr, d_flag_off_, d_dinv_off_, d_err_};
    if (elem_ == 4)
      launches_solve_ = launch_solve_fused<float>(sy_, (const float*)d_L_, (const float*)d_dinv_, (float*)d_W_,
                                                  (float*)d_spart_, d_b, d_x, a, d_parent_, d_rel_off_, d_rel_,
                                                  d_tasks_, d_prefix_, fa, d_sync_, s);
    else
      launches_solve_ = launch_solve_fused<double>(sy_, (const double*)d_L_, (const double*)d_dinv_, (double*)d_W_,
                                                   (double*)d_spart_, d_b, d_x, a, d_parent_, d_rel_off_, d_rel_,
                                                   d_tasks_, d_prefix_, fa, d_sync_, s);
    return;
  }
  if (elem_ == 4)
    launches_solve_ = launch_solve<float>(sy_, (const float*)d_L_, (float*)d_W_, (float*)d_part_, d_b, d_x, a,
                                          d_parent_, d_rel_off_, d_rel_, d_tasks_, d_prefix_, s);
  else
    launches_solve_ = launch_solve<double>(sy_, (const double*)d_L_, (double*)d_W_, (double*)d_part_, d_b, d_x, a,
                                           d_parent_, d_rel_off_, d_rel_, d_tasks_, d_prefix_, s);
}

std::string GpuCholesky::solve_graph(const double* d_b, double* d_x, int64_t ld, int nrhs, cudaStream_t s) {
  if (!graph_exec_ || g_b_ != d_b || g_x_ != d_x || g_ld_ != ld || g_nrhs_ != nrhs) {
    if (graph_exec_) {
      cudaGraphExecDestroy(graph_exec_);
      graph_exec_ = nullptr;
    }
    cudaGraph_t g = nullptr;
    TDEM_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    solve(d_b, d_x, ld, nrhs, s);
    TDEM_CUDA_TRY(cudaStreamEndCapture(s, &g));
    const cudaError_t ie = cudaGraphInstantiate(&graph_exec_, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) {
      graph_exec_ = nullptr;
      return std::string("cudaGraphInstantiate: ") + cudaGetErrorString(ie);
    }
    g_b_ = d_b;
    g_x_ = d_x;
    g_ld_ = ld;
    g_nrhs_ = nrhs;
  }
  TDEM_CUDA_TRY(cudaGraphLaunch(graph_exec_, s));
  return "";
}

int GpuCholesky::status(cudaStream_t s) {
  int h = 0;
  cudaMemcpyAsync(&h, d_err_, sizeof(int), cudaMemcpyDeviceToHost, s);
  cudaStreamSynchronize(s);
  return h;
}

int GpuCholesky::solve_status(cudaStream_t s) {
  int h[2] = {0, 0};
  cudaMemcpyAsync(h, d_err_ + 1, 2 * sizeof(int), cudaMemcpyDeviceToHost, s);
  cudaStreamSynchronize(s);
  return h[0] ? 1 : (h[1] ? 2 : 0);
}

}  // namespace tdem
