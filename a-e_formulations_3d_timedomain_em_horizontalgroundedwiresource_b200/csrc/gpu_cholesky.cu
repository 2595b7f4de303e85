// GPU multifrontal Cholesky (FP64): batched dense front kernels driven level by
// level and panel by panel from the host plan in symbolic.h.
//
// Layout in HBM
//   L   persistent factor; front s owns an m x k column-major block (ld = m) at l_off[s]
//   U   update workspace; front s owns an r x r block (ld = r, r = m - k) at u_off[s]
//       while it waits for its parent (offsets planned on the host, first fit)
//   W   solve front vectors, m x nrhs per front at w_off[s] * nrhs (ld = m)
// Every kernel receives a task list (fronts + CTA prefix sums) and finds its
// front by binary search over the prefix, so one launch covers every front of a
// level that takes part in the current panel.
#include "gpu_cholesky.h"

#include <algorithm>
#include <cstdio>

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
__device__ __forceinline__ double* felem(double* L, double* U, int64_t lo, int64_t uo, int m, int k,
                                         int i, int c) {
  return (c < k) ? L + lo + i + (int64_t)c * m : U + uo + (i - k) + (int64_t)(c - k) * (m - k);
}

// ---------------------------------------------------------------------------
// factorization kernels
// ---------------------------------------------------------------------------
__global__ void k_scatter_entries(double* __restrict__ L, const int64_t* __restrict__ dst,
                                  const double* __restrict__ val, int64_t nnz) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nnz;
       q += (int64_t)gridDim.x * blockDim.x)
    L[dst[q]] = val[q];
}

// Zero the update blocks of the fronts of one level (kSolveRows columns per CTA).
__global__ void k_zero_u(double* __restrict__ U, Fronts f, const int* __restrict__ fronts,
                         const int64_t* __restrict__ prefix, int count) {
  const int idx = find_task(prefix, count, blockIdx.x);
  const int s = fronts[idx];
  const int m = f.m[s], k = f.k[s], r = m - k;
  const int64_t t = blockIdx.x - prefix[idx];
  const int c0 = (int)t * kSolveRows, c1 = min(r, c0 + kSolveRows);
  double* u = U + f.u_off[s];
  for (int c = c0; c < c1; ++c)
    for (int i = threadIdx.x; i < r; i += blockDim.x) u[i + (int64_t)c * r] = 0.0;
}

// Extend-add of the children's update blocks into their parents (one child per
// parent per launch, so no two CTAs write the same parent element).  One warp
// per child column, 8 columns per CTA.
__global__ void k_extend_add(double* __restrict__ L, double* __restrict__ U, Fronts f,
                             const int* __restrict__ parent, const int64_t* __restrict__ rel_off,
                             const int* __restrict__ rel, const int* __restrict__ kids,
                             const int64_t* __restrict__ prefix, int count) {
  const int idx = find_task(prefix, count, blockIdx.x);
  const int c = kids[idx];
  const int p = parent[c];
  const int mc = f.m[c], kc = f.k[c], rc = mc - kc;
  const int mp = f.m[p], kp = f.k[p];
  const int64_t lo = f.l_off[p], uo = f.u_off[p];
  const int* rl = rel + rel_off[c];
  const double* uc = U + f.u_off[c];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int b = (int)(blockIdx.x - prefix[idx]) * 8 + warp;
  if (b >= rc) return;
  const int pc = rl[b];
  for (int a = b + lane; a < rc; a += 32) {
    const int pr = rl[a];
    *felem(L, U, lo, uo, mp, kp, pr, pc) += uc[a + (int64_t)b * rc];
  }
}

// Cholesky of the w x w diagonal block of panel [j0, j0 + w) (one CTA per front).
__global__ void k_potrf(double* __restrict__ L, Fronts f, const int* __restrict__ fronts, int j0,
                        int* __restrict__ err, const int* __restrict__ c0_of) {
  __shared__ double A[P][P + 1];
  const int s = fronts[blockIdx.x];
  const int m = f.m[s], k = f.k[s];
  const int w = min(P, k - j0);
  double* F = L + f.l_off[s];
  for (int idx = threadIdx.x; idx < w * w; idx += blockDim.x) {
    const int i = idx % w, j = idx / w;
    A[i][j] = (i >= j) ? F[(j0 + i) + (int64_t)(j0 + j) * m] : 0.0;
  }
  __syncthreads();
  for (int j = 0; j < w; ++j) {
    if (threadIdx.x == 0) {
      double d = A[j][j];
      if (!(d > 0.0)) {
        atomicCAS(err, 0, c0_of[s] + j0 + j + 1);
        d = 1.0;
      }
      A[j][j] = sqrt(d);
    }
    __syncthreads();
    const double inv = 1.0 / A[j][j];
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
__global__ void __launch_bounds__(kTrsmRows) k_trsm(double* __restrict__ L, Fronts f,
                                                    const int* __restrict__ fronts,
                                                    const int64_t* __restrict__ prefix, int count, int j0) {
  extern __shared__ double sm_trsm[];
  double(*Ld)[P + 1] = reinterpret_cast<double(*)[P + 1]>(sm_trsm);
  double(*X)[P + 1] = reinterpret_cast<double(*)[P + 1]>(sm_trsm + P * (P + 1));
  const int idx = find_task(prefix, count, blockIdx.x);
  const int s = fronts[idx];
  const int m = f.m[s], k = f.k[s];
  const int w = min(P, k - j0), j1 = j0 + w;
  double* F = L + f.l_off[s];
  const int r0 = j1 + (int)(blockIdx.x - prefix[idx]) * kTrsmRows;
  for (int idx2 = threadIdx.x; idx2 < w * w; idx2 += blockDim.x) {
    const int i = idx2 % w, j = idx2 / w;
    Ld[i][j] = (i >= j) ? F[(j0 + i) + (int64_t)(j0 + j) * m] : 0.0;
  }
  for (int idx2 = threadIdx.x; idx2 < kTrsmRows * w; idx2 += blockDim.x) {
    const int i = idx2 % kTrsmRows, j = idx2 / kTrsmRows;
    const int row = r0 + i;
    X[i][j] = (row < m) ? F[row + (int64_t)(j0 + j) * m] : 0.0;
  }
  __syncthreads();
  const int t = threadIdx.x;
  for (int c = 0; c < w; ++c) {
    double v = X[t][c];
    for (int cc = 0; cc < c; ++cc) v -= X[t][cc] * Ld[c][cc];
    X[t][c] = v / Ld[c][c];
  }
  __syncthreads();
  for (int idx2 = threadIdx.x; idx2 < kTrsmRows * w; idx2 += blockDim.x) {
    const int i = idx2 % kTrsmRows, j = idx2 / kTrsmRows;
    const int row = r0 + i;
    if (row < m) F[row + (int64_t)(j0 + j) * m] = X[i][j];
  }
}

// Trailing update F[j1:m, j1:m] -= X X^T (lower triangle), X = panel rows [j1, m).
// One 64 x 64 tile per CTA, 256 threads with 4 x 4 outputs each.
__global__ void __launch_bounds__(256) k_syrk(double* __restrict__ L, double* __restrict__ U, Fronts f,
                                              const int* __restrict__ fronts,
                                              const int64_t* __restrict__ prefix, int count, int j0) {
  constexpr int T = kTileSyrk;
  extern __shared__ double sm_syrk[];
  double(*As)[P + 1] = reinterpret_cast<double(*)[P + 1]>(sm_syrk);
  double(*Bs)[P + 1] = reinterpret_cast<double(*)[P + 1]>(sm_syrk + T * (P + 1));
  const int idx = find_task(prefix, count, blockIdx.x);
  const int s = fronts[idx];
  const int m = f.m[s], k = f.k[s];
  const int w = min(P, k - j0), j1 = j0 + w;
  const int64_t lo = f.l_off[s], uo = f.u_off[s];
  const double* F = L + lo;
  const int64_t t = blockIdx.x - prefix[idx];
  // decode the lower-triangle tile index t -> (bi, bj), bj <= bi
  int bi = (int)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
  while ((int64_t)(bi + 1) * (bi + 2) / 2 <= t) ++bi;
  while ((int64_t)bi * (bi + 1) / 2 > t) --bi;
  const int bj = (int)(t - (int64_t)bi * (bi + 1) / 2);
  const int r0 = j1 + bi * T, c0 = j1 + bj * T;
  for (int q = threadIdx.x; q < T * w; q += blockDim.x) {
    const int i = q % T, p = q / T;
    As[i][p] = (r0 + i < m) ? F[(r0 + i) + (int64_t)(j0 + p) * m] : 0.0;
    Bs[i][p] = (c0 + i < m) ? F[(c0 + i) + (int64_t)(j0 + p) * m] : 0.0;
  }
  __syncthreads();
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  double acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
  for (int p = 0; p < w; ++p) {
    double av[4], bv[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) av[a] = As[tx + 16 * a][p];
#pragma unroll
    for (int b = 0; b < 4; ++b) bv[b] = Bs[ty + 16 * b][p];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) acc[a][b] = fma(av[a], bv[b], acc[a][b]);
  }
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const int r = r0 + tx + 16 * a;
    if (r >= m) continue;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int c = c0 + ty + 16 * b;
      if (c >= m || c > r) continue;
      *felem(L, U, lo, uo, m, k, r, c) -= acc[a][b];
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

__global__ void k_fwd_init(double* __restrict__ W, const double* __restrict__ b, SolveArgs a,
                           const int* __restrict__ fronts, const int64_t* __restrict__ prefix, int count) {
  const int idx = find_task(prefix, count, blockIdx.x);
  const int s = fronts[idx];
  const int m = a.m[s], k = a.k[s];
  const int i = (int)(blockIdx.x - prefix[idx]) * kSolveRows + threadIdx.x;
  if (i >= m) return;
  double* w = W + a.w_off[s] * a.nrhs;
  const int pos = (i < k) ? a.rows[a.rows_off[s] + i] : -1;
  for (int r = 0; r < a.nrhs; ++r) w[i + (int64_t)r * m] = (i < k) ? b[pos + r * a.ld] : 0.0;
}

__global__ void k_fwd_extend(double* __restrict__ W, SolveArgs a, const int* __restrict__ parent,
                             const int64_t* __restrict__ rel_off, const int* __restrict__ rel,
                             const int* __restrict__ kids, const int64_t* __restrict__ prefix, int count) {
  const int idx = find_task(prefix, count, blockIdx.x);
  const int c = kids[idx], p = parent[c];
  const int mc = a.m[c], kc = a.k[c], rc = mc - kc, mp = a.m[p];
  const int i = (int)(blockIdx.x - prefix[idx]) * kSolveRows + threadIdx.x;
  if (i >= rc) return;
  const double* wc = W + a.w_off[c] * a.nrhs;
  double* wp = W + a.w_off[p] * a.nrhs;
  const int pr = rel[rel_off[c] + i];
  for (int r = 0; r < a.nrhs; ++r) wp[pr + (int64_t)r * mp] += wc[kc + i + (int64_t)r * mc];
}

// Forward diagonal-block solve of panel [j0, j0 + w) (one CTA per front).
__global__ void k_fwd_diag(const double* __restrict__ L, double* __restrict__ W, SolveArgs a,
                           const int* __restrict__ fronts, int j0) {
  __shared__ double Ld[P][P + 1];
  extern __shared__ double Y[];  // w x nrhs
  const int s = fronts[blockIdx.x];
  const int m = a.m[s], k = a.k[s];
  const int w = min(P, k - j0);
  const double* F = L + a.l_off[s];
  double* wv = W + a.w_off[s] * a.nrhs;
  const int nr = a.nrhs;
  for (int q = threadIdx.x; q < w * w; q += blockDim.x) {
    const int i = q % w, j = q / w;
    Ld[i][j] = (i >= j) ? F[(j0 + i) + (int64_t)(j0 + j) * m] : 0.0;
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
__global__ void __launch_bounds__(kSolveRows) k_fwd_update(const double* __restrict__ L,
                                                           double* __restrict__ W, SolveArgs a,
                                                           const int* __restrict__ fronts,
                                                           const int64_t* __restrict__ prefix,
                                                           int count, int j0) {
  extern __shared__ double Y[];  // P x nrhs
  const int idx = find_task(prefix, count, blockIdx.x);
  const int s = fronts[idx];
  const int m = a.m[s], k = a.k[s];
  const int w = min(P, k - j0), j1 = j0 + w;
  const double* F = L + a.l_off[s];
  double* wv = W + a.w_off[s] * a.nrhs;
  const int nr = a.nrhs;
  for (int q = threadIdx.x; q < w * nr; q += blockDim.x) {
    const int i = q % w, r = q / w;
    Y[i + r * P] = wv[j0 + i + (int64_t)r * m];
  }
  __syncthreads();
  const int row = j1 + (int)(blockIdx.x - prefix[idx]) * kSolveRows + threadIdx.x;
  if (row >= m) return;
  for (int r = 0; r < nr; ++r) {
    double acc = 0.0;
    for (int c = 0; c < w; ++c) acc = fma(F[row + (int64_t)(j0 + c) * m], Y[c + r * P], acc);
    wv[row + (int64_t)r * m] -= acc;
  }
}

__global__ void k_bwd_init(double* __restrict__ W, const double* __restrict__ x, SolveArgs a,
                           const int* __restrict__ fronts, const int64_t* __restrict__ prefix, int count) {
  const int idx = find_task(prefix, count, blockIdx.x);
  const int s = fronts[idx];
  const int m = a.m[s], k = a.k[s];
  const int i = (int)(blockIdx.x - prefix[idx]) * kSolveRows + threadIdx.x;
  if (i < k || i >= m) return;
  double* w = W + a.w_off[s] * a.nrhs;
  const int pos = a.rows[a.rows_off[s] + i];
  for (int r = 0; r < a.nrhs; ++r) w[i + (int64_t)r * m] = x[pos + r * a.ld];
}

// Partial sums of L[j1:m, panel]^T W[j1:m] over one row chunk.
__global__ void __launch_bounds__(kSolveRows) k_bwd_partial(const double* __restrict__ L,
                                                            const double* __restrict__ W, SolveArgs a,
                                                            double* __restrict__ part,
                                                            const int* __restrict__ fronts,
                                                            const int64_t* __restrict__ prefix,
                                                            int count, int j0) {
  __shared__ double red[kSolveRows / 32][P];
  const int idx = find_task(prefix, count, blockIdx.x);
  const int s = fronts[idx];
  const int m = a.m[s], k = a.k[s];
  const int w = min(P, k - j0), j1 = j0 + w;
  const double* F = L + a.l_off[s];
  const double* wv = W + a.w_off[s] * a.nrhs;
  const int row = j1 + (int)(blockIdx.x - prefix[idx]) * kSolveRows + threadIdx.x;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int r = 0; r < a.nrhs; ++r) {
    const double xv = (row < m) ? wv[row + (int64_t)r * m] : 0.0;
    for (int c = 0; c < w; ++c) {
      double v = (row < m) ? F[row + (int64_t)(j0 + c) * m] * xv : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      if (lane == 0) red[warp][c] = v;
    }
    __syncthreads();
    if (threadIdx.x < w) {
      double v = 0.0;
      for (int q = 0; q < kSolveRows / 32; ++q) v += red[q][threadIdx.x];
      part[((int64_t)blockIdx.x * a.nrhs + r) * P + threadIdx.x] = v;
    }
    __syncthreads();
  }
}

// Backward diagonal-block solve of panel [j0, j0 + w) after subtracting the partials.
__global__ void k_bwd_diag(const double* __restrict__ L, double* __restrict__ W, SolveArgs a,
                           const double* __restrict__ part, const int* __restrict__ fronts,
                           const int64_t* __restrict__ prefix, int j0) {
  __shared__ double Ld[P][P + 1];
  extern __shared__ double Y[];
  const int s = fronts[blockIdx.x];
  const int m = a.m[s], k = a.k[s];
  const int w = min(P, k - j0);
  const double* F = L + a.l_off[s];
  double* wv = W + a.w_off[s] * a.nrhs;
  const int nr = a.nrhs;
  const int64_t b0 = prefix[blockIdx.x], b1 = prefix[blockIdx.x + 1];
  for (int q = threadIdx.x; q < w * w; q += blockDim.x) {
    const int i = q % w, j = q / w;
    Ld[i][j] = (i >= j) ? F[(j0 + i) + (int64_t)(j0 + j) * m] : 0.0;
  }
  for (int q = threadIdx.x; q < w * nr; q += blockDim.x) {
    const int i = q % w, r = q / w;
    double v = wv[j0 + i + (int64_t)r * m];
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

__global__ void k_bwd_store(const double* __restrict__ W, double* __restrict__ x, SolveArgs a,
                            const int* __restrict__ fronts, const int64_t* __restrict__ prefix, int count) {
  const int idx = find_task(prefix, count, blockIdx.x);
  const int s = fronts[idx];
  const int k = a.k[s], m = a.m[s];
  const int i = (int)(blockIdx.x - prefix[idx]) * kSolveRows + threadIdx.x;
  if (i >= k) return;
  const double* w = W + a.w_off[s] * a.nrhs;
  const int pos = a.rows[a.rows_off[s] + i];
  for (int r = 0; r < a.nrhs; ++r) x[pos + r * a.ld] = w[i + (int64_t)r * m];
}

#define TDEM_CUDA_TRY(x)                                                          \
  do {                                                                             \
    cudaError_t e_ = (x);                                                          \
    if (e_ != cudaSuccess) return std::string(#x ": ") + cudaGetErrorString(e_);   \
  } while (0)

inline unsigned grid_of(int64_t ctas) { return (unsigned)ctas; }
constexpr size_t kTrsmSmem = sizeof(double) * (P + kTrsmRows) * (P + 1);
constexpr size_t kSyrkSmem = sizeof(double) * 2 * kTileSyrk * (P + 1);

}  // namespace

GpuCholesky::~GpuCholesky() {
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

std::string GpuCholesky::setup(Symbolic&& sy, const std::vector<int>& perm_to_vec, int nrhs_max,
                               cudaStream_t s) {
  sy_ = std::move(sy);
  nrhs_max_ = std::max(1, nrhs_max);
  if ((int)perm_to_vec.size() != sy_.n) return "perm_to_vec size mismatch";
  if (nrhs_max_ * P * (int)sizeof(double) > 96 * 1024) return "too many right-hand sides";
  std::string e;
  if (!(e = alloc((void**)&d_L_, sizeof(double) * std::max<int64_t>(1, sy_.nnz_l))).empty()) return e;
  if (!(e = alloc((void**)&d_U_, sizeof(double) * std::max<int64_t>(1, sy_.u_elems))).empty()) return e;
  if (!(e = alloc((void**)&d_W_, sizeof(double) * std::max<int64_t>(1, sy_.wvec_elems) * nrhs_max_)).empty())
    return e;
  if (!(e = alloc((void**)&d_part_, sizeof(double) * std::max<int64_t>(1, sy_.solve_partials) * nrhs_max_)).empty())
    return e;
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
  if (!(e = alloc((void**)&d_err_, sizeof(int))).empty()) return e;
  TDEM_CUDA_TRY(cudaMemsetAsync(d_err_, 0, sizeof(int), s));
  TDEM_CUDA_TRY(cudaFuncSetAttribute(k_trsm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrsmSmem));
  TDEM_CUDA_TRY(cudaFuncSetAttribute(k_syrk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSyrkSmem));
  TDEM_CUDA_TRY(cudaFuncSetAttribute(k_fwd_diag, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024));
  TDEM_CUDA_TRY(cudaFuncSetAttribute(k_bwd_diag, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024));
  TDEM_CUDA_TRY(cudaFuncSetAttribute(k_fwd_update, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024));
  TDEM_CUDA_TRY(cudaStreamSynchronize(s));
  return "";
}

void GpuCholesky::factor(const double* d_vals, cudaStream_t s) {
  int launches = 0;
  Fronts fr{d_l_off_, d_u_off_, d_m_, d_k_};
  cudaMemsetAsync(d_L_, 0, sizeof(double) * sy_.nnz_l, s);
  {
    const int64_t nnz = sy_.nnz_lower;
    const unsigned g = (unsigned)std::min<int64_t>((nnz + 255) / 256, 148 * 32);
    if (nnz > 0) {
      k_scatter_entries<<<g, 256, 0, s>>>(d_L_, d_entry_, d_vals, nnz);
      ++launches;
    }
  }
  const int* T = d_tasks_;
  const int64_t* Pf = d_prefix_;
  for (const LevelPlan& lp : sy_.levels) {
    if (lp.assemble.ctas > 0) {
      k_zero_u<<<grid_of(lp.assemble.ctas), 256, 0, s>>>(d_U_, fr, T + lp.assemble.off, Pf + lp.assemble.pre,
                                                        lp.assemble.count);
      ++launches;
    }
    for (const TaskList& tl : lp.extend_slots) {
      if (tl.ctas == 0) continue;
      k_extend_add<<<grid_of(tl.ctas), 256, 0, s>>>(d_L_, d_U_, fr, d_parent_, d_rel_off_, d_rel_, T + tl.off,
                                                    Pf + tl.pre, tl.count);
      ++launches;
    }
    for (const PanelStep& ps : lp.panels) {
      k_potrf<<<ps.potrf.count, 256, 0, s>>>(d_L_, fr, T + ps.potrf.off, ps.j0, d_err_, d_c0_);
      ++launches;
      if (ps.trsm.ctas > 0) {
        k_trsm<<<grid_of(ps.trsm.ctas), kTrsmRows, kTrsmSmem, s>>>(d_L_, fr, T + ps.trsm.off, Pf + ps.trsm.pre,
                                                           ps.trsm.count, ps.j0);
        ++launches;
      }
      if (ps.syrk.ctas > 0) {
        k_syrk<<<grid_of(ps.syrk.ctas), 256, kSyrkSmem, s>>>(d_L_, d_U_, fr, T + ps.syrk.off, Pf + ps.syrk.pre,
                                                     ps.syrk.count, ps.j0);
        ++launches;
      }
    }
  }
  launches_factor_ = launches;
}

void GpuCholesky::solve(const double* d_b, double* d_x, int64_t ld, int nrhs, cudaStream_t s) {
  int launches = 0;
  SolveArgs a{d_l_off_, d_w_off_, d_m_, d_k_, d_rows_off_, d_rows_, nrhs, ld};
  const int* T = d_tasks_;
  const int64_t* Pf = d_prefix_;
  const size_t ysm = sizeof(double) * P * nrhs;
  for (const LevelPlan& lp : sy_.levels) {
    k_fwd_init<<<grid_of(lp.assemble.ctas), kSolveRows, 0, s>>>(d_W_, d_b, a, T + lp.assemble.off,
                                                                Pf + lp.assemble.pre, lp.assemble.count);
    ++launches;
    for (const TaskList& tl : lp.extend_vec) {
      if (tl.ctas == 0) continue;
      k_fwd_extend<<<grid_of(tl.ctas), kSolveRows, 0, s>>>(d_W_, a, d_parent_, d_rel_off_, d_rel_, T + tl.off,
                                                           Pf + tl.pre, tl.count);
      ++launches;
    }
    for (const PanelStep& ps : lp.panels) {
      k_fwd_diag<<<ps.potrf.count, 256, ysm, s>>>(d_L_, d_W_, a, T + ps.potrf.off, ps.j0);
      ++launches;
      if (ps.solve_upd.ctas > 0) {
        k_fwd_update<<<grid_of(ps.solve_upd.ctas), kSolveRows, ysm, s>>>(
            d_L_, d_W_, a, T + ps.solve_upd.off, Pf + ps.solve_upd.pre, ps.solve_upd.count, ps.j0);
        ++launches;
      }
    }
  }
  for (int l = (int)sy_.levels.size() - 1; l >= 0; --l) {
    const LevelPlan& lp = sy_.levels[l];
    k_bwd_init<<<grid_of(lp.assemble.ctas), kSolveRows, 0, s>>>(d_W_, d_x, a, T + lp.assemble.off,
                                                                Pf + lp.assemble.pre, lp.assemble.count);
    ++launches;
    for (int p = (int)lp.panels.size() - 1; p >= 0; --p) {
      const PanelStep& ps = lp.panels[p];
      if (ps.solve_upd.ctas > 0) {
        k_bwd_partial<<<grid_of(ps.solve_upd.ctas), kSolveRows, 0, s>>>(
            d_L_, d_W_, a, d_part_, T + ps.solve_upd.off, Pf + ps.solve_upd.pre, ps.solve_upd.count, ps.j0);
        ++launches;
      }
      k_bwd_diag<<<ps.potrf.count, 256, ysm, s>>>(d_L_, d_W_, a, d_part_, T + ps.solve_upd.off,
                                                   Pf + ps.solve_upd.pre, ps.j0);
      ++launches;
    }
    k_bwd_store<<<grid_of(lp.assemble.ctas), kSolveRows, 0, s>>>(d_W_, d_x, a, T + lp.assemble.off,
                                                                 Pf + lp.assemble.pre, lp.assemble.count);
    ++launches;
  }
  launches_solve_ = launches;
}

int GpuCholesky::status(cudaStream_t s) {
  int h = 0;
  cudaMemcpyAsync(&h, d_err_, sizeof(int), cudaMemcpyDeviceToHost, s);
  cudaStreamSynchronize(s);
  return h;
}

}  // namespace tdem
