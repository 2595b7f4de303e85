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
// triangular solve of the rows below, rank-64 update of the rest of the kOuter-wide
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
  // the lower triangle only: the updates, the extend-add and the trailing update
  // read and write rows i >= c of column c and nothing above
  for (int c = c0; c < c1; ++c)
    for (int i = c + threadIdx.x; i < r; i += blockDim.x) u[i + (int64_t)c * r] = (T)0;
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

// Cholesky of the w x w diagonal block of panel [j0, j0 + w) (one CTA of 256
// threads per front), right-looking in shared memory with one barrier per column.
// Thread t owns row i = t % 64 and, of it, the columns c = t / 64 (mod 4).  Step j
// scales column j on the fly (L(r, j) = A(r, j) / sqrt(A(j, j)), recomputed by
// every thread that needs it) and subtracts L(i, j) L(c, j) from A(i, c) for
// j < c <= i; the finished column goes to the upper triangle A[j][r] (r > j) and
// the diagonal to diag[j], which no later step reads, so column j is read
// unchanged throughout its step.  Same operations in the same order per element
// as a column-at-a-time factorization: the result does not depend on the thread
// layout.
// With dinv (FP64 factorization) the CTA also inverts the finished block into the
// front's inverted diagonal blocks (dinv_off[s] + 64 * 64 * (j0 / 64), column-major,
// leading dimension w): the operand of the panel solve k_trsm_dmma and of the
// triangular solves (by 16 x 16 blocks, see below).
template <class T>
__global__ void __launch_bounds__(256) k_potrf(T* __restrict__ L, Fronts f, const int* __restrict__ fronts, int j0,
                                               int* __restrict__ err, const int* __restrict__ c0_of,
                                               T* __restrict__ dinv = nullptr,
                                               const int64_t* __restrict__ dinv_off = nullptr) {
  __shared__ T A[P][P + 1];
  __shared__ T diag[P];
  __shared__ T xd[P];
  __shared__ T tb[3][16][16];  // band products of the blocked inverse
  const int s = fronts[blockIdx.x];
  const int m = f.m[s], k = f.k[s];
  const int w = min(P, k - j0);
  T* F = L + f.l_off[s];
  for (int idx = threadIdx.x; idx < w * w; idx += blockDim.x) {
    const int i = idx % w, j = idx / w;
    A[i][j] = (i >= j) ? F[(j0 + i) + (int64_t)(j0 + j) * m] : (T)0;
  }
  __syncthreads();
  const int i = threadIdx.x & (P - 1), g = threadIdx.x >> 6;
  for (int j = 0; j < w; ++j) {
    T d = A[j][j];
    if (!(d > (T)0)) {
      if (threadIdx.x == 0) atomicCAS(err, 0, c0_of[s] + j0 + j + 1);
      d = (T)1;
    }
    const T sd = tsqrt(d);
    const T inv = (T)1 / sd;
    if (i > j && i < w) {
      const T lij = A[i][j] * inv;
      // first column of this thread's group after j
      int c = j + 1 + ((g - (j + 1)) & 3);
      for (; c <= i; c += 4) A[i][c] -= lij * (A[c][j] * inv);
      if (g == 0) A[j][i] = lij;
    }
    if (threadIdx.x == 0) diag[j] = sd;
    __syncthreads();
  }
  for (int idx = threadIdx.x; idx < w * w; idx += blockDim.x) {
    const int r = idx % w, c = idx / w;
    if (r >= c) F[(j0 + r) + (int64_t)(j0 + c) * m] = (r == c) ? diag[c] : A[c][r];
  }
  if (dinv == nullptr) return;
  // L(r, c) = A[c][r] (r > c) or diag[r]; the inverse X(r, c) (r > c) goes to the
  // lower triangle, whose working values are dead, and its diagonal to xd.  By
  // 16 x 16 blocks: the diagonal blocks by substitution, four threads per column
  // running X(r, c) = -(sum_{c <= l < r} L(r, l) X(l, c)) / L(r, r) over at most 15
  // rows; then the blocks below them band by band, X_ij = -X_ii sum_{j <= k < i}
  // L_ik X_kj, every element of a band at once (a column-long substitution would
  // chain 63 dependent steps).
  constexpr int QB = 16;
  auto Xv = [&](int l, int c) -> T { return l == c ? xd[c] : (l > c ? A[l][c] : (T)0); };
  {
    const int c = threadIdx.x >> 2, part = threadIdx.x & 3;
    const unsigned mask = 0xFu << ((threadIdx.x & 31) & ~3);
    if (c < w) {
      const int bend = min(w, (c / QB + 1) * QB);
      if (part == 0) xd[c] = (T)1 / diag[c];
      __syncwarp(mask);
      for (int r = c + 1; r < bend; ++r) {
        T sum = (T)0;
        for (int l = c + part; l < r; l += 4) sum = fma(A[l][r], l == c ? xd[c] : A[l][c], sum);
        sum += __shfl_xor_sync(mask, sum, 1);
        sum += __shfl_xor_sync(mask, sum, 2);
        if (part == 0) A[r][c] = -sum / diag[r];
        __syncwarp(mask);
      }
    }
  }
  __syncthreads();
  const int nb = (w + QB - 1) / QB;
  for (int d = 1; d < nb; ++d) {
    const int np = nb - d;  // block pairs (j + d, j) of band d
    for (int e = threadIdx.x; e < np * QB * QB; e += blockDim.x) {
      const int j = e / (QB * QB), rr = (e / QB) % QB, cc = e % QB;
      const int r = (j + d) * QB + rr, c = j * QB + cc;
      T t = (T)0;
      if (r < w && c < w)
        for (int l = j * QB; l < (j + d) * QB; ++l) t = fma(A[l][r], Xv(l, c), t);
      tb[j][rr][cc] = t;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < np * QB * QB; e += blockDim.x) {
      const int j = e / (QB * QB), rr = (e / QB) % QB, cc = e % QB;
      const int i0 = (j + d) * QB, r = i0 + rr, c = j * QB + cc;
      if (r < w && c < w) {
        T x = (T)0;
        for (int l = i0; l <= r; ++l) x = fma(Xv(r, l), tb[j][l - i0][cc], x);
        A[r][c] = -x;
      }
    }
    __syncthreads();
  }
  T* D = dinv + dinv_off[s] + (int64_t)(j0 / P) * P * P;
  for (int q = threadIdx.x; q < w * w; q += blockDim.x) {
    const int r = q % w, c = q / w;
    D[q] = (r > c) ? A[r][c] : (r == c ? xd[c] : (T)0);
  }
}

// Panel triangular solve: rows [j1, m) of the panel columns times L_dd^-T.
// kTrsmRows rows per CTA, one row per thread held in registers (the substitution
// is unrolled over the 64 columns, so every element has a fixed register); the
// diagonal block is read from shared memory, the same address for the whole warp.
template <class T>
__global__ void __launch_bounds__(kTrsmRows) k_trsm(T* __restrict__ L, Fronts f, const int* __restrict__ fronts,
                                                    const int64_t* __restrict__ prefix, int count, int j0) {
  __shared__ T Ld[P][P];  // Ld[c][cc] = L_dd(c, cc), cc <= c
  const int idx = find_task(prefix, count, blockIdx.x);
  const int s = fronts[idx];
  const int m = f.m[s], k = f.k[s];
  const int w = min(P, k - j0), j1 = j0 + w;
  T* F = L + f.l_off[s];
  for (int q = threadIdx.x; q < w * w; q += blockDim.x) {
    const int i = q % w, j = q / w;
    Ld[i][j] = (i >= j) ? F[(j0 + i) + (int64_t)(j0 + j) * m] : (T)0;
  }
  const int row = j1 + (int)(blockIdx.x - prefix[idx]) * kTrsmRows + threadIdx.x;
  const bool live = row < m;
  T x[P];
#pragma unroll
  for (int c = 0; c < P; ++c) x[c] = (live && c < w) ? F[row + (int64_t)(j0 + c) * m] : (T)0;
  __syncthreads();
#pragma unroll
  for (int c = 0; c < P; ++c) {
    if (c < w) {
      T v = x[c];
#pragma unroll
      for (int cc = 0; cc < c; ++cc) v -= x[cc] * Ld[c][cc];
      x[c] = v / Ld[c][c];
    }
  }
  if (live) {
#pragma unroll
    for (int c = 0; c < P; ++c)
      if (c < w) F[row + (int64_t)(j0 + c) * m] = x[c];
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
// outer panel rows [J1, m), columns [J0, J1).  The task list counts 128 x 128
// lower-triangle tiles; each is done by two CTAs of 128 threads (column halves of
// 64), two CTAs per SM, so one CTA's operand loads and read-modify-write of its
// tile overlap the other's FMAs.  A CTA streams K in chunks of KC through two
// shared-memory buffers filled by cp.async (the next chunk lands while the
// current one is consumed); each thread keeps an 8 x 8 block of the tile in
// registers (rows tx + 16 a, columns ty + 8 b).
constexpr int KC = 32;
constexpr int kBigThreads = 128;
constexpr int kBigCols = 64;  // columns per CTA (half a 128 x 128 tile)

// cp.async of one element (4 or 8 bytes); src_bytes = 0 stores a zero instead.
template <int BYTES>
__device__ __forceinline__ void cp_async_elem(void* dst, const void* src, int src_bytes) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;" ::"r"(d), "l"(src), "n"(BYTES), "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

template <class T>
__global__ void __launch_bounds__(kBigThreads, 2) k_syrk_big(T* __restrict__ L, T* __restrict__ U, Fronts f,
                                                              const int* __restrict__ fronts,
                                                              const int64_t* __restrict__ prefix, int count, int j0) {
  constexpr int TB = kTileBig, TC = kBigCols;
  extern __shared__ __align__(16) unsigned char sm_raw[];
  // buffer s: As[s][p][i] (KC x TB), then Bs[s][p][j] (KC x TC)
  T* sbuf = reinterpret_cast<T*>(sm_raw);
  const int idx = find_task(prefix, count, blockIdx.x >> 1);
  const int s = fronts[idx];
  const int m = f.m[s], k = f.k[s];
  const int J0 = (j0 / kOuter) * kOuter, J1 = min(k, J0 + kOuter);
  const int64_t lo = f.l_off[s], uo = f.u_off[s];
  const T* F = L + lo;
  const int64_t t = (blockIdx.x >> 1) - prefix[idx];
  int bi = (int)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
  while ((int64_t)(bi + 1) * (bi + 2) / 2 <= t) ++bi;
  while ((int64_t)bi * (bi + 1) / 2 > t) --bi;
  const int bj = (int)(t - (int64_t)bi * (bi + 1) / 2);
  const int r0 = J1 + bi * TB, c0 = J1 + bj * TB + (blockIdx.x & 1) * TC;
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  // the upper half of a diagonal tile's right column half is above the diagonal
  if (c0 >= m || (bi == bj && (blockIdx.x & 1) && r0 + TB <= c0)) return;
  const int K = J1 - J0, nch = (K + KC - 1) / KC;
  // thread tid copies rows tid of A (all KC columns) and rows tid % 64 of B
  // (columns tid / 64 + 2 j): coalesced 256-byte rows per warp
  const bool arow = r0 + tid < m;
  const int bi_row = tid & (TC - 1), bp0 = tid >> 6;
  const bool brow = c0 + bi_row < m;
  auto load_chunk = [&](int ch, int buf) {
    T* As = sbuf + (size_t)buf * KC * (TB + TC);
    T* Bs = As + KC * TB;
    const int k0 = ch * KC, kc = min(KC, K - k0);
#pragma unroll 8
    for (int p = 0; p < KC; ++p) {
      const bool ok = arow && p < kc;
      const T* src = ok ? F + (r0 + tid) + (int64_t)(J0 + k0 + p) * m : F;
      cp_async_elem<(int)sizeof(T)>(As + p * TB + tid, src, ok ? (int)sizeof(T) : 0);
    }
#pragma unroll 8
    for (int j = 0; j < KC / 2; ++j) {
      const int p = bp0 + 2 * j;
      const bool ok = brow && p < kc;
      const T* src = ok ? F + (c0 + bi_row) + (int64_t)(J0 + k0 + p) * m : F;
      cp_async_elem<(int)sizeof(T)>(Bs + p * TC + bi_row, src, ok ? (int)sizeof(T) : 0);
    }
  };
  T acc[8][8];
#pragma unroll
  for (int a = 0; a < 8; ++a)
#pragma unroll
    for (int b = 0; b < 8; ++b) acc[a][b] = (T)0;
  load_chunk(0, 0);
  cp_async_commit();
  for (int ch = 0; ch < nch; ++ch) {
    if (ch + 1 < nch) load_chunk(ch + 1, (ch + 1) & 1);
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    const T* As = sbuf + (size_t)(ch & 1) * KC * (TB + TC);
    const T* Bs = As + KC * TB;
    const int kc = min(KC, K - ch * KC);
#pragma unroll 4
    for (int p = 0; p < kc; ++p) {
      T av[8], bv[8];
#pragma unroll
      for (int a = 0; a < 8; ++a) av[a] = As[p * TB + tx + 16 * a];
#pragma unroll
      for (int b = 0; b < 8; ++b) bv[b] = Bs[p * TC + ty + 8 * b];
#pragma unroll
      for (int a = 0; a < 8; ++a)
#pragma unroll
        for (int b = 0; b < 8; ++b) acc[a][b] = fma(av[a], bv[b], acc[a][b]);
    }
    // the buffer is refilled by the next iteration's copies
    __syncthreads();
  }
  cp_async_wait_all();
  // per output row: the 8 loads first, then the 8 stores (the element pointers may
  // alias as far as the compiler knows, which would serialise load-store pairs)
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    const int r = r0 + tx + 16 * a;
    if (r >= m) continue;
    T old[8];
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      const int c = c0 + ty + 8 * b;
      old[b] = (c < m && c <= r) ? *felem(L, U, lo, uo, m, k, r, c) : (T)0;
    }
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      const int c = c0 + ty + 8 * b;
      if (c < m && c <= r) *felem(L, U, lo, uo, m, k, r, c) = old[b] - acc[a][b];
    }
  }
}

// FP64 trailing update on the FP64 tensor pipe (mma.sync m16n8k16 .f64): same
// task list and tile split as k_syrk_big (two 128-thread CTAs per 128 x 128 tile,
// two CTAs per SM), K streamed through kDStages cp.async stage buffers of KD
// columns (three in flight), and each warp owns a 64 x 32 block of its CTA's
// 128 x 64 tile as 4 x 4 MMA tiles, so one instruction does 2,048 multiply-adds
// instead of 32 and the issue slots stay free for the loads.
// Shared layouts are k-major with the row (column) stride padded to 4 mod 16
// doubles.  A 64-bit shared access is served per half-warp; a fragment load's
// half-warp reads 4 rows x 4 k, which this stride spreads over all 32 banks.
// The epilogue tile's column stride is 2 mod 8 for the same reason (its
// fragment elements step two columns per q).
constexpr int kLdA = kTileBig + 4;   // 132
constexpr int kLdB = kBigCols + 4;   // 68
constexpr int kLdC = kTileBig + 2;   // 130, epilogue tile columns (fits in the operand buffers)
constexpr int KD = 16;               // K per stage of the tensor-pipe update (one k16 step)
constexpr int kDStages = 4;          // stage buffers (three chunks in flight)
static_assert(kBigCols * kLdC <= kDStages * KD * (kLdA + kLdB), "epilogue tile must fit the operand buffers");

__device__ __forceinline__ void dmma16816(double (&c)[4], const double (&a)[8], const double (&b)[4]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7,%8,%9,%10,%11}, "
      "{%12,%13,%14,%15}, {%0,%1,%2,%3};"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]), "d"(b[0]),
        "d"(b[1]), "d"(b[2]), "d"(b[3]));
}

// Panel triangular solve on the FP64 tensor pipe: rows [j1, m) of the panel columns
// times L_dd^-T, with L_dd^-1 the inverse k_potrf wrote (dinv_off[s] + 64 * 64 *
// (j0 / 64), column-major, leading dimension w).  kTrsmRows = 128 rows per CTA
// (the task list of k_trsm), 256 threads: warp v owns rows 16 v .. 16 v + 15 and
// all 64 columns (8 MMA tiles of m16n8k16), K = the 64 panel columns.  The rows are
// staged k-major (stride 4 mod 16 doubles: conflict-free fragment loads), the
// product is staged back the same way and written column by column, coalesced.
// A substitution would chain 64 dependent steps per row; the product has none.
constexpr int kLdT = kTrsmRows + 4;  // 132
constexpr int kLdI = P + 4;          // 68
constexpr size_t trsm_dmma_smem() { return sizeof(double) * P * (kLdT + kLdI); }

__global__ void __launch_bounds__(256) k_trsm_dmma(double* __restrict__ L, Fronts f, const int* __restrict__ fronts,
                                                   const int64_t* __restrict__ prefix, int count, int j0,
                                                   const double* __restrict__ dinv,
                                                   const int64_t* __restrict__ dinv_off) {
  extern __shared__ __align__(16) unsigned char sm_raw[];
  double(*As)[kLdT] = reinterpret_cast<double(*)[kLdT]>(sm_raw);                          // As[l][row]
  double(*Bs)[kLdI] = reinterpret_cast<double(*)[kLdI]>(sm_raw + sizeof(double) * P * kLdT);  // Bs[l][c]
  const int idx = find_task(prefix, count, blockIdx.x);
  const int s = fronts[idx];
  const int m = f.m[s], k = f.k[s];
  const int w = min(P, k - j0), j1 = j0 + w;
  double* F = L + f.l_off[s];
  const int row0 = j1 + (int)(blockIdx.x - prefix[idx]) * kTrsmRows;
  const int t = threadIdx.x;
  // rows: thread t reads row t % 128 of columns t / 128 + 2 e
  {
    const int r = t & (kTrsmRows - 1), l0 = t >> 7;
    const bool live = row0 + r < m;
#pragma unroll 8
    for (int l = l0; l < P; l += 2) As[l][r] = (live && l < w) ? F[(row0 + r) + (int64_t)(j0 + l) * m] : 0.0;
  }
  // B(l, c) = L_dd^-1(c, l) = D[c + l w] (zero above the diagonal and outside w)
  {
    const double* D = dinv + dinv_off[s] + (int64_t)(j0 / P) * P * P;
    for (int q = t; q < P * P; q += 256) {
      const int c = q & (P - 1), l = q >> 6;
      Bs[l][c] = (c < w && l < w) ? D[c + l * w] : 0.0;
    }
  }
  __syncthreads();
  const int lane = t & 31, warp = t >> 5, g = lane >> 2, q = lane & 3;
  double acc[8][4];
#pragma unroll
  for (int j = 0; j < 8; ++j)
#pragma unroll
    for (int e = 0; e < 4; ++e) acc[j][e] = 0.0;
#pragma unroll
  for (int k16 = 0; k16 < P; k16 += 16) {
    double af[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) af[i] = As[k16 + q + 4 * (i >> 1)][16 * warp + g + 8 * (i & 1)];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      double bf[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) bf[i] = Bs[k16 + q + 4 * i][8 * nt + g];
      dmma16816(acc[nt], af, bf);
    }
  }
  __syncthreads();
#pragma unroll
  for (int nt = 0; nt < 8; ++nt)
#pragma unroll
    for (int i = 0; i < 4; ++i) As[8 * nt + 2 * q + (i & 1)][16 * warp + g + 8 * (i >> 1)] = acc[nt][i];
  __syncthreads();
  {
    const int r = t & (kTrsmRows - 1), l0 = t >> 7;
    if (row0 + r < m) {
#pragma unroll 8
      for (int l = l0; l < w; l += 2) F[(row0 + r) + (int64_t)(j0 + l) * m] = As[l][r];
    }
  }
}

// One 128 x 64 tile of F -= X X^T on the FP64 tensor pipe: rows [r0, r0 + 128)
// below m, columns [c0, c0 + 64) below cend, lower triangle only; X is column
// block [kb, kb + K) of the front (rows of X = rows and columns of the tile).
// Called by all 128 threads of a CTA with kBigThreads threads and dmma_smem()
// bytes of dynamic shared memory.
__device__ __forceinline__ void dmma_tile(double* __restrict__ L, double* __restrict__ U, int64_t lo, int64_t uo,
                                          int m, int k, int r0, int c0, int cend, int kb, int K, double* sbuf) {
  constexpr int TC = kBigCols;
  const double* F = L + lo;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, q = lane & 3;
  const int wr = (warp >> 1) * 64, wc = (warp & 1) * 32;  // warp block within the CTA tile
  const int nch = (K + KD - 1) / KD;
  const bool arow = r0 + tid < m;
  const int bi_row = tid & (TC - 1), bp0 = tid >> 6;
  const bool brow = c0 + bi_row < cend;
  constexpr int kBuf = KD * (kLdA + kLdB);
  // chunk ch of K (KD columns) into stage buffer buf; commits one cp.async group
  // (empty past the last chunk, which keeps the group count per iteration fixed)
  auto load_chunk = [&](int ch, int buf) {
    if (ch < nch) {
      double* As = sbuf + buf * kBuf;
      double* Bs = As + KD * kLdA;
      const int k0 = ch * KD, kc = min(KD, K - k0);
#pragma unroll
      for (int p = 0; p < KD; ++p) {
        const bool ok = arow && p < kc;
        const double* src = ok ? F + (r0 + tid) + (int64_t)(kb + k0 + p) * m : F;
        cp_async_elem<8>(As + p * kLdA + tid, src, ok ? 8 : 0);
      }
#pragma unroll
      for (int j = 0; j < KD / 2; ++j) {
        const int p = bp0 + 2 * j;
        const bool ok = brow && p < kc;
        const double* src = ok ? F + (c0 + bi_row) + (int64_t)(kb + k0 + p) * m : F;
        cp_async_elem<8>(Bs + p * kLdB + bi_row, src, ok ? 8 : 0);
      }
    }
    cp_async_commit();
  };
  double acc[4][4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b)
#pragma unroll
      for (int i = 0; i < 4; ++i) acc[a][b][i] = 0.0;
  // kDStages - 1 chunks in flight ahead of the one being multiplied; one barrier
  // per chunk: after it every thread has finished the previous chunk, whose
  // buffer is then refilled
#pragma unroll
  for (int st = 0; st < kDStages - 1; ++st) load_chunk(st, st);
  for (int ch = 0; ch < nch; ++ch) {
    cp_async_wait<kDStages - 2>();
    __syncthreads();
    load_chunk(ch + kDStages - 1, (ch + kDStages - 1) % kDStages);
    const double* As = sbuf + (ch % kDStages) * kBuf;
    const double* Bs = As + KD * kLdA;
    // zero-filled past K, so every chunk is one full k16 step
    double bf[4][4];
#pragma unroll
    for (int n = 0; n < 4; ++n)
#pragma unroll
      for (int i = 0; i < 4; ++i) bf[n][i] = Bs[(q + 4 * i) * kLdB + wc + 8 * n + g];
#pragma unroll
    for (int mt = 0; mt < 4; ++mt) {
      double af[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) af[i] = As[(q + 4 * (i >> 1)) * kLdA + wr + 16 * mt + g + 8 * (i & 1)];
#pragma unroll
      for (int n = 0; n < 4; ++n) dmma16816(acc[mt][n], af, bf[n]);
    }
  }
  cp_async_wait_all();
  __syncthreads();
  // Epilogue through shared memory (the operand buffers are free now): the tile's
  // old values arrive in one round of cp.async (row tid of every column), the
  // accumulators are subtracted in place, and each column goes back as one
  // coalesced store per warp.  Cs[c][r] holds column c, row r of the CTA tile.
  double* Cs = sbuf;
  const int tile_cols = min(TC, cend - c0);
#pragma unroll 8
  for (int c = 0; c < TC; ++c) {
    const int rr = r0 + tid, cc = c0 + c;
    const bool ok = c < tile_cols && rr < m && cc <= rr;
    const double* src = ok ? felem(L, U, lo, uo, m, k, rr, cc) : F;
    cp_async_elem<8>(Cs + c * kLdC + tid, src, ok ? 8 : 0);
  }
  cp_async_commit();
  cp_async_wait_all();
  __syncthreads();
  // element (mt, n, i): row wr + 16 mt + g + 8 (i / 2), column wc + 8 n + 2 q + (i & 1)
#pragma unroll
  for (int mt = 0; mt < 4; ++mt)
#pragma unroll
    for (int n = 0; n < 4; ++n)
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int rl = wr + 16 * mt + g + 8 * (i >> 1), cl = wc + 8 * n + 2 * q + (i & 1);
        Cs[cl * kLdC + rl] -= acc[mt][n][i];
      }
  __syncthreads();
  for (int c = 0; c < tile_cols; ++c) {
    const int rr = r0 + tid, cc = c0 + c;
    if (rr < m && cc <= rr) *felem(L, U, lo, uo, m, k, rr, cc) = Cs[c * kLdC + tid];
  }
}

// Trailing update of an outer panel on the FP64 tensor pipe (two CTAs per task-list
// tile of 128 x 128, one per 64-column half).
__global__ void __launch_bounds__(kBigThreads, 2) k_syrk_big_dmma(double* __restrict__ L, double* __restrict__ U,
                                                                   Fronts f, const int* __restrict__ fronts,
                                                                   const int64_t* __restrict__ prefix, int count,
                                                                   int j0) {
  extern __shared__ __align__(16) unsigned char sm_raw[];
  const int idx = find_task(prefix, count, blockIdx.x >> 1);
  const int s = fronts[idx];
  const int m = f.m[s], k = f.k[s];
  const int J0 = (j0 / kOuter) * kOuter, J1 = min(k, J0 + kOuter);
  const int64_t t = (blockIdx.x >> 1) - prefix[idx];
  int bi = (int)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
  while ((int64_t)(bi + 1) * (bi + 2) / 2 <= t) ++bi;
  while ((int64_t)bi * (bi + 1) / 2 > t) --bi;
  const int bj = (int)(t - (int64_t)bi * (bi + 1) / 2);
  const int r0 = J1 + bi * kTileBig, c0 = J1 + bj * kTileBig + (blockIdx.x & 1) * kBigCols;
  if (c0 >= m) return;
  dmma_tile(L, U, f.l_off[s], f.u_off[s], m, k, r0, c0, m, J0, J1 - J0,
            reinterpret_cast<double*>(sm_raw));
}

// Update of the rest of the outer panel by the inner panel [j0, j1) on the FP64
// tensor pipe: F[r, c] -= sum_p X[r, p] X[c, p] for c in [j1, J1), r >= c, in 128 x
// 64 tiles.  Column tile bj pairs with row tiles bi >= bj / 2 (the ones reaching
// the diagonal), so a front has sum over bj of (nr - bj / 2) tiles.
__global__ void __launch_bounds__(kBigThreads, 2) k_panel_dmma(double* __restrict__ L, double* __restrict__ U,
                                                                Fronts f, const int* __restrict__ fronts,
                                                                const int64_t* __restrict__ prefix, int count,
                                                                int j0, int bj0 = 0) {
  extern __shared__ __align__(16) unsigned char sm_raw[];
  const int idx = find_task(prefix, count, blockIdx.x);
  const int s = fronts[idx];
  const int m = f.m[s], k = f.k[s];
  const int w = min(kPanel, k - j0), j1 = j0 + w;
  const int J0 = (j0 / kOuter) * kOuter, J1 = min(k, J0 + kOuter);
  const int nr = (m - j1 + kTileBig - 1) / kTileBig;
  // tiles from column tile bj0 on (the task list's counts say how many)
  int t = (int)(blockIdx.x - prefix[idx]), bj = bj0;
  while (t >= nr - bj / 2) {
    t -= nr - bj / 2;
    ++bj;
  }
  const int bi = bj / 2 + t;
  dmma_tile(L, U, f.l_off[s], f.u_off[s], m, k, j1 + bi * kTileBig, j1 + bj * kBigCols, J1, j0, w,
            reinterpret_cast<double*>(sm_raw));
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
  const int* units;        // units of this launch (kUnitInts ints each, Symbolic::solve_units)
  int64_t count;           // units in this launch
  int* ticket;             // launch-order counter (zeroed before the solve)
  int* flags;              // one per pivot block (zeroed before the solve)
  int* counters;           // finished chunk units per row (zeroed before the solve)
  int* err;                // set to 1 when a wait gave up (the solver's err[1])
};

// A level-solve unit as unpacked from its 64-byte record.
struct Unit {
  int R, lo, hi, slot, cnt, nparts, fin, m, k, flag0;
  int64_t l_off, w_off, dinv_off;
};

__device__ __forceinline__ int64_t join64(int lo, int hi) {
  return (int64_t)(((uint64_t)(uint32_t)hi << 32) | (uint64_t)(uint32_t)lo);
}

// Every thread reads the same 64 bytes (one broadcast request per 16 bytes).
__device__ __forceinline__ Unit load_unit(const int* __restrict__ units, int64_t idx) {
  const int4* p = reinterpret_cast<const int4*>(units + (int64_t)kUnitInts * idx);
  const int4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2), d = __ldg(p + 3);
  Unit u;
  u.R = a.x; u.lo = a.y; u.hi = a.z; u.slot = a.w;
  u.cnt = b.x; u.nparts = b.y; u.fin = b.z; u.m = b.w;
  u.k = c.x; u.flag0 = c.y;
  u.l_off = join64(c.z, c.w);
  u.w_off = join64(d.x, d.y);
  u.dinv_off = join64(d.z, d.w);
  return u;
}

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
// (i + 64 c) mod 256, slot (i + 64 c) / 256, i.e. thread t holds row t % 64 of
// columns t / 64 + 4 e.
template <class T>
__device__ __forceinline__ void load_block(T (&pre)[16], const T* __restrict__ F, int64_t ld, int r0, int nr, int c0,
                                           int nc) {
#pragma unroll
  for (int e = 0; e < 16; ++e) {
    const int q = threadIdx.x + 256 * e;
    const int i = q & 63, c = q >> 6;
    pre[e] = (i < nr && c < nc) ? __ldg(F + (r0 + i) + (int64_t)(c0 + c) * ld) : (T)0;
  }
}
// registers -> Ls[c][i]
constexpr int kLdL = SB + 4;  // 68: fragment loads along either index hit all 32 banks
template <class T>
__device__ __forceinline__ void store_block(T (*Ls)[kLdL], const T (&pre)[16]) {
#pragma unroll
  for (int e = 0; e < 16; ++e) {
    const int q = threadIdx.x + 256 * e;
    Ls[q >> 6][q & 63] = pre[e];
  }
}

// Leading dimension of the staged solution values of a block (64 x nrhs): the
// right-hand sides rounded up to MMA tiles of 8, plus 4 (4 mod 16 doubles keeps a
// half-warp's fragment load on distinct banks).
__host__ __device__ constexpr int ys_ld(int nrhs) { return 8 * ((nrhs + 7) / 8) + 4; }

// acc[r][c-tile] += M (64 x 64) * V (64 x nrhs) on the FP64 tensor pipe for one
// 64 x 64 block, M read from Ls: element (row, k) at Ls[k][row] (TRANS = false) or
// Ls[row][k] (TRANS = true); V element (k, r) at Vs[k * ld + r].  Warp w owns row
// tile w % 4 and column tiles w / 4 + 2 j; NTW = column tiles per warp.
template <bool TRANS, int NTW>
__device__ __forceinline__ void block_dmma(double (&acc)[NTW][4], const double (*Ls)[kLdL], const double* Vs, int ld,
                                           int ntiles) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, q = lane & 3;
  const int mt = warp & 3;
#pragma unroll
  for (int k16 = 0; k16 < SB; k16 += 16) {
    double af[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int row = 16 * mt + g + 8 * (i & 1), kk = k16 + q + 4 * (i >> 1);
      af[i] = TRANS ? Ls[row][kk] : Ls[kk][row];
    }
#pragma unroll
    for (int j = 0; j < NTW; ++j) {
      const int nt = (warp >> 2) + 2 * j;
      if (nt < ntiles) {
        double bf[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) bf[i] = Vs[(k16 + q + 4 * i) * ld + 8 * nt + g];
        dmma16816(acc[j], af, bf);
      }
    }
  }
}

// MMA accumulators -> Out[row * ld + r] (64 x 8 ntiles)
template <int NTW>
__device__ __forceinline__ void store_acc(const double (&acc)[NTW][4], double* Out, int ld, int ntiles) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, q = lane & 3;
  const int mt = warp & 3;
#pragma unroll
  for (int j = 0; j < NTW; ++j) {
    const int nt = (warp >> 2) + 2 * j;
    if (nt < ntiles) {
#pragma unroll
      for (int i = 0; i < 4; ++i) Out[(16 * mt + g + 8 * (i >> 1)) * ld + 8 * nt + 2 * q + (i & 1)] = acc[j][i];
    }
  }
}

// Forward unit (many right-hand sides): row block R of front s (R < pb: pivot rows
// [64R, ..); else update rows [k + 64 (R - pb), ..)), accumulating L_Rq y_q for
// the pivot blocks q in [lo, hi).  Chunk units publish partial sums; the final
// unit (q = the last one the row needs) adds them, then a pivot row solves
// y_R = Dinv_R (w_R - sum) and raises its flag, an update row stores w_R - sum
// for the parent.  One unit per CTA.  In FP64 the block products run on the
// tensor pipe (the right-hand sides make them compute-bound).
// Thread t: row i = t % 64 of the block, right-hand sides r = t / 64 + 4 j.
template <class T, int RPT>
__global__ void __launch_bounds__(256, 2) k_fwd_level(const T* __restrict__ L, const T* __restrict__ Dinv, T* W, T* part,
                                                   int nr_rhs, FusedArgs fa) {
  __shared__ T Ls[SB][kLdL];
  __shared__ int s_item;
  extern __shared__ __align__(16) unsigned char sm_raw[];
  T* Ys = reinterpret_cast<T*>(sm_raw);  // SB x ysl, [c * ysl + r]
  const int ysl = ys_ld(nr_rhs), ntl = (nr_rhs + 7) / 8;
  constexpr bool kMma = std::is_same<T, double>::value;
  constexpr int NTW = (RPT + 3) / 4;  // column tiles per warp (nrhs <= 4 RPT)
  const int t = threadIdx.x, i = t & 63, g = t >> 6;
  if (t == 0) s_item = atomicAdd(fa.ticket, 1);
  __syncthreads();
  const Unit u = load_unit(fa.units, s_item);
  const int R = u.R, lo = u.lo, hi = u.hi, m = u.m, k = u.k, fin = u.fin;
  const int pb = (k + SB - 1) / SB;
  const bool piv = R < pb;
  const int r0 = piv ? SB * R : k + SB * (R - pb);
  const int nr = min(SB, (piv ? k : m) - r0);
  const T* F = L + u.l_off;
  T* w = W + u.w_off * nr_rhs;
  const int* flags = fa.flags + u.flag0;
  T acc[RPT];
#pragma unroll
  for (int j = 0; j < RPT; ++j) acc[j] = (T)0;
  double macc[NTW][4];
#pragma unroll
  for (int j = 0; j < NTW; ++j)
#pragma unroll
    for (int e = 0; e < 4; ++e) macc[j][e] = 0.0;
  // final pivot unit: its inverted diagonal block and its own rows of W do not
  // depend on this launch, so they are read before any wait
  // (with many right-hand sides the registers go to the accumulators instead and
  // the inverse is read after the last block)
  constexpr bool kPreD = RPT <= 2;
  const T* D = Dinv + u.dinv_off + (int64_t)R * SB * SB;
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
      wrow[j] = (r < nr_rhs && i < nr) ? __ldcg(w + r0 + i + (int64_t)r * m) : (T)0;
    }
  }
  T* my_part = part + (int64_t)u.slot * SB * nr_rhs;
  T tot[RPT];
#pragma unroll
  for (int j = 0; j < RPT; ++j) tot[j] = (T)0;
  // the chunk partials of this row are ready long before the last block's flag
  if (fin) gather_partials<T, RPT>(my_part, u.nparts, nr_rhs, fa.counters + u.cnt, fa.err, tot);
  T pre[16];
  if (lo < hi) load_block(pre, F, m, r0, nr, SB * lo, min(SB, k - SB * lo));
  for (int q = lo; q < hi; ++q) {
    const int wq = min(SB, k - SB * q);
    if (t == 0) wait_flag(flags + q, fa.err);
    __syncthreads();
    store_block(Ls, pre);
    // the block's solution values, one right-hand side (64 contiguous values of
    // W) per pair of warps: coalesced reads; columns up to the last MMA tile
    for (int e = t; e < SB * 8 * ntl; e += 256) {
      const int c = e & (SB - 1), r = e / SB;
      Ys[c * ysl + r] = (c < wq && r < nr_rhs) ? __ldcg(w + SB * q + c + (int64_t)r * m) : (T)0;
    }
    __syncthreads();
    if (q + 1 < hi) load_block(pre, F, m, r0, nr, SB * (q + 1), min(SB, k - SB * (q + 1)));
    if constexpr (kMma) {
      block_dmma<false, NTW>(macc, Ls, Ys, ysl, ntl);
    } else {
#pragma unroll 8
      for (int c = 0; c < SB; ++c) {
        const T l = Ls[c][i];
#pragma unroll
        for (int j = 0; j < RPT; ++j) {
          const int r = g + 4 * j;
          if (r < nr_rhs) acc[j] = fma(l, Ys[c * ysl + r], acc[j]);
        }
      }
    }
  }
  if constexpr (kMma) {
    // the tensor-pipe sums go to the thread layout through the (now free) block tile
    T* Acc = &Ls[0][0];
    __syncthreads();
    store_acc<NTW>(macc, Acc, kLdL, ntl);
    __syncthreads();
#pragma unroll
    for (int j = 0; j < RPT; ++j) {
      const int r = g + 4 * j;
      if (r < nr_rhs) acc[j] = Acc[i * kLdL + r];
    }
  }
  if (!fin) {
    publish_partial<T, RPT>(my_part, acc, nr_rhs, fa.counters + u.cnt);
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
    if (r < nr_rhs) Ys[i * ysl + r] = (i < nr) ? wrow[j] - acc[j] : (T)0;
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
      if (r < nr_rhs) y[j] = fma(l, Ys[c * ysl + r], y[j]);
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
  if (t == 0) publish_flag(fa.flags + u.flag0 + R);
}

// Backward unit (many right-hand sides): column block p of front s, accumulating
// L_Rp^T x_R over the row blocks R in [lo, hi) (R < pb: pivot rows, waited for;
// else update rows, whose x come from ancestors and were staged in W by
// k_bwd_init).  The final unit (row block p + 1) adds the chunk partials and
// solves x_p = Dinv_p^T (y_p - sum), written to W and to the caller's vector,
// then raises the column's flag.  One unit per CTA; FP64 block products on the
// tensor pipe.
// Thread t: column c = t % 64 of the block, right-hand sides r = t / 64 + 4 j.
template <class T, int RPT>
__global__ void __launch_bounds__(256, 2) k_bwd_level(const T* __restrict__ L, const T* __restrict__ Dinv, T* W, T* part,
                                                   double* __restrict__ x, const int* __restrict__ rows, int64_t ldx,
                                                   int nr_rhs, FusedArgs fa) {
  __shared__ T Ls[SB][kLdL];
  __shared__ int s_item;
  extern __shared__ __align__(16) unsigned char sm_raw[];
  T* Ws = reinterpret_cast<T*>(sm_raw);  // SB x ysl, [row * ysl + r]
  const int ysl = ys_ld(nr_rhs), ntl = (nr_rhs + 7) / 8;
  constexpr bool kMma = std::is_same<T, double>::value;
  constexpr int NTW = (RPT + 3) / 4;
  const int t = threadIdx.x, c = t & 63, g = t >> 6;
  if (t == 0) s_item = atomicAdd(fa.ticket, 1);
  __syncthreads();
  const Unit u = load_unit(fa.units, s_item);
  const int p = u.R, lo = u.lo, hi = u.hi, m = u.m, k = u.k, fin = u.fin;
  const int pb = (k + SB - 1) / SB;
  const int c0 = SB * p, wc = min(SB, k - c0);
  const T* F = L + u.l_off;
  T* w = W + u.w_off * nr_rhs;
  const int* flags = fa.flags + u.flag0;
  T acc[RPT];
#pragma unroll
  for (int j = 0; j < RPT; ++j) acc[j] = (T)0;
  double macc[NTW][4];
#pragma unroll
  for (int j = 0; j < NTW; ++j)
#pragma unroll
    for (int e = 0; e < 4; ++e) macc[j][e] = 0.0;
  constexpr bool kPreD = RPT <= 2;
  const T* D = Dinv + u.dinv_off + (int64_t)p * SB * SB;
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
      wrow[j] = (r < nr_rhs && c < wc) ? __ldcg(w + c0 + c + (int64_t)r * m) : (T)0;
    }
  }
  T* my_part = part + (int64_t)u.slot * SB * nr_rhs;
  T tot[RPT];
#pragma unroll
  for (int j = 0; j < RPT; ++j) tot[j] = (T)0;
  if (fin) gather_partials<T, RPT>(my_part, u.nparts, nr_rhs, fa.counters + u.cnt, fa.err, tot);
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
    // coalesced as in k_fwd_level
    for (int e = t; e < SB * 8 * ntl; e += 256) {
      const int ii = e & (SB - 1), r = e / SB;
      Ws[ii * ysl + r] = (ii < nr && r < nr_rhs) ? __ldcg(w + r0 + ii + (int64_t)r * m) : (T)0;
    }
    __syncthreads();
    if (R - 1 >= lo) {
      int r1, n1;
      rows_of(R - 1, r1, n1);
      load_block(pre, F, m, r1, n1, c0, wc);
    }
    if constexpr (kMma) {
      block_dmma<true, NTW>(macc, Ls, Ws, ysl, ntl);
    } else {
#pragma unroll 8
      for (int ii = 0; ii < SB; ++ii) {
        const T l = Ls[c][ii];
#pragma unroll
        for (int j = 0; j < RPT; ++j) {
          const int r = g + 4 * j;
          if (r < nr_rhs) acc[j] = fma(l, Ws[ii * ysl + r], acc[j]);
        }
      }
    }
  }
  if constexpr (kMma) {
    T* Acc = &Ls[0][0];
    __syncthreads();
    store_acc<NTW>(macc, Acc, kLdL, ntl);
    __syncthreads();
#pragma unroll
    for (int j = 0; j < RPT; ++j) {
      const int r = g + 4 * j;
      if (r < nr_rhs) acc[j] = Acc[c * kLdL + r];
    }
  }
  if (!fin) {
    publish_partial<T, RPT>(my_part, acc, nr_rhs, fa.counters + u.cnt);
    return;
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < RPT; ++j) {
    const int r = g + 4 * j;
    if (r < nr_rhs) Ws[c * ysl + r] = (c < wc) ? wrow[j] - (tot[j] + acc[j]) : (T)0;
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
      if (r < nr_rhs) xv[j] = fma(l, Ws[ii * ysl + r], xv[j]);
    }
  }
  if (c < wc) {
    const int pos = rows[u.w_off + c0 + c];
#pragma unroll
    for (int j = 0; j < RPT; ++j) {
      const int r = g + 4 * j;
      if (r < nr_rhs) {
        w[c0 + c + (int64_t)r * m] = xv[j];
        x[pos + (int64_t)r * ldx] = (double)xv[j];
      }
    }
  }
  __syncthreads();
  if (t == 0) publish_flag(fa.flags + u.flag0 + p);
}

// ---------------------------------------------------------------------------
// Streaming level solves for one or two right-hand sides.
//
// Persistent CTAs (as many as fit on the device) take units by ticket until the
// level's list is exhausted; the next ticket is taken when a unit starts, so its
// latency hides behind the unit's work.  Each thread copies its own elements of
// the unit's blocks into shared memory with cp.async, kStages blocks ahead of
// their use (and the inverted diagonal block of a final unit at the start), so
// a CTA keeps several 32 KB loads in flight without holding them in registers;
// since a thread only reads back what it copied, no CTA barrier is needed
// between copy and use.  Each warp waits for the pivot blocks it needs itself
// (lane 0 polls, then a warp barrier).  The four column groups (forward) or 64
// rows (backward) of a block are combined once per unit, in a fixed order, so
// results are deterministic.
// ---------------------------------------------------------------------------
constexpr int kStages = 2;

// This thread's 16 elements (row t % 64, columns t / 64 + 4 e) of the 64 x 64
// block at rows [r0, r0 + nr), columns [c0, c0 + nc) of F (zero outside) into
// buf[e * 256 + t].  Does not commit.
template <class T>
__device__ __forceinline__ void cp_block(T* buf, const T* __restrict__ F, int64_t ld, int r0, int nr, int c0, int nc) {
  const int t = threadIdx.x, i = t & 63, g = t >> 6;
#pragma unroll
  for (int e = 0; e < 16; ++e) {
    const int c = g + 4 * e;
    const bool ok = i < nr && c < nc;
    const T* src = ok ? F + (r0 + i) + (int64_t)(c0 + c) * ld : F;
    cp_async_elem<(int)sizeof(T)>(buf + e * 256 + t, src, ok ? (int)sizeof(T) : 0);
  }
}

// Sum over the 32 lanes of a warp of v[e] for each e < 16 (recursive halving):
// afterwards lane l holds the total of e = (l >> 1) & 15.  The additions happen
// in an order fixed by the lane pattern alone.
template <class T>
__device__ __forceinline__ T warp_sum16(const T (&v)[16], int lane) {
  T a8[8], a4[4], a2[2];
  bool up = (lane & 16) != 0;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const T mine = up ? v[8 + j] : v[j], other = up ? v[j] : v[8 + j];
    a8[j] = mine + __shfl_xor_sync(0xffffffffu, other, 16);
  }
  up = (lane & 8) != 0;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const T mine = up ? a8[4 + j] : a8[j], other = up ? a8[j] : a8[4 + j];
    a4[j] = mine + __shfl_xor_sync(0xffffffffu, other, 8);
  }
  up = (lane & 4) != 0;
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    const T mine = up ? a4[2 + j] : a4[j], other = up ? a4[j] : a4[2 + j];
    a2[j] = mine + __shfl_xor_sync(0xffffffffu, other, 4);
  }
  up = (lane & 2) != 0;
  const T mine = up ? a2[1] : a2[0], other = up ? a2[0] : a2[1];
  const T a1 = mine + __shfl_xor_sync(0xffffffffu, other, 2);
  return a1 + __shfl_xor_sync(0xffffffffu, a1, 1);
}

// Lane 0 of the calling warp waits for *flag; the warp barrier then orders the
// other lanes' later loads after the acquire.
__device__ __forceinline__ void warp_wait_flag(const int* flag, int* err, int lane) {
  if (lane == 0) wait_flag(flag, err);
  __syncwarp();
}
__device__ __forceinline__ void warp_wait_count(const int* c, int target, int* err, int lane) {
  if (lane == 0) wait_count(c, target, err);
  __syncwarp();
}

// One thread waits for *flag like wait_flag, but the polls back off to
// sleep_max ns: units queued early (bulk work waiting for the dependency chain)
// then keep the L2 slice that holds the flags free for the chain itself.
__device__ void wait_flag_backoff(const int* flag, int* err, unsigned sleep_max) {
  if (*(volatile int*)err != 0) return;
  unsigned ns = 32;
  for (unsigned it = 0; it < kSpinLimit; ++it) {
    if (ld_acquire(flag) != 0) return;
    __nanosleep(ns);
    ns = min(2 * ns, sleep_max);
  }
  atomicExch(err, 1);
}


// Dynamic shared memory of the streaming kernels: kStages block buffers and the
// inverted diagonal block, 64 x 64 entries each.
template <class T>
constexpr size_t stream_smem() { return sizeof(T) * (kStages + 1) * SB * SB; }

// Forward unit, streaming form (see k_fwd_level for the unit's meaning).
// Thread t holds row i = t % 64 of columns g + 4 e (g = t / 64, e < 16) of each
// block and accumulates its share of the row sums for every right-hand side.
template <class T, int NR>
__global__ void __launch_bounds__(256, 2) k_fwd_stream(const T* __restrict__ L, const T* __restrict__ Dinv, T* W,
                                                    T* part, int nr_rhs, FusedArgs fa) {
  extern __shared__ __align__(16) unsigned char sm_raw[];
  T* stage = reinterpret_cast<T*>(sm_raw);     // kStages x 4096
  T* dsm = stage + kStages * SB * SB;          // inverted diagonal block, 4096
  __shared__ T red[4][SB][NR];  // per column group: partial row sums
  __shared__ T zs[SB][NR];      // pivot rows: w - sum, the input of the inverse
  __shared__ T ys[kUnitBlocks][SB][NR];  // y of every block of the unit (when staged)
  __shared__ int s_tk[2], s_ready;
  const int t = threadIdx.x, i = t & 63, g = t >> 6, lane = t & 31;
  if (t == 0) s_tk[0] = atomicAdd(fa.ticket, 1);
  __syncthreads();
  for (int par = 0;; par ^= 1) {
    const int tk = s_tk[par];
    if (tk >= fa.count) break;
    int next = 0;
    if (t == 0) next = atomicAdd(fa.ticket, 1);
    const Unit u = load_unit(fa.units, tk);
    const int R = u.R, lo = u.lo, hi = u.hi, m = u.m, k = u.k;
    const bool fin = u.fin != 0;
    const int pb = (k + SB - 1) / SB;
    const bool piv = R < pb;
    const int r0 = piv ? SB * R : k + SB * (R - pb);
    const int nr = min(SB, (piv ? k : m) - r0);
    const T* F = L + u.l_off;
    T* w = W + u.w_off * nr_rhs;
    const int* flags = fa.flags + u.flag0;
    // final pivot unit: the inverted diagonal block (independent of this launch)
    if (fin && piv) cp_block(dsm, Dinv + u.dinv_off + (int64_t)R * SB * SB, nr, 0, nr, 0, nr);
#pragma unroll
    for (int j = 0; j < kStages; ++j) {
      const int q = lo + j;
      if (q < hi) cp_block(stage + j * SB * SB, F, m, r0, nr, SB * q, min(SB, k - SB * q));
      cp_async_commit();
    }
    T wrow[NR];
    if (fin && g == 0) {
#pragma unroll
      for (int r = 0; r < NR; ++r) wrow[r] = (r < nr_rhs && i < nr) ? __ldcg(w + r0 + i + (int64_t)r * m) : (T)0;
    }
    T acc[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) acc[r] = (T)0;
    // chunk partials of this row (warps of column group 0): gathered before the
    // wait for the newest block, which is the last input of a chain unit
    T tot[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) tot[r] = (T)0;
    T* my_part = part + (int64_t)u.slot * SB * nr_rhs;
    auto gather = [&]() {
      if (fin && g == 0 && u.nparts > 0) {
        warp_wait_count(fa.counters + u.cnt, u.nparts, fa.err, lane);
        for (int c = 0; c < u.nparts; ++c)
#pragma unroll
          for (int r = 0; r < NR; ++r)
            if (r < nr_rhs) tot[r] += __ldcg(my_part + (int64_t)c * SB * nr_rhs + i + SB * r);
      }
    };
    // The flags of a front are set in chain order (the unit that sets flag q has
    // waited for flag q - 1), so the newest flag of the range stands for all of
    // them.  A unit other than a chain unit (final unit of a pivot row) waits for
    // it on one thread and stages the y of all its blocks with one barrier; a
    // chain unit checks it once and, unless it is set, takes its blocks as their
    // flags appear.
    const bool chain = fin && piv;
    if (t == 0) {
      int ready = 1;
      if (lo < hi) {
        if (!chain) wait_flag_backoff(flags + hi - 1, fa.err, 1024);
        else ready = ld_acquire(flags + hi - 1) != 0;
      }
      s_ready = ready;
    }
    __syncthreads();
    const bool staged = s_ready != 0;
    if (staged && lo < hi) {
      for (int e = t; e < (hi - lo) * SB * NR; e += 256) {
        const int b = e / (SB * NR), c = (e / NR) % SB, r = e % NR;
        const int q = lo + b;
        ys[b][c][r] = (r < nr_rhs && c < min(SB, k - SB * q)) ? __ldcg(w + SB * q + c + (int64_t)r * m) : (T)0;
      }
      __syncthreads();
    }
    if (lo == hi) gather();
    for (int q = lo; q < hi; ++q) {
      const int slot = (q - lo) % kStages;
      if (q == hi - 1) gather();
      const T* blk = stage + slot * SB * SB + t;
      if (!staged) {
        warp_wait_flag(flags + q, fa.err, lane);
        const int wq = min(SB, k - SB * q), c = g + 4 * (lane & 15);
        T yv[NR];
#pragma unroll
        for (int r = 0; r < NR; ++r) yv[r] = (r < nr_rhs && c < wq) ? __ldcg(w + SB * q + c + (int64_t)r * m) : (T)0;
        cp_async_wait<kStages - 1>();
#pragma unroll
        for (int e = 0; e < 16; ++e) {
          const T l = blk[e * 256];
#pragma unroll
          for (int r = 0; r < NR; ++r) acc[r] = fma(l, __shfl_sync(0xffffffffu, yv[r], e), acc[r]);
        }
      } else {
        cp_async_wait<kStages - 1>();
        const T(*yb)[NR] = ys[q - lo];
#pragma unroll
        for (int e = 0; e < 16; ++e) {
          const T l = blk[e * 256];
#pragma unroll
          for (int r = 0; r < NR; ++r) acc[r] = fma(l, yb[g + 4 * e][r], acc[r]);
        }
      }
      // the slot's values are in registers and used: refill it
      const int qn = q + kStages;
      if (qn < hi) cp_block(stage + slot * SB * SB, F, m, r0, nr, SB * qn, min(SB, k - SB * qn));
      cp_async_commit();
    }
    // row totals: chunk partials (in order), then the four column groups
    if (g != 0) {
#pragma unroll
      for (int r = 0; r < NR; ++r) red[g][i][r] = acc[r];
    }
    __syncthreads();
    if (g == 0) {
#pragma unroll
      for (int r = 0; r < NR; ++r) acc[r] = ((acc[r] + red[1][i][r]) + red[2][i][r]) + red[3][i][r];
      if (!fin) {
#pragma unroll
        for (int r = 0; r < NR; ++r)
          if (r < nr_rhs) my_part[i + SB * r] = acc[r];
      } else if (!piv) {
        if (i < nr) {
#pragma unroll
          for (int r = 0; r < NR; ++r)
            if (r < nr_rhs) w[r0 + i + (int64_t)r * m] -= tot[r] + acc[r];
        }
      } else {
#pragma unroll
        for (int r = 0; r < NR; ++r) zs[i][r] = (i < nr) ? wrow[r] - (tot[r] + acc[r]) : (T)0;
      }
    }
    if (fin && piv) {
      // y_R = Dinv_R z: thread (i, g) sums its 16 columns, then the groups are added
      cp_async_wait_all();
      __syncthreads();
      T y[NR];
#pragma unroll
      for (int r = 0; r < NR; ++r) y[r] = (T)0;
#pragma unroll
      for (int e = 0; e < 16; ++e) {
        const T d = dsm[e * 256 + t];
#pragma unroll
        for (int r = 0; r < NR; ++r) y[r] = fma(d, zs[g + 4 * e][r], y[r]);
      }
      if (g != 0) {
#pragma unroll
        for (int r = 0; r < NR; ++r) red[g][i][r] = y[r];
      }
      __syncthreads();
      if (g == 0 && i < nr) {
#pragma unroll
        for (int r = 0; r < NR; ++r)
          if (r < nr_rhs) w[r0 + i + (int64_t)r * m] = ((y[r] + red[1][i][r]) + red[2][i][r]) + red[3][i][r];
      }
    }
    const bool publish = !fin || piv;
    if (t == 0) s_tk[par ^ 1] = next;
    __syncthreads();
    if (t == 0 && publish) {
      if (fin) publish_flag(fa.flags + u.flag0 + R);
      else publish_add(fa.counters + u.cnt);
    }
  }
  cp_async_wait_all();
}

// Backward unit, streaming form (see k_bwd_level for the unit's meaning).
// Thread t holds row i = t % 64 of columns g + 4 e of each block and accumulates
// L(i, c) x(i) per column; the 64 rows of a column are added once per unit.
template <class T, int NR>
__global__ void __launch_bounds__(256, 2) k_bwd_stream(const T* __restrict__ L, const T* __restrict__ Dinv, T* W,
                                                    T* part, double* __restrict__ x, const int* __restrict__ rows,
                                                    int64_t ldx, int nr_rhs, FusedArgs fa) {
  extern __shared__ __align__(16) unsigned char sm_raw[];
  T* stage = reinterpret_cast<T*>(sm_raw);
  T* dsm = stage + kStages * SB * SB;
  __shared__ T red[2][SB][NR];  // per row half: column sums
  __shared__ T zs[SB][NR];      // y_p - sum, the input of the inverse
  __shared__ T xs[kUnitBlocks][SB][NR];  // x of the row blocks of the unit (when staged)
  __shared__ int s_tk[2], s_ready;
  const int t = threadIdx.x, i = t & 63, g = t >> 6, lane = t & 31, half = (t >> 5) & 1;
  // column of the warp-reduced value this lane holds
  const int cl = g + 4 * ((lane >> 1) & 15);
  if (t == 0) s_tk[0] = atomicAdd(fa.ticket, 1);
  __syncthreads();
  for (int par = 0;; par ^= 1) {
    const int tk = s_tk[par];
    if (tk >= fa.count) break;
    int next = 0;
    if (t == 0) next = atomicAdd(fa.ticket, 1);
    const Unit u = load_unit(fa.units, tk);
    const int p = u.R, lo = u.lo, hi = u.hi, m = u.m, k = u.k;
    const bool fin = u.fin != 0;
    const int pb = (k + SB - 1) / SB;
    const int c0 = SB * p, wc = min(SB, k - c0);
    const T* F = L + u.l_off;
    T* w = W + u.w_off * nr_rhs;
    const int* flags = fa.flags + u.flag0;
    auto rows_of = [&](int R, int& r0, int& nr) {
      r0 = (R < pb) ? SB * R : k + SB * (R - pb);
      nr = min(SB, (R < pb ? k : m) - r0);
    };
    if (fin) cp_block(dsm, Dinv + u.dinv_off + (int64_t)p * SB * SB, wc, 0, wc, 0, wc);
    // rows farthest from the diagonal first (their x are known earliest)
#pragma unroll
    for (int j = 0; j < kStages; ++j) {
      const int R = hi - 1 - j;
      if (R >= lo) {
        int r0, nr;
        rows_of(R, r0, nr);
        cp_block(stage + j * SB * SB, F, m, r0, nr, c0, wc);
      }
      cp_async_commit();
    }
    T wrow[NR];
    if (fin && t < SB) {
#pragma unroll
      for (int r = 0; r < NR; ++r) wrow[r] = (r < nr_rhs && t < wc) ? __ldcg(w + c0 + t + (int64_t)r * m) : (T)0;
    }
    T acc[NR][16];
#pragma unroll
    for (int r = 0; r < NR; ++r)
#pragma unroll
      for (int e = 0; e < 16; ++e) acc[r][e] = (T)0;
    // chunk partials of this column (warps 0 and 1), gathered before the wait for
    // the newest row block
    T tot[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) tot[r] = (T)0;
    T* my_part = part + (int64_t)u.slot * SB * nr_rhs;
    auto gather = [&]() {
      if (fin && t < SB && u.nparts > 0) {
        warp_wait_count(fa.counters + u.cnt, u.nparts, fa.err, lane);
        for (int c = 0; c < u.nparts; ++c)
#pragma unroll
          for (int r = 0; r < NR; ++r)
            if (r < nr_rhs) tot[r] += __ldcg(my_part + (int64_t)c * SB * nr_rhs + t + SB * r);
      }
    };
    // Flags are set in chain order (last column first), so flag lo stands for
    // every pivot row block of the range.  A chunk waits for it on one thread and
    // stages x of all its row blocks with one barrier; the final unit (a link of
    // the chain) checks it once and, unless it is set, stages only the update
    // rows (no flag) and takes the pivot row blocks as their flags appear.
    if (t == 0) {
      int ready = 1;
      if (lo < hi && lo < pb) {
        if (!fin) wait_flag_backoff(flags + lo, fa.err, 1024);
        else ready = ld_acquire(flags + lo) != 0;
      }
      s_ready = ready;
    }
    __syncthreads();
    const bool staged = s_ready != 0;
    const int sfirst = staged ? lo : max(lo, pb);  // first staged row block
    if (sfirst < hi) {
      for (int e = t; e < (hi - sfirst) * SB * NR; e += 256) {
        const int b = e / (SB * NR), ii = (e / NR) % SB, r = e % NR;
        int r0, nr;
        rows_of(sfirst + b, r0, nr);
        xs[sfirst - lo + b][ii][r] = (r < nr_rhs && ii < nr) ? __ldcg(w + r0 + ii + (int64_t)r * m) : (T)0;
      }
      __syncthreads();
    }
    if (lo == hi) gather();
    for (int R = hi - 1; R >= lo; --R) {
      const int slot = (hi - 1 - R) % kStages;
      int r0, nr;
      rows_of(R, r0, nr);
      if (R == lo) gather();
      T xv[NR];
      if (R < sfirst) {
        warp_wait_flag(flags + R, fa.err, lane);
#pragma unroll
        for (int r = 0; r < NR; ++r) xv[r] = (r < nr_rhs && i < nr) ? __ldcg(w + r0 + i + (int64_t)r * m) : (T)0;
      } else {
#pragma unroll
        for (int r = 0; r < NR; ++r) xv[r] = xs[R - lo][i][r];
      }
      cp_async_wait<kStages - 1>();
      const T* blk = stage + slot * SB * SB + t;
#pragma unroll
      for (int e = 0; e < 16; ++e) {
        const T l = blk[e * 256];
#pragma unroll
        for (int r = 0; r < NR; ++r) acc[r][e] = fma(l, xv[r], acc[r][e]);
      }
      const int Rn = R - kStages;
      if (Rn >= lo) {
        int rn0, nrn;
        rows_of(Rn, rn0, nrn);
        cp_block(stage + slot * SB * SB, F, m, rn0, nrn, c0, wc);
      }
      cp_async_commit();
    }
    // column totals: rows within the warp, then the two row halves
#pragma unroll
    for (int r = 0; r < NR; ++r) {
      const T v = warp_sum16(acc[r], lane);
      if ((lane & 1) == 0) red[half][cl][r] = v;
    }
    __syncthreads();
    if (t < SB) {
      T s[NR];
#pragma unroll
      for (int r = 0; r < NR; ++r) s[r] = red[0][t][r] + red[1][t][r];
      if (!fin) {
#pragma unroll
        for (int r = 0; r < NR; ++r)
          if (r < nr_rhs) my_part[t + SB * r] = s[r];
      } else {
#pragma unroll
        for (int r = 0; r < NR; ++r) zs[t][r] = (t < wc) ? wrow[r] - (tot[r] + s[r]) : (T)0;
      }
    }
    if (fin) {
      // x_p = Dinv_p^T z: thread (i, g) forms D(i, c) z(i) for its 16 columns, then
      // the rows are added as above
      cp_async_wait_all();
      __syncthreads();
#pragma unroll
      for (int r = 0; r < NR; ++r) {
        const T zi = zs[i][r];
#pragma unroll
        for (int e = 0; e < 16; ++e) acc[r][e] = dsm[e * 256 + t] * zi;
      }
#pragma unroll
      for (int r = 0; r < NR; ++r) {
        const T v = warp_sum16(acc[r], lane);
        if ((lane & 1) == 0) red[half][cl][r] = v;
      }
      __syncthreads();
      if (t < wc) {
        const int pos = rows[u.w_off + c0 + t];
#pragma unroll
        for (int r = 0; r < NR; ++r)
          if (r < nr_rhs) {
            const T xs = red[0][t][r] + red[1][t][r];
            w[c0 + t + (int64_t)r * m] = xs;
            x[pos + (int64_t)r * ldx] = (double)xs;
          }
      }
    }
    if (t == 0) s_tk[par ^ 1] = next;
    __syncthreads();
    if (t == 0) {
      if (fin) publish_flag(fa.flags + u.flag0 + p);
      else publish_add(fa.counters + u.cnt);
    }
  }
  cp_async_wait_all();
}

// ---------------------------------------------------------------------------
// Persistent level solves for many right-hand sides (FP64, 3..32 columns).
//
// The units and their meaning are those of k_fwd_level / k_bwd_level; the CTAs
// are persistent (as many as fit, two per SM) and take units by ticket like the
// streaming kernels.  A unit's 64 x 64 factor blocks and 64 x nrhs solution
// blocks are copied into two shared-memory stages with cp.async, the next block
// while the current one is multiplied on the FP64 tensor pipe (block_dmma).  A
// unit whose inputs are all solved (every unit except a chain link caught before
// its newest block is ready) waits once and prefetches solution blocks as well;
// a chain link waits per block and reads that block's solution values directly.
// Diagonal inverses of final pivot units are held in registers from the start.
// Results are bitwise those of k_fwd_level / k_bwd_level (same products in the
// same order).
// ---------------------------------------------------------------------------
constexpr int kMrStages = 2;
constexpr int kMrYld = ys_ld(32);  // solution-block stage leading dimension (32 columns)
constexpr size_t mr_smem() { return sizeof(double) * kMrStages * (SB * kLdL + SB * kMrYld); }

// This thread's 16 elements (row t % 64, columns t / 64 + 4 e) of the 64 x 64 block
// at rows [r0, r0 + nr), columns [c0, c0 + nc) of F into Ls[c][i] (zero outside).
// Does not commit.
__device__ __forceinline__ void cp_block_ls(double (*Ls)[kLdL], const double* __restrict__ F, int64_t ld, int r0,
                                            int nr, int c0, int nc) {
  const int t = threadIdx.x, i = t & 63, g = t >> 6;
#pragma unroll
  for (int e = 0; e < 16; ++e) {
    const int c = g + 4 * e;
    const bool ok = i < nr && c < nc;
    cp_async_elem<8>(&Ls[c][i], ok ? F + (r0 + i) + (int64_t)(c0 + c) * ld : F, ok ? 8 : 0);
  }
}

// rows [r0, r0 + nr) of the front vectors w (ld m), columns < nr_rhs, into
// Vs[row * ysl + r] for columns up to 8 ntl (zero outside).  Does not commit.
__device__ __forceinline__ void cp_vec_block(double* Vs, int ysl, const double* w, int64_t m, int r0, int nr,
                                             int nr_rhs, int ntl) {
  for (int e = threadIdx.x; e < SB * 8 * ntl; e += 256) {
    const int c = e & (SB - 1), r = e / SB;
    const bool ok = c < nr && r < nr_rhs;
    cp_async_elem<8>(Vs + c * ysl + r, ok ? w + r0 + c + (int64_t)r * m : w, ok ? 8 : 0);
  }
}
__device__ __forceinline__ void ld_vec_block(double* Vs, int ysl, const double* w, int64_t m, int r0, int nr,
                                             int nr_rhs, int ntl) {
  for (int e = threadIdx.x; e < SB * 8 * ntl; e += 256) {
    const int c = e & (SB - 1), r = e / SB;
    Vs[c * ysl + r] = (c < nr && r < nr_rhs) ? __ldcg(w + r0 + c + (int64_t)r * m) : 0.0;
  }
}

template <int RPT>
__global__ void __launch_bounds__(256, 2) k_fwd_mrhs(const double* __restrict__ L, const double* __restrict__ Dinv,
                                                  double* W, double* part, int nr_rhs, FusedArgs fa) {
  extern __shared__ __align__(16) unsigned char sm_raw[];
  double(*Lst)[SB][kLdL] = reinterpret_cast<double(*)[SB][kLdL]>(sm_raw);
  double* Yst = reinterpret_cast<double*>(sm_raw + sizeof(double) * kMrStages * SB * kLdL);
  __shared__ int s_tk[2], s_ready;
  constexpr int NTW = (RPT + 3) / 4;
  const int ysl = ys_ld(nr_rhs), ntl = (nr_rhs + 7) / 8;
  const int t = threadIdx.x, i = t & 63, g = t >> 6;
  if (t == 0) s_tk[0] = atomicAdd(fa.ticket, 1);
  __syncthreads();
  for (int par = 0;; par ^= 1) {
    const int tk = s_tk[par];
    if (tk >= fa.count) break;
    int next = 0;
    if (t == 0) next = atomicAdd(fa.ticket, 1);
    const Unit u = load_unit(fa.units, tk);
    const int R = u.R, lo = u.lo, hi = u.hi, m = u.m, k = u.k;
    const bool fin = u.fin != 0;
    const int pb = (k + SB - 1) / SB;
    const bool piv = R < pb;
    const int r0 = piv ? SB * R : k + SB * (R - pb);
    const int nr = min(SB, (piv ? k : m) - r0);
    const double* F = L + u.l_off;
    double* w = W + u.w_off * nr_rhs;
    const int* flags = fa.flags + u.flag0;
#pragma unroll
    for (int j = 0; j < kMrStages; ++j) {
      const int q = lo + j;
      if (q < hi) cp_block_ls(Lst[j], F, m, r0, nr, SB * q, min(SB, k - SB * q));
      cp_async_commit();
    }
    // final pivot unit: its inverted diagonal block and its own rows of W do not
    // depend on this launch
    double dpre[16], wrow[RPT];
    if (fin && piv) {
      const double* D = Dinv + u.dinv_off + (int64_t)R * SB * SB;
#pragma unroll
      for (int e = 0; e < 16; ++e) {
        const int q = t + 256 * e, ii = q & 63, c = q >> 6;
        dpre[e] = (ii < nr && c < nr) ? __ldg(D + ii + c * nr) : 0.0;
      }
#pragma unroll
      for (int j = 0; j < RPT; ++j) {
        const int r = g + 4 * j;
        wrow[j] = (r < nr_rhs && i < nr) ? __ldcg(w + r0 + i + (int64_t)r * m) : 0.0;
      }
    }
    double* my_part = part + (int64_t)u.slot * SB * nr_rhs;
    double tot[RPT];
#pragma unroll
    for (int j = 0; j < RPT; ++j) tot[j] = 0.0;
    if (fin) gather_partials<double, RPT>(my_part, u.nparts, nr_rhs, fa.counters + u.cnt, fa.err, tot);
    // flags of a front are set in chain order: the newest flag of the range stands
    // for all of them (see k_fwd_stream)
    const bool chain = fin && piv;
    if (t == 0) {
      int ready = 1;
      if (lo < hi) {
        if (!chain) wait_flag_backoff(flags + hi - 1, fa.err, 1024);
        else ready = ld_acquire(flags + hi - 1) != 0;
      }
      s_ready = ready;
    }
    __syncthreads();
    const bool staged = s_ready != 0;
    if (staged) {
#pragma unroll
      for (int j = 0; j < kMrStages; ++j) {
        const int q = lo + j;
        if (q < hi) cp_vec_block(Yst + j * SB * kMrYld, ysl, w, m, SB * q, min(SB, k - SB * q), nr_rhs, ntl);
        cp_async_commit();
      }
    }
    double macc[NTW][4];
#pragma unroll
    for (int j = 0; j < NTW; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) macc[j][e] = 0.0;
    for (int q = lo; q < hi; ++q) {
      const int st = (q - lo) % kMrStages;
      double* Ys = Yst + st * SB * kMrYld;
      if (!staged) {
        if (t == 0) wait_flag(flags + q, fa.err);
        __syncthreads();
        ld_vec_block(Ys, ysl, w, m, SB * q, min(SB, k - SB * q), nr_rhs, ntl);
      }
      cp_async_wait<1>();
      __syncthreads();
      block_dmma<false, NTW>(macc, Lst[st], Ys, ysl, ntl);
      __syncthreads();
      const int qn = q + kMrStages;
      if (qn < hi) {
        cp_block_ls(Lst[st], F, m, r0, nr, SB * qn, min(SB, k - SB * qn));
        if (staged) cp_vec_block(Ys, ysl, w, m, SB * qn, min(SB, k - SB * qn), nr_rhs, ntl);
      }
      cp_async_commit();
    }
    cp_async_wait_all();
    // the tensor-pipe sums to the thread layout through stage 0
    double* Acc = &Lst[0][0][0];
    __syncthreads();
    store_acc<NTW>(macc, Acc, kLdL, ntl);
    __syncthreads();
    double acc[RPT];
#pragma unroll
    for (int j = 0; j < RPT; ++j) {
      const int r = g + 4 * j;
      acc[j] = (r < nr_rhs) ? Acc[i * kLdL + r] : 0.0;
    }
    if (!fin) {
#pragma unroll
      for (int j = 0; j < RPT; ++j) {
        const int r = g + 4 * j;
        if (r < nr_rhs) my_part[i + SB * r] = acc[j];
      }
    } else if (!piv) {
      if (i < nr) {
#pragma unroll
        for (int j = 0; j < RPT; ++j) {
          const int r = g + 4 * j;
          if (r < nr_rhs) w[r0 + i + (int64_t)r * m] -= tot[j] + acc[j];
        }
      }
    } else {
      // y_R = Dinv_R (w_R - sum): z through stage 0 of the vectors, Dinv through stage 1
      double* Zs = Yst;
      double(*Ds)[kLdL] = Lst[1];
      __syncthreads();
#pragma unroll
      for (int j = 0; j < RPT; ++j) {
        const int r = g + 4 * j;
        if (r < nr_rhs) Zs[i * ysl + r] = (i < nr) ? wrow[j] - (tot[j] + acc[j]) : 0.0;
      }
#pragma unroll
      for (int e = 0; e < 16; ++e) {
        const int q = t + 256 * e;
        Ds[q >> 6][q & 63] = dpre[e];
      }
      __syncthreads();
      double y[RPT];
#pragma unroll
      for (int j = 0; j < RPT; ++j) y[j] = 0.0;
#pragma unroll 8
      for (int c = 0; c < SB; ++c) {
        const double l = Ds[c][i];
#pragma unroll
        for (int j = 0; j < RPT; ++j) {
          const int r = g + 4 * j;
          if (r < nr_rhs) y[j] = fma(l, Zs[c * ysl + r], y[j]);
        }
      }
      if (i < nr) {
#pragma unroll
        for (int j = 0; j < RPT; ++j) {
          const int r = g + 4 * j;
          if (r < nr_rhs) w[r0 + i + (int64_t)r * m] = y[j];
        }
      }
    }
    const bool publish = !fin || piv;
    if (t == 0) s_tk[par ^ 1] = next;
    __syncthreads();
    if (t == 0 && publish) {
      if (fin) publish_flag(fa.flags + u.flag0 + R);
      else publish_add(fa.counters + u.cnt);
    }
  }
  cp_async_wait_all();
}

template <int RPT>
__global__ void __launch_bounds__(256, 2) k_bwd_mrhs(const double* __restrict__ L, const double* __restrict__ Dinv,
                                                  double* W, double* part, double* __restrict__ x,
                                                  const int* __restrict__ rows, int64_t ldx, int nr_rhs,
                                                  FusedArgs fa) {
  extern __shared__ __align__(16) unsigned char sm_raw[];
  double(*Lst)[SB][kLdL] = reinterpret_cast<double(*)[SB][kLdL]>(sm_raw);
  double* Wst = reinterpret_cast<double*>(sm_raw + sizeof(double) * kMrStages * SB * kLdL);
  __shared__ int s_tk[2], s_ready;
  constexpr int NTW = (RPT + 3) / 4;
  const int ysl = ys_ld(nr_rhs), ntl = (nr_rhs + 7) / 8;
  const int t = threadIdx.x, c = t & 63, g = t >> 6;
  if (t == 0) s_tk[0] = atomicAdd(fa.ticket, 1);
  __syncthreads();
  for (int par = 0;; par ^= 1) {
    const int tk = s_tk[par];
    if (tk >= fa.count) break;
    int next = 0;
    if (t == 0) next = atomicAdd(fa.ticket, 1);
    const Unit u = load_unit(fa.units, tk);
    const int p = u.R, lo = u.lo, hi = u.hi, m = u.m, k = u.k;
    const bool fin = u.fin != 0;
    const int pb = (k + SB - 1) / SB;
    const int c0 = SB * p, wc = min(SB, k - c0);
    const double* F = L + u.l_off;
    double* w = W + u.w_off * nr_rhs;
    const int* flags = fa.flags + u.flag0;
    auto rows_of = [&](int Rr, int& rr0, int& nrr) {
      rr0 = (Rr < pb) ? SB * Rr : k + SB * (Rr - pb);
      nrr = min(SB, (Rr < pb ? k : m) - rr0);
    };
    // row blocks from the farthest (hi - 1) down to lo
#pragma unroll
    for (int j = 0; j < kMrStages; ++j) {
      const int Rr = hi - 1 - j;
      if (Rr >= lo) {
        int rr0, nrr;
        rows_of(Rr, rr0, nrr);
        cp_block_ls(Lst[j], F, m, rr0, nrr, c0, wc);
      }
      cp_async_commit();
    }
    double dpre[16], wrow[RPT];
    if (fin) {
      const double* D = Dinv + u.dinv_off + (int64_t)p * SB * SB;
#pragma unroll
      for (int e = 0; e < 16; ++e) {
        const int q = t + 256 * e, ii = q & 63, cc = q >> 6;
        dpre[e] = (ii < wc && cc < wc) ? __ldg(D + ii + cc * wc) : 0.0;
      }
#pragma unroll
      for (int j = 0; j < RPT; ++j) {
        const int r = g + 4 * j;
        wrow[j] = (r < nr_rhs && c < wc) ? __ldcg(w + c0 + c + (int64_t)r * m) : 0.0;
      }
    }
    double* my_part = part + (int64_t)u.slot * SB * nr_rhs;
    double tot[RPT];
#pragma unroll
    for (int j = 0; j < RPT; ++j) tot[j] = 0.0;
    if (fin) gather_partials<double, RPT>(my_part, u.nparts, nr_rhs, fa.counters + u.cnt, fa.err, tot);
    // flags are set last column first: flag lo stands for every pivot row block of
    // the range (see k_bwd_stream); update rows need no flag
    if (t == 0) {
      int ready = 1;
      if (lo < hi && lo < pb) {
        if (!fin) wait_flag_backoff(flags + lo, fa.err, 1024);
        else ready = ld_acquire(flags + lo) != 0;
      }
      s_ready = ready;
    }
    __syncthreads();
    const bool staged = s_ready != 0;
    // a row block's x values may be prefetched when staged or when it is an update row
    auto prefetchable = [&](int Rr) { return staged || Rr >= pb; };
#pragma unroll
    for (int j = 0; j < kMrStages; ++j) {
      const int Rr = hi - 1 - j;
      if (Rr >= lo && prefetchable(Rr)) {
        int rr0, nrr;
        rows_of(Rr, rr0, nrr);
        cp_vec_block(Wst + j * SB * kMrYld, ysl, w, m, rr0, nrr, nr_rhs, ntl);
      }
      cp_async_commit();
    }
    double macc[NTW][4];
#pragma unroll
    for (int j = 0; j < NTW; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) macc[j][e] = 0.0;
    for (int Rr = hi - 1; Rr >= lo; --Rr) {
      const int st = (hi - 1 - Rr) % kMrStages;
      double* Ws = Wst + st * SB * kMrYld;
      if (!prefetchable(Rr)) {
        if (t == 0) wait_flag(flags + Rr, fa.err);
        __syncthreads();
        int rr0, nrr;
        rows_of(Rr, rr0, nrr);
        ld_vec_block(Ws, ysl, w, m, rr0, nrr, nr_rhs, ntl);
      }
      cp_async_wait<1>();
      __syncthreads();
      block_dmma<true, NTW>(macc, Lst[st], Ws, ysl, ntl);
      __syncthreads();
      const int Rn = Rr - kMrStages;
      if (Rn >= lo) {
        int rn0, nrn;
        rows_of(Rn, rn0, nrn);
        cp_block_ls(Lst[st], F, m, rn0, nrn, c0, wc);
        if (prefetchable(Rn)) cp_vec_block(Ws, ysl, w, m, rn0, nrn, nr_rhs, ntl);
      }
      cp_async_commit();
    }
    cp_async_wait_all();
    double* Acc = &Lst[0][0][0];
    __syncthreads();
    store_acc<NTW>(macc, Acc, kLdL, ntl);
    __syncthreads();
    double acc[RPT];
#pragma unroll
    for (int j = 0; j < RPT; ++j) {
      const int r = g + 4 * j;
      acc[j] = (r < nr_rhs) ? Acc[c * kLdL + r] : 0.0;
    }
    if (!fin) {
#pragma unroll
      for (int j = 0; j < RPT; ++j) {
        const int r = g + 4 * j;
        if (r < nr_rhs) my_part[c + SB * r] = acc[j];
      }
    } else {
      // x_p = Dinv_p^T (y_p - sum): z through stage 0 of the vectors, Dinv through stage 1
      double* Zs = Wst;
      double(*Ds)[kLdL] = Lst[1];
      __syncthreads();
#pragma unroll
      for (int j = 0; j < RPT; ++j) {
        const int r = g + 4 * j;
        if (r < nr_rhs) Zs[c * ysl + r] = (c < wc) ? wrow[j] - (tot[j] + acc[j]) : 0.0;
      }
#pragma unroll
      for (int e = 0; e < 16; ++e) {
        const int q = t + 256 * e;
        Ds[q >> 6][q & 63] = dpre[e];
      }
      __syncthreads();
      double xv[RPT];
#pragma unroll
      for (int j = 0; j < RPT; ++j) xv[j] = 0.0;
#pragma unroll 8
      for (int ii = 0; ii < SB; ++ii) {
        const double l = Ds[c][ii];
#pragma unroll
        for (int j = 0; j < RPT; ++j) {
          const int r = g + 4 * j;
          if (r < nr_rhs) xv[j] = fma(l, Zs[ii * ysl + r], xv[j]);
        }
      }
      if (c < wc) {
        const int pos = rows[u.w_off + c0 + c];
#pragma unroll
        for (int j = 0; j < RPT; ++j) {
          const int r = g + 4 * j;
          if (r < nr_rhs) {
            w[c0 + c + (int64_t)r * m] = xv[j];
            x[pos + (int64_t)r * ldx] = xv[j];
          }
        }
      }
    }
    if (t == 0) s_tk[par ^ 1] = next;
    __syncthreads();
    if (t == 0) {
      if (fin) publish_flag(fa.flags + u.flag0 + p);
      else publish_add(fa.counters + u.cnt);
    }
  }
  cp_async_wait_all();
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
// dst[i] = (float)src[i], two elements per thread and iteration (16-byte loads
// where the pair is aligned; n may be odd), grid-stride.
__global__ void __launch_bounds__(256) k_round_to_float(const double* __restrict__ src, float* __restrict__ dst,
                                                        int64_t n) {
  const int64_t pairs = n / 2;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < pairs; p += (int64_t)gridDim.x * blockDim.x) {
    const double2 v = __ldcs(reinterpret_cast<const double2*>(src) + p);
    __stcs(reinterpret_cast<float2*>(dst) + p, make_float2((float)v.x, (float)v.y));
  }
  if ((n & 1) && blockIdx.x == 0 && threadIdx.x == 0) dst[n - 1] = (float)src[n - 1];
}

template <class T>
constexpr size_t syrk_smem() { return sizeof(T) * 2 * kTileSyrk * (P + 1); }
template <class T>
constexpr size_t big_smem() { return sizeof(T) * 2 * KC * (kTileBig + kBigCols); }
constexpr size_t dmma_smem() { return sizeof(double) * kDStages * KD * (kLdA + kLdB); }

template <class T>
std::string set_attributes() {
  TDEM_CUDA_TRY(cudaFuncSetAttribute(k_syrk_panel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)syrk_smem<T>()));
  TDEM_CUDA_TRY(cudaFuncSetAttribute(k_syrk_big<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)big_smem<T>()));
  TDEM_CUDA_TRY(cudaFuncSetAttribute(k_syrk_big_dmma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dmma_smem()));
  TDEM_CUDA_TRY(cudaFuncSetAttribute(k_panel_dmma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dmma_smem()));
  TDEM_CUDA_TRY(
      cudaFuncSetAttribute(k_trsm_dmma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)trsm_dmma_smem()));
  TDEM_CUDA_TRY(cudaFuncSetAttribute(k_fwd_diag<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024));
  TDEM_CUDA_TRY(cudaFuncSetAttribute(k_bwd_diag<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024));
  TDEM_CUDA_TRY(cudaFuncSetAttribute(k_fwd_update<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024));
  return "";
}

// Look-ahead of the FP64 panel chain: the update of the outer panel's columns
// right of the next inner panel (syrk_rest) runs on a side stream while the main
// stream factors and solves the next panel.  Per inner panel j:
//   main: potrf_j, trsm_j, wait(rest_{j-1}), record(solved), next_j
//   side: wait(solved), rest_j, record(rest)
// rest_{j-1} and next_j write the same columns (panel j + 1), hence the wait;
// rest_j touches neither panel j + 1 nor the trailing columns of the outer panel
// (the syrk_big input is final once every rest with work has been waited for by
// the next next_; a rest of the outer panel's last two inner panels has none).
// The side stream joins the main one at the end.
struct LookAhead {
  cudaStream_t side = nullptr;
  cudaEvent_t solved = nullptr, rest = nullptr, join = nullptr;
};

template <class T>
int launch_factor(const Symbolic& sy, T* L, T* U, const double* vals, const int64_t* entry, Fronts fr,
                  const int* parent, const int64_t* rel_off, const int* rel, const int* tasks,
                  const int64_t* prefix, int* err, const int* c0, bool use_tc, cudaStream_t s,
                  const OzakiBuffers* oz = nullptr, const int64_t* aux = nullptr,
                  std::vector<cudaEvent_t>* oz_ev = nullptr, size_t* oz_used = nullptr, T* dinv = nullptr,
                  const int64_t* dinv_off = nullptr, const LookAhead* la = nullptr) {
  // dinv (FP64): k_potrf also writes the inverted diagonal blocks, and the panel
  // solves run on the FP64 tensor pipe with them (k_trsm_dmma)
  int launches = 0;
  bool rest_pending = false, side_used = false;
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
      k_potrf<T><<<ps.potrf.count, 256, 0, s>>>(L, fr, tasks + ps.potrf.off, ps.j0, err, c0, dinv, dinv_off);
      ++launches;
      if (ps.trsm.ctas > 0) {
        bool done = false;
        if constexpr (std::is_same<T, double>::value) {
          if (dinv) {
            k_trsm_dmma<<<grid_of(ps.trsm.ctas), 256, trsm_dmma_smem(), s>>>(
                L, fr, tasks + ps.trsm.off, prefix + ps.trsm.pre, ps.trsm.count, ps.j0, dinv, dinv_off);
            done = true;
          }
        }
        if (!done)
          k_trsm<T><<<grid_of(ps.trsm.ctas), kTrsmRows, 0, s>>>(L, fr, tasks + ps.trsm.off, prefix + ps.trsm.pre,
                                                                ps.trsm.count, ps.j0);
        ++launches;
      }
      if (ps.syrk.ctas > 0) {
        if constexpr (std::is_same<T, double>::value) {
          if (la && la->side) {
            if (rest_pending) cudaStreamWaitEvent(s, la->rest, 0);
            rest_pending = false;
            if (ps.syrk_rest.ctas > 0) {
              cudaEventRecord(la->solved, s);
              cudaStreamWaitEvent(la->side, la->solved, 0);
              k_panel_dmma<<<grid_of(ps.syrk_rest.ctas), kBigThreads, dmma_smem(), la->side>>>(
                  L, U, fr, tasks + ps.syrk_rest.off, prefix + ps.syrk_rest.pre, ps.syrk_rest.count, ps.j0, 1);
              cudaEventRecord(la->rest, la->side);
              rest_pending = side_used = true;
              ++launches;
            }
            k_panel_dmma<<<grid_of(ps.syrk_next.ctas), kBigThreads, dmma_smem(), s>>>(
                L, U, fr, tasks + ps.syrk_next.off, prefix + ps.syrk_next.pre, ps.syrk_next.count, ps.j0, 0);
          } else {
            k_panel_dmma<<<grid_of(ps.syrk_wide.ctas), kBigThreads, dmma_smem(), s>>>(
                L, U, fr, tasks + ps.syrk_wide.off, prefix + ps.syrk_wide.pre, ps.syrk_wide.count, ps.j0, 0);
          }
        } else
          k_syrk_panel<T><<<grid_of(ps.syrk.ctas), 256, syrk_smem<T>(), s>>>(L, fr, tasks + ps.syrk.off,
                                                                             prefix + ps.syrk.pre, ps.syrk.count,
                                                                             ps.j0);
        ++launches;
      }
      if (ps.syrk_big.ctas > 0) {
        if constexpr (std::is_same<T, double>::value) {
          if (oz && ps.ozaki) {
            // digits of the panel rows, then the update on the integer tensor pipe
            launch_ozaki_slice(L, fr.l_off, fr.m, fr.k, tasks + ps.oz_slice.off, prefix + ps.oz_slice.pre,
                               aux + ps.oz_slice.off, ps.oz_slice.count, ps.oz_slice.ctas, ps.j0, *oz, s);
            cudaEvent_t ev[2] = {nullptr, nullptr};
            if (oz_ev) {
              while (oz_ev->size() < 2 * (*oz_used + 1)) {
                cudaEvent_t e;
                if (cudaEventCreate(&e) != cudaSuccess) break;
                oz_ev->push_back(e);
              }
              if (oz_ev->size() >= 2 * (*oz_used + 1)) {
                ev[0] = (*oz_ev)[2 * *oz_used];
                ev[1] = (*oz_ev)[2 * *oz_used + 1];
                ++*oz_used;
                cudaEventRecord(ev[0], s);
              }
            }
            launch_ozaki_update(L, U, fr.l_off, fr.u_off, fr.m, fr.k, tasks + ps.syrk_big.off,
                                prefix + ps.syrk_big.pre, aux + ps.syrk_big.off, ps.syrk_big.count,
                                ps.syrk_big.ctas, ps.j0, *oz, err, s);
            if (ev[1]) cudaEventRecord(ev[1], s);
            ++launches;
          } else {
            k_syrk_big_dmma<<<grid_of(2 * ps.syrk_big.ctas), kBigThreads, dmma_smem(), s>>>(
                L, U, fr, tasks + ps.syrk_big.off, prefix + ps.syrk_big.pre, ps.syrk_big.count, ps.j0);
          }
        } else if (use_tc) {
          launch_syrk_tc((float*)L, (float*)U, fr.l_off, fr.u_off, fr.m, fr.k, tasks + ps.syrk_big.off,
                         prefix + ps.syrk_big.pre, ps.syrk_big.count, ps.syrk_big.ctas, ps.j0, err, s);
        } else {
          k_syrk_big<T><<<grid_of(2 * ps.syrk_big.ctas), kBigThreads, big_smem<T>(), s>>>(
              L, U, fr, tasks + ps.syrk_big.off, prefix + ps.syrk_big.pre, ps.syrk_big.count, ps.j0);
        }
        ++launches;
      }
    }
  }
  if (side_used) {
    cudaEventRecord(la->join, la->side);
    cudaStreamWaitEvent(s, la->join, 0);
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

// One forward and one backward launch per level (plus the front-vector set-up).
// STREAM: the persistent streaming kernels (nrhs <= NR <= 4, grid = resident
// CTAs); MR: the persistent many-column kernels (FP64, 3..32 columns, grid =
// resident CTAs); otherwise the one-unit-per-CTA kernels with RPT right-hand
// sides per thread.
template <class T, int RPT, bool STREAM, bool MR = false>
void launch_level_solves(const Symbolic& sy, const T* L, const T* Dinv, T* W, T* part, const double* b, double* x,
                         SolveArgs a, const int* parent, const int64_t* rel_off, const int* rel, const int* tasks,
                         const int64_t* prefix, FusedArgs fa, int* sync, const int (&resident)[2], int& launches,
                         cudaStream_t s) {
  static_assert(!MR || std::is_same<T, double>::value, "the many-column persistent kernels are FP64");
  const int nlev = (int)sy.levels.size();
  int* tickets = sync;
  int* fflags = sync + 2 * nlev;
  int* bflags = fflags + sy.n_flags;
  fa.counters = bflags + sy.n_flags;
  cudaMemsetAsync(sync, 0, sizeof(int) * (2 * nlev + 2 * sy.n_flags + sy.n_counters), s);
  const size_t ysm = STREAM ? stream_smem<T>() : (MR ? mr_smem() : sizeof(T) * SB * ys_ld(a.nrhs));
  auto grid = [&](int64_t count, int dir) {
    return (STREAM || MR) ? (unsigned)std::min<int64_t>(count, resident[dir]) : grid_of(count);
  };
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
    if (lp.fwd_count == 0) continue;
    FusedArgs f = fa;
    f.units = fa.units + (int64_t)kUnitInts * lp.fwd_off;
    f.count = lp.fwd_count;
    f.ticket = tickets + 2 * l;
    f.flags = fflags;
    if constexpr (MR)
      k_fwd_mrhs<RPT><<<grid(lp.fwd_count, 0), 256, ysm, s>>>(L, Dinv, W, part, a.nrhs, f);
    else if constexpr (STREAM)
      k_fwd_stream<T, RPT><<<grid(lp.fwd_count, 0), 256, ysm, s>>>(L, Dinv, W, part, a.nrhs, f);
    else
      k_fwd_level<T, RPT><<<grid(lp.fwd_count, 0), 256, ysm, s>>>(L, Dinv, W, part, a.nrhs, f);
    ++launches;
  }
  for (int l = nlev - 1; l >= 0; --l) {
    const LevelPlan& lp = sy.levels[l];
    k_bwd_init<T><<<grid_of(lp.assemble.ctas), kSolveRows, 0, s>>>(W, x, a, tasks + lp.assemble.off,
                                                                   prefix + lp.assemble.pre, lp.assemble.count);
    ++launches;
    if (lp.bwd_count == 0) continue;
    FusedArgs f = fa;
    f.units = fa.units + (int64_t)kUnitInts * lp.bwd_off;
    f.count = lp.bwd_count;
    f.ticket = tickets + 2 * l + 1;
    f.flags = bflags;
    if constexpr (MR)
      k_bwd_mrhs<RPT><<<grid(lp.bwd_count, 1), 256, ysm, s>>>(L, Dinv, W, part, x, a.rows, a.ld, a.nrhs, f);
    else if constexpr (STREAM)
      k_bwd_stream<T, RPT><<<grid(lp.bwd_count, 1), 256, ysm, s>>>(L, Dinv, W, part, x, a.rows, a.ld, a.nrhs, f);
    else
      k_bwd_level<T, RPT><<<grid(lp.bwd_count, 1), 256, ysm, s>>>(L, Dinv, W, part, x, a.rows, a.ld, a.nrhs, f);
    ++launches;
  }
}

template <class T>
int launch_solve_fused(const Symbolic& sy, const T* L, const T* Dinv, T* W, T* part, const double* b, double* x,
                       SolveArgs a, const int* parent, const int64_t* rel_off, const int* rel, const int* tasks,
                       const int64_t* prefix, FusedArgs fa, int* sync, const int (&resident)[2][2], cudaStream_t s) {
  int launches = 0;
#define TDEM_LEVELS(R, ST, RES) \
  launch_level_solves<T, R, ST>(sy, L, Dinv, W, part, b, x, a, parent, rel_off, rel, tasks, prefix, fa, sync, RES, \
                                launches, s)
  if (a.nrhs == 1)
    TDEM_LEVELS(1, true, resident[0]);
  else if (a.nrhs == 2)
    TDEM_LEVELS(2, true, resident[1]);
  else if (a.nrhs <= 4)
    TDEM_LEVELS(1, false, resident[0]);
  else if (a.nrhs <= 8)
    TDEM_LEVELS(2, false, resident[0]);
  else if (a.nrhs <= 16)
    TDEM_LEVELS(4, false, resident[0]);
  else if (a.nrhs <= 32)
    TDEM_LEVELS(8, false, resident[0]);
  else
    TDEM_LEVELS(16, false, resident[0]);
#undef TDEM_LEVELS
  return launches;
}

// The persistent many-column level solves (FP64, 3 <= nrhs <= 32).
int launch_solve_mr(const Symbolic& sy, const double* L, const double* Dinv, double* W, double* part, const double* b,
                    double* x, SolveArgs a, const int* parent, const int64_t* rel_off, const int* rel,
                    const int* tasks, const int64_t* prefix, FusedArgs fa, int* sync, const int (&resident)[2],
                    cudaStream_t s) {
  int launches = 0;
#define TDEM_MR(R) \
  launch_level_solves<double, R, false, true>(sy, L, Dinv, W, part, b, x, a, parent, rel_off, rel, tasks, prefix, \
                                              fa, sync, resident, launches, s)
  if (a.nrhs <= 4)
    TDEM_MR(1);
  else if (a.nrhs <= 8)
    TDEM_MR(2);
  else if (a.nrhs <= 16)
    TDEM_MR(4);
  else
    TDEM_MR(8);
#undef TDEM_MR
  return launches;
}

// Resident CTAs of the persistent many-column kernels ([forward, backward]).
std::string mr_residency(int (&resident)[2], int sms) {
  const int sm = (int)mr_smem();
  int occ[2][4] = {};
#define TDEM_OCC(J, R)                                                                                              \
  TDEM_CUDA_TRY(cudaFuncSetAttribute(k_fwd_mrhs<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));             \
  TDEM_CUDA_TRY(cudaFuncSetAttribute(k_bwd_mrhs<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));             \
  TDEM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[0][J], k_fwd_mrhs<R>, 256, sm));                \
  TDEM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[1][J], k_bwd_mrhs<R>, 256, sm));
  TDEM_OCC(0, 1)
  TDEM_OCC(1, 2)
  TDEM_OCC(2, 4)
  TDEM_OCC(3, 8)
#undef TDEM_OCC
  for (int d = 0; d < 2; ++d) {
    int least = occ[d][0];
    for (int j = 1; j < 4; ++j) least = std::min(least, occ[d][j]);
    if (least < 1) return "many-column level solve does not fit on an SM";
    resident[d] = least * sms;
  }
  return "";
}

// Resident CTAs on the device of each streaming kernel ([NR = 1, 2][forward, backward]).
template <class T>
std::string stream_residency(int (&resident)[2][2], int& sms) {
  int dev = 0;
  TDEM_CUDA_TRY(cudaGetDevice(&dev));
  TDEM_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int sm = (int)stream_smem<T>();
  TDEM_CUDA_TRY(cudaFuncSetAttribute(k_fwd_stream<T, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
  TDEM_CUDA_TRY(cudaFuncSetAttribute(k_fwd_stream<T, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
  TDEM_CUDA_TRY(cudaFuncSetAttribute(k_bwd_stream<T, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
  TDEM_CUDA_TRY(cudaFuncSetAttribute(k_bwd_stream<T, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
  int occ[2][2] = {};
  TDEM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[0][0], k_fwd_stream<T, 1>, 256, sm));
  TDEM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[1][0], k_fwd_stream<T, 2>, 256, sm));
  TDEM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[0][1], k_bwd_stream<T, 1>, 256, sm));
  TDEM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[1][1], k_bwd_stream<T, 2>, 256, sm));
  for (int j = 0; j < 2; ++j)
    for (int d = 0; d < 2; ++d) {
      if (occ[j][d] < 1) return "streaming level solve does not fit on an SM";
      resident[j][d] = occ[j][d] * sms;
    }
  return "";
}

template <class T>
std::string set_fused_attributes() {
  const int ysm = (int)(sizeof(T) * SB * ys_ld(kMaxRhs));
  TDEM_CUDA_TRY(cudaFuncSetAttribute(k_fwd_level<T, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, ysm));
  TDEM_CUDA_TRY(cudaFuncSetAttribute(k_fwd_level<T, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, ysm));
  TDEM_CUDA_TRY(cudaFuncSetAttribute(k_fwd_level<T, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, ysm));
  TDEM_CUDA_TRY(cudaFuncSetAttribute(k_fwd_level<T, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, ysm));
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
  for (SolveGraph& g : graph_)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  for (cudaEvent_t e : la_ev_)
    if (e) cudaEventDestroy(e);
  if (la_side_) cudaStreamDestroy(la_side_);
  for (cudaEvent_t e : oz_events_) cudaEventDestroy(e);
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

int64_t GpuCholesky::slot_bytes(const Symbolic& sy, int precision_bytes) {
  const int64_t el = (precision_bytes == 4) ? 4 : 8;
  return el * (std::max<int64_t>(1, sy.nnz_l) + std::max<int64_t>(1, sy.dinv_elems));
}

int64_t GpuCholesky::bytes_needed(const Symbolic& sy, int nrhs_max, int precision_bytes, int nslots,
                                  int factor_bytes) {
  const int64_t el = (precision_bytes == 4) ? 4 : 8, nr = std::max(1, nrhs_max);
  const int64_t fel = factor_bytes == 0 ? el : (factor_bytes == 4 ? 4 : 8);
  int64_t b = fel * sy.u_elems + el * (sy.wvec_elems * nr + sy.solve_partials * nr + sy.solve_slots * kPanel * nr);
  b += std::max(1, std::min(nslots, kMaxSlots)) * slot_bytes(sy, precision_bytes);
  if (fel != el) b += slot_bytes(sy, (int)fel);  // the FP64 work factor of a demoted setup
  if (fel == 8) b += sy.oz_rows_max * ((int64_t)kOzSlices * kOzK + 4);  // digit slices + exponents
  b += 8 * (int64_t)sy.task_aux.size();
  b += 8 * (int64_t)(sy.l_off.size() + sy.u_off.size() + sy.wvec_off.size() + sy.entry_dst.size() +
                     sy.rel_off.size() + sy.rows_off.size() + sy.task_prefix.size() + sy.dinv_off.size());
  b += 4 * (int64_t)(sy.front_m.size() + sy.front_k.size() + sy.rel.size() + sy.rows_all.size() + sy.tasks.size() +
                     sy.front_parent.size() + sy.front_c0.size() + sy.solve_items.size() + sy.solve_units.size() +
                     2 * sy.levels.size() + 2 * sy.n_flags + sy.n_counters + 4);
  return b;
}

std::string GpuCholesky::setup(Symbolic&& sy, const std::vector<int>& perm_to_vec, int nrhs_max,
                               cudaStream_t s, int precision_bytes, int nslots, int factor_bytes) {
  sy_ = std::move(sy);
  nrhs_max_ = std::max(1, nrhs_max);
  elem_ = (precision_bytes == 4) ? 4 : 8;
  fac_elem_ = factor_bytes == 0 ? elem_ : (factor_bytes == 4 ? 4 : 8);
  if (fac_elem_ < elem_) return "the factorization cannot be less precise than the held factor";
  if ((int)perm_to_vec.size() != sy_.n) return "perm_to_vec size mismatch";
  if (nrhs_max_ > kMaxRhs) return "too many right-hand sides";
  if (nslots < 1 || nslots > kMaxSlots) return "factor slots must be 1 or 2";
  nslots_ = nslots;
  std::string e;
  for (int k = 0; k < nslots_; ++k) {
    if (!(e = alloc(&d_L_[k], elem_ * std::max<int64_t>(1, sy_.nnz_l))).empty()) return e;
    if (!(e = alloc(&d_dinv_[k], elem_ * std::max<int64_t>(1, sy_.dinv_elems))).empty()) return e;
  }
  if (demoted()) {
    if (!(e = alloc(&d_Lw_, sizeof(double) * std::max<int64_t>(1, sy_.nnz_l))).empty()) return e;
    if (!(e = alloc(&d_dinvw_, sizeof(double) * std::max<int64_t>(1, sy_.dinv_elems))).empty()) return e;
  }
  if (!(e = alloc(&d_U_, fac_elem_ * std::max<int64_t>(1, sy_.u_elems))).empty()) return e;
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
  if (!(e = upload(&d_task_aux_, sy_.task_aux, s)).empty()) return e;
  if (fac_elem_ == 8 && ozaki_ && sy_.oz_rows_max > 0) {
    oz_.rows = sy_.oz_rows_max;
    if (!(e = alloc((void**)&oz_.slices, (size_t)kOzSlices * kOzK * oz_.rows)).empty()) return e;
    if (!(e = alloc((void**)&oz_.exps, sizeof(int) * (size_t)oz_.rows)).empty()) return e;
    if (!(e = ozaki_setup(oz_)).empty()) return e;
  }
  if (!(e = upload(&d_parent_, sy_.front_parent, s)).empty()) return e;
  if (!(e = upload(&d_c0_, sy_.front_c0, s)).empty()) return e;
  if (!(e = upload(&d_items_, sy_.solve_items, s)).empty()) return e;
  if (!(e = upload(&d_dinv_off_, sy_.dinv_off, s)).empty()) return e;
  if (!(e = upload(&d_units_, sy_.solve_units, s)).empty()) return e;
  if (!(e = alloc(&d_spart_, elem_ * std::max<int64_t>(1, sy_.solve_slots) * kPanel * nrhs_max_)).empty()) return e;
  if (!(e = alloc((void**)&d_sync_,
                  sizeof(int) * (2 * sy_.levels.size() + 2 * sy_.n_flags + sy_.n_counters + 1))).empty())
    return e;
  if (!(e = alloc((void**)&d_err_, 3 * sizeof(int))).empty()) return e;
  TDEM_CUDA_TRY(cudaMemsetAsync(d_err_, 0, 3 * sizeof(int), s));
  if (fac_elem_ == 4 && tc_update_ && !(e = tc_update_setup()).empty()) return e;
  if (!(e = (elem_ == 4 ? set_attributes<float>() : set_attributes<double>())).empty()) return e;
  if (demoted() && !(e = set_attributes<double>()).empty()) return e;
  if (!(e = (elem_ == 4 ? set_fused_attributes<float>() : set_fused_attributes<double>())).empty()) return e;
  if (!(e = (elem_ == 4 ? stream_residency<float>(resident_, sms_) : stream_residency<double>(resident_, sms_)))
           .empty())
    return e;
  if (elem_ == 8 && !(e = mr_residency(resident_mr_, sms_)).empty()) return e;
  TDEM_CUDA_TRY(cudaStreamSynchronize(s));
  return "";
}

bool GpuCholesky::lookahead_ready(cudaStream_t s) {
  if (!lookahead_) return false;
  int prio = 0;
  if (cudaStreamGetPriority(s, &prio) != cudaSuccess) return false;
  if (la_side_ && prio != la_prio_) {
    cudaStreamSynchronize(la_side_);
    cudaStreamDestroy(la_side_);
    la_side_ = nullptr;
  }
  if (!la_side_) {
    if (cudaStreamCreateWithPriority(&la_side_, cudaStreamNonBlocking, prio) != cudaSuccess) {
      la_side_ = nullptr;
      return false;
    }
    la_prio_ = prio;
  }
  for (cudaEvent_t& e : la_ev_)
    if (!e && cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
      e = nullptr;
      return false;
    }
  return true;
}

void GpuCholesky::factor(const double* d_vals, cudaStream_t s, int slot) {
  Fronts fr{d_l_off_, d_u_off_, d_m_, d_k_};
  LookAhead la;
  if (elem_ == 8 || demoted()) {
    if (lookahead_ready(s)) {
      la.side = la_side_;
      la.solved = la_ev_[0];
      la.rest = la_ev_[1];
      la.join = la_ev_[2];
    }
  }
  const unsigned ni = (unsigned)sy_.inv_count;
  const size_t ism = 2 * sizeof(double) * SB * (SB + 1);
  void* Lp = d_L_[slot];
  void* Dp = d_dinv_[slot];
  if (demoted()) {
    // FP64 factorization into the work factor, then both arrays rounded into the slot
    launches_factor_ = launch_factor<double>(sy_, (double*)d_Lw_, (double*)d_U_, d_vals, d_entry_, fr, d_parent_,
                                             d_rel_off_, d_rel_, d_tasks_, d_prefix_, d_err_, d_c0_, false, s,
                                             ozaki() ? &oz_ : nullptr, d_task_aux_,
                                             oz_timing_ ? &oz_events_ : nullptr, &oz_used_, (double*)d_dinvw_,
                                             d_dinv_off_, &la);
    const int64_t nl = std::max<int64_t>(1, sy_.nnz_l), nd = std::max<int64_t>(1, sy_.dinv_elems);
    k_round_to_float<<<(unsigned)std::min<int64_t>((nl / 2 + 255) / 256, 148 * 16), 256, 0, s>>>(
        (const double*)d_Lw_, (float*)Lp, nl);
    k_round_to_float<<<(unsigned)std::min<int64_t>((nd / 2 + 255) / 256, 148 * 16), 256, 0, s>>>(
        (const double*)d_dinvw_, (float*)Dp, nd);
    launches_factor_ += 2;
    return;
  }
  if (elem_ == 4) {
    launches_factor_ = launch_factor<float>(sy_, (float*)Lp, (float*)d_U_, d_vals, d_entry_, fr, d_parent_,
                                            d_rel_off_, d_rel_, d_tasks_, d_prefix_, d_err_, d_c0_, tc_update_, s);
    if (ni) k_diag_inverse<float><<<ni, 256, ism, s>>>((const float*)Lp, (float*)Dp, fr, d_dinv_off_,
                                                       d_items_ + 2 * sy_.inv_off);
  } else {
    launches_factor_ = launch_factor<double>(sy_, (double*)Lp, (double*)d_U_, d_vals, d_entry_, fr, d_parent_,
                                             d_rel_off_, d_rel_, d_tasks_, d_prefix_, d_err_, d_c0_, false, s,
                                             ozaki() ? &oz_ : nullptr, d_task_aux_,
                                             oz_timing_ ? &oz_events_ : nullptr, &oz_used_, (double*)Dp,
                                             d_dinv_off_, &la);
    return;
  }
  if (ni) ++launches_factor_;
}

SolveSchedule GpuCholesky::schedule_for(int nrhs) const {
  SolveSchedule d;
  if (panel_solve_) {
    d.kind = 1;
    return d;
  }
  if (has_forced_ && nrhs > 2) return forced_;
  for (const auto& t : tuned_)
    if (t.first == nrhs) return t.second;
  return d;
}

void GpuCholesky::solve(const double* d_b, double* d_x, int64_t ld, int nrhs, cudaStream_t s, int slot) {
  solve_with(schedule_for(nrhs), d_b, d_x, ld, nrhs, s, slot);
}

void GpuCholesky::solve_with(const SolveSchedule& sc, const double* d_b, double* d_x, int64_t ld, int nrhs,
                             cudaStream_t s, int slot) {
  if (sc.split > 1 && nrhs > 1) {
    // column groups one after another (each its own complete solve)
    const int per = (nrhs + sc.split - 1) / sc.split;
    SolveSchedule one = sc;
    one.split = 1;
    int total = 0;
    for (int c = 0; c < nrhs; c += per) {
      solve_with(one, d_b + (int64_t)c * ld, d_x + (int64_t)c * ld, ld, std::min(per, nrhs - c), s, slot);
      total += launches_solve_;
    }
    launches_solve_ = total;
    return;
  }
  SolveArgs a{d_l_off_, d_w_off_, d_m_, d_k_, d_rows_off_, d_rows_, nrhs, ld};
  const void* Lp = d_L_[slot];
  const void* Dp = d_dinv_[slot];
  if (sc.kind == 2 && elem_ == 8 && nrhs > 2 && nrhs <= 32) {
    FusedArgs fa{d_units_, 0, nullptr, nullptr, nullptr, d_err_ + 1};
    int res[2];
    for (int d = 0; d < 2; ++d)
      res[d] = solve_ctas_cap_ > 0 ? std::min(resident_mr_[d], solve_ctas_cap_ * sms_) : resident_mr_[d];
    launches_solve_ = launch_solve_mr(sy_, (const double*)Lp, (const double*)Dp, (double*)d_W_, (double*)d_spart_,
                                      d_b, d_x, a, d_parent_, d_rel_off_, d_rel_, d_tasks_, d_prefix_, fa, d_sync_,
                                      res, s);
    return;
  }
  if (sc.kind != 1) {
    FusedArgs fa{d_units_, 0, nullptr, nullptr, nullptr, d_err_ + 1};
    int res[2][2];
    for (int j = 0; j < 2; ++j)
      for (int d = 0; d < 2; ++d)
        res[j][d] = solve_ctas_cap_ > 0 ? std::min(resident_[j][d], solve_ctas_cap_ * sms_) : resident_[j][d];
    if (elem_ == 4)
      launches_solve_ = launch_solve_fused<float>(sy_, (const float*)Lp, (const float*)Dp, (float*)d_W_,
                                                  (float*)d_spart_, d_b, d_x, a, d_parent_, d_rel_off_, d_rel_,
                                                  d_tasks_, d_prefix_, fa, d_sync_, res, s);
    else
      launches_solve_ = launch_solve_fused<double>(sy_, (const double*)Lp, (const double*)Dp, (double*)d_W_,
                                                   (double*)d_spart_, d_b, d_x, a, d_parent_, d_rel_off_, d_rel_,
                                                   d_tasks_, d_prefix_, fa, d_sync_, res, s);
    return;
  }
  if (elem_ == 4)
    launches_solve_ = launch_solve<float>(sy_, (const float*)Lp, (float*)d_W_, (float*)d_part_, d_b, d_x, a,
                                          d_parent_, d_rel_off_, d_rel_, d_tasks_, d_prefix_, s);
  else
    launches_solve_ = launch_solve<double>(sy_, (const double*)Lp, (double*)d_W_, (double*)d_part_, d_b, d_x, a,
                                           d_parent_, d_rel_off_, d_rel_, d_tasks_, d_prefix_, s);
}

// Times every candidate schedule for nrhs columns on the factor in `slot` (stream
// s, CUDA events, the median of three solves after one warm-up each) with scratch
// copies of zero right-hand sides, and keeps the fastest.  Run before the solve's
// graph is captured, so the graph replays the chosen schedule.
std::string GpuCholesky::tune_solve(int nrhs, int64_t ld, cudaStream_t s, int slot) {
  std::vector<SolveSchedule> cand;
  for (int kind = 0; kind < 3; ++kind)
    for (int split : {1, 2, 4})
      if ((split == 1 || nrhs / split >= 2) &&
          (kind != 2 || (elem_ == 8 && (nrhs + split - 1) / split > 2 && (nrhs + split - 1) / split <= 32))) {
        SolveSchedule c;
        c.kind = kind;
        c.split = split;
        cand.push_back(c);
      }
  double* tb = nullptr;
  const size_t vb = sizeof(double) * (size_t)ld * nrhs;
  TDEM_CUDA_TRY(cudaMallocAsync((void**)&tb, 2 * vb, s));
  struct Free {
    double* p;
    cudaStream_t s;
    ~Free() { cudaFreeAsync(p, s); }
  } fr{tb, s};
  TDEM_CUDA_TRY(cudaMemsetAsync(tb, 0, 2 * vb, s));
  cudaEvent_t ev[2];
  TDEM_CUDA_TRY(cudaEventCreate(&ev[0]));
  TDEM_CUDA_TRY(cudaEventCreate(&ev[1]));
  std::string err;
  size_t best = 0;
  for (size_t i = 0; i < cand.size() && err.empty(); ++i) {
    solve_with(cand[i], tb, tb + (size_t)ld * nrhs, ld, nrhs, s, slot);  // warm-up
    float t[3];
    for (float& ti : t) {
      cudaEventRecord(ev[0], s);
      solve_with(cand[i], tb, tb + (size_t)ld * nrhs, ld, nrhs, s, slot);
      cudaEventRecord(ev[1], s);
      if (cudaEventSynchronize(ev[1]) != cudaSuccess || cudaEventElapsedTime(&ti, ev[0], ev[1]) != cudaSuccess) {
        err = "CUDA: solve autotuner timing failed";
        break;
      }
    }
    std::sort(t, t + 3);
    cand[i].ms = t[1];
    if (cand[i].ms < cand[best].ms) best = i;
  }
  cudaEventDestroy(ev[0]);
  cudaEventDestroy(ev[1]);
  if (!err.empty()) return err;
  TDEM_CUDA_TRY(cudaGetLastError());
  tuned_.emplace_back(nrhs, cand[best]);
  tune_log_.emplace_back(nrhs, cand);
  return "";
}

std::string GpuCholesky::solve_graph(const double* d_b, double* d_x, int64_t ld, int nrhs, cudaStream_t s,
                                     int slot) {
  SolveGraph& sg = graph_[slot];
  if (autotune_ && !panel_solve_ && !has_forced_ && nrhs > 2) {
    bool known = false;
    for (const auto& t : tuned_) known = known || t.first == nrhs;
    if (!known) {
      const std::string e = tune_solve(nrhs, ld, s, slot);
      if (!e.empty()) return e;
    }
  }
  if (!sg.exec || sg.b != d_b || sg.x != d_x || sg.ld != ld || sg.nrhs != nrhs) {
    if (sg.exec) {
      cudaGraphExecDestroy(sg.exec);
      sg.exec = nullptr;
    }
    cudaGraph_t g = nullptr;
    TDEM_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    solve(d_b, d_x, ld, nrhs, s, slot);
    TDEM_CUDA_TRY(cudaStreamEndCapture(s, &g));
    const cudaError_t ie = cudaGraphInstantiate(&sg.exec, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) {
      sg.exec = nullptr;
      return std::string("cudaGraphInstantiate: ") + cudaGetErrorString(ie);
    }
    sg.b = d_b;
    sg.x = d_x;
    sg.ld = ld;
    sg.nrhs = nrhs;
  }
  TDEM_CUDA_TRY(cudaGraphLaunch(sg.exec, s));
  return "";
}

double GpuCholesky::take_ozaki_ms() {
  double tot = 0.0;
  for (size_t i = 0; i < oz_used_; ++i) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, oz_events_[2 * i], oz_events_[2 * i + 1]) == cudaSuccess) tot += ms;
  }
  oz_used_ = 0;
  return tot;
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
