// FEM kernels of the transient solve (see fem_kernels.h).
//
// Local matrices of the lowest-order Nedelec brick element.  With hx, hy, hz the
// brick edges, the reference-cube coordinates in [-1, 1], L0 = (1 - t)/2,
// L1 = (1 + t)/2 and the basis of local edge j scaled by 2/h along its axis
// (CalcNonstat3DLine/T_Brick.cpp:741-836: edges 0-3 along x indexed by (y, z)
// sides, 4-7 along y by (z, x), 8-11 along z by (x, y)), the 1D integrals
//   M1[a][b] = int La Lb = {2/3, 1/3},  K1[a][b] = int La' Lb' = s_a s_b / 2,
//   int La = 1,  int La' = s_a  (s_0 = -1, s_1 = +1)
// give closed forms for the mass matrix C (T_Brick.cpp:311-474) and the curl-curl
// matrix B (T_Brick.cpp:142-310); they are evaluated entry by entry here.
#include "fem_kernels.h"

#include <algorithm>

namespace tdem {
namespace {

__device__ __forceinline__ double m1(int a, int b) { return a == b ? (2.0 / 3.0) : (1.0 / 3.0); }
__device__ __forceinline__ double k1(int a, int b) { return a == b ? 0.5 : -0.5; }
__device__ __forceinline__ double sg(int a) { return a ? 1.0 : -1.0; }

// direction (0 = x, 1 = y, 2 = z) and the two side indices (first, second) of local edge j
__device__ __forceinline__ void edge_desc(int j, int& dir, int& p, int& q) {
  dir = j >> 2;
  p = j & 1;          // first side index
  q = (j >> 1) & 1;   // second side index
}

// Mass and curl-curl entries between local edges i and j of a brick.
__device__ void local_entry(int i, int j, double hx, double hy, double hz, double& c, double& b) {
  int di, ai, bi, dj, aj, bj;
  edge_desc(i, di, ai, bi);
  edge_desc(j, dj, aj, bj);
  const double h[3] = {hx, hy, hz};
  c = 0.0;
  b = 0.0;
  if (di == dj) {
    // edge along axis d; its sides are the two other axes (u, v) in the order
    // x: (y, z), y: (z, x), z: (x, y)
    const int u = (di + 1) % 3, v = (di + 2) % 3;
    const double scale = h[u] * h[v] / h[di];
    c = scale * m1(ai, aj) * m1(bi, bj);
    // curl components along u and v
    b = scale * (4.0 / (h[v] * h[v]) * m1(ai, aj) * k1(bi, bj) +
                 4.0 / (h[u] * h[u]) * k1(ai, aj) * m1(bi, bj));
    return;
  }
  // different directions: the curls share the component along the third axis w
  // (x-edge with y-edge -> z; y with z -> x; x with z -> y)
  int dA = di, aA = ai, bA = bi, dB = dj, aB = aj, bB = bj;
  if ((dA + 1) % 3 != dB) {  // order the pair so that dB follows dA cyclically
    dA = dj; aA = aj; bA = bj;
    dB = di; aB = ai; bB = bi;
  }
  const int w = (dA + 2) % 3;  // shared curl component
  // Edge along dA has sides (dA+1, dA+2) = (dB, w): index aA on dB, bA on w.
  // Edge along dB has sides (dB+1, dB+2) = (w, dA): index aB on w, bB on dA.
  // Integral: -(2 h_w / (h_dA h_dB)) * s(aA) * s(bB) * M1(bA, aB).
  b = -(2.0 * h[w] / (h[dA] * h[dB])) * sg(aA) * sg(bB) * m1(bA, aB);
}

__global__ void k_assemble(ElemDev E, const int* __restrict__ elems, int nelems,
                           const int64_t* __restrict__ rowptr, const int* __restrict__ col,
                           double* __restrict__ Cval, double* __restrict__ Bval) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= (int64_t)nelems * 144) return;
  const int e = elems[t / 144];
  const int ij = (int)(t % 144), i = ij / 12, j = ij % 12;
  const int gi = E.ed[e * 12 + i], gj = E.ed[e * 12 + j];
  double c, b;
  local_entry(i, j, E.h[3 * e], E.h[3 * e + 1], E.h[3 * e + 2], c, b);
  // locate column gj in row gi
  int64_t lo = rowptr[gi], hi = rowptr[gi + 1] - 1;
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (col[mid] < gj) lo = mid + 1;
    else hi = mid;
  }
  if (col[lo] != gj) return;  // cannot happen for a pattern built from the same elements
  Cval[lo] += c * E.sigma[e];
  if (Bval) Bval[lo] += b * E.inv_mu[e];
}

__global__ void k_normal_field(const float* __restrict__ f, const int* __restrict__ idx,
                               const double* __restrict__ len, int nanom, int n, int npls,
                               double* __restrict__ En) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= (int64_t)nanom * npls) return;
  const int p = (int)(t / nanom), k = (int)(t % nanom);
  En[idx[k] + (int64_t)p * n] = (double)f[t] * len[k] * 0.5;
}

// One warp per row: rhs += C_dsigma * En (time_approx.cpp:682, mult_symmetr on the
// lower-stored C_dsigma; here the full symmetric pattern).
__global__ void k_anomaly_rhs(const int64_t* __restrict__ rowptr, const int* __restrict__ col,
                              const double* __restrict__ Cds, const double* __restrict__ En,
                              const uint8_t* __restrict__ bound, int n, int npls, double* __restrict__ rhs) {
  const int row = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (row >= n || bound[row]) return;
  const int64_t b = rowptr[row], e = rowptr[row + 1];
  for (int p = 0; p < npls; ++p) {
    const double* x = En + (int64_t)p * n;
    double acc = 0.0;
    for (int64_t q = b + lane; q < e; q += 32) acc = fma(Cds[q], x[col[q]], acc);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if (lane == 0) rhs[row + (int64_t)p * n] += acc;
  }
}

__global__ void k_combine(const double* __restrict__ C, const double* __restrict__ B,
                          const int64_t* __restrict__ src, const uint8_t* __restrict__ diag, int64_t nnz,
                          double mult, double* __restrict__ out) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nnz;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = src[q];
    double v = C[p] * mult + B[p];
    if (diag[q]) v += v * 1e-12;
    out[q] = v;
  }
}

// Eight lanes per row, four rows per warp: a row holds about 33 entries, so each
// lane takes four or five of them (a warp per row would leave most lanes idle on
// the second pass and spend five shuffle steps per row), and three shuffle steps
// within the group of eight combine the lanes.  Every lane reaches the shuffles.
constexpr int kRhsLanes = 8;
__global__ void k_history_rhs(const int64_t* __restrict__ rowptr, const int* __restrict__ col,
                              const double* __restrict__ C, const double* __restrict__ u1,
                              const double* __restrict__ u2, double m1c, double m2c,
                              const double* __restrict__ S, double coef, const uint8_t* __restrict__ bound,
                              int n, int npls, double* __restrict__ rhs) {
  const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int row = (int)(tid / kRhsLanes);
  const int sub = threadIdx.x & (kRhsLanes - 1);
  const bool live = row < n;
  const bool zero = live && bound[row] != 0;
  int64_t b = 0, e = 0;
  if (live && !zero) {
    b = __ldg(rowptr + row);
    e = __ldg(rowptr + row + 1);
  }
  for (int p = 0; p < npls; ++p) {
    const double* a1 = u1 + (int64_t)p * n;
    const double* a2 = u2 + (int64_t)p * n;
    double acc = 0.0;
    for (int64_t q = b + sub; q < e; q += kRhsLanes) {
      const int j = __ldg(col + q);
      acc = fma(__ldg(C + q), a1[j] * m1c + a2[j] * m2c, acc);
    }
#pragma unroll
    for (int o = kRhsLanes / 2; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o, kRhsLanes);
    if (live && sub == 0) {
      double v = zero ? 0.0 : acc;
      if (!zero && coef != 0.0) v += coef * S[row + (int64_t)p * n];
      rhs[row + (int64_t)p * n] = v;
    }
  }
}

// Several sources: one warp per row, the sources in groups of 8.  Lane l takes the
// entries q = b + l, b + l + 32, ... of the row (the row's columns and values are
// read once per group, not once per source) and sums its products for the 8
// sources; the 32 lanes' sums are combined by recursive halving (each round a
// lane keeps half of its values and adds its partner's other half), after which
// lane l holds the row total of source 4 ((l >> 4) & 1) + 2 ((l >> 3) & 1) +
// ((l >> 2) & 1) of the group.  The additions happen in an order fixed by the
// lane pattern alone.
__global__ void k_history_rhs_multi(const int64_t* __restrict__ rowptr, const int* __restrict__ col,
                                    const double* __restrict__ C, const double* __restrict__ u1,
                                    const double* __restrict__ u2, double m1c, double m2c,
                                    const double* __restrict__ S, double coef, const uint8_t* __restrict__ bound,
                                    int n, int npls, double* __restrict__ rhs) {
  const int row = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (row >= n) return;
  if (bound[row]) {
    for (int p = lane; p < npls; p += 32) rhs[row + (int64_t)p * n] = 0.0;
    return;
  }
  const int64_t b = rowptr[row], e = rowptr[row + 1];
  for (int p0 = 0; p0 < npls; p0 += 8) {
    double v[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) v[r] = 0.0;
    for (int64_t q = b + lane; q < e; q += 32) {
      const double c = C[q];
      const int64_t j = col[q];
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        const int64_t off = j + (int64_t)(p0 + r) * n;
        if (p0 + r < npls) v[r] = fma(c, m2c != 0.0 ? u1[off] * m1c + u2[off] * m2c : u1[off] * m1c, v[r]);
      }
    }
    double a4[4], a2[2];
    bool up = (lane & 16) != 0;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const double mine = up ? v[4 + r] : v[r], other = up ? v[r] : v[4 + r];
      a4[r] = mine + __shfl_xor_sync(0xffffffffu, other, 16);
    }
    up = (lane & 8) != 0;
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const double mine = up ? a4[2 + r] : a4[r], other = up ? a4[r] : a4[2 + r];
      a2[r] = mine + __shfl_xor_sync(0xffffffffu, other, 8);
    }
    up = (lane & 4) != 0;
    double a1 = (up ? a2[1] : a2[0]) + __shfl_xor_sync(0xffffffffu, up ? a2[0] : a2[1], 4);
    a1 += __shfl_xor_sync(0xffffffffu, a1, 2);
    a1 += __shfl_xor_sync(0xffffffffu, a1, 1);
    if ((lane & 3) == 0) {
      const int p = p0 + 4 * ((lane >> 4) & 1) + 2 * ((lane >> 3) & 1) + ((lane >> 2) & 1);
      if (p < npls) {
        double t = a1;
        if (coef != 0.0) t += coef * S[row + (int64_t)p * n];
        rhs[row + (int64_t)p * n] = t;
      }
    }
  }
}

__global__ void k_receivers(const int64_t* __restrict__ rowptr, const int* __restrict__ col,
                            const double* __restrict__ val, const int* __restrict__ src, int nrows,
                            const double* __restrict__ u, int64_t ld, double* __restrict__ out) {
  const int row = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (row >= nrows) return;
  const double* x = u + (int64_t)src[row] * ld;
  double acc = 0.0;
  for (int64_t q = rowptr[row] + lane; q < rowptr[row + 1]; q += 32) acc = fma(val[q], x[col[q]], acc);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if (lane == 0) out[row] = acc;
}

__global__ void k_time_diff(const double* __restrict__ F, int nt, int nser, int t0,
                            const double* __restrict__ time, const int* __restrict__ vpre1,
                            const int* __restrict__ vpre2, int scheme, double sign, double* __restrict__ out) {
  const int sidx = blockIdx.x * blockDim.x + threadIdx.x;
  if (sidx >= nser || nt < 3) return;
  auto val = [&](int layer) { return F[(int64_t)(layer - t0) * nser + sidx]; };
  auto put = [&](int layer, double v) { out[(int64_t)(layer - t0) * nser + sidx] = sign * v; };
  const int tl = t0 + nt - 1;
  int j = t0, j1 = j + 1, j2 = j1 + 1;
  double f0 = val(j), f1 = val(j1), f2 = val(j2);
  double dt = time[j2] - time[j], dt1 = time[j1] - time[j], dt0 = time[j2] - time[j1];
  double mt0 = -(dt + dt1) / (dt1 * dt), mt1 = dt / (dt1 * dt0), mt2 = -dt1 / (dt * dt0);
  put(j, f0 * mt0 + f1 * mt1 + f2 * mt2);
  for (;;) {
    if (scheme == 2) {
      mt0 = -1.0 / (time[j1] - time[j]);
      mt1 = 1.0 / (time[j1] - time[j]);
      mt2 = 0.0;
    } else {
      mt0 = (-dt0) / (dt1 * dt);
      mt1 = -(dt1 - dt0) / (dt1 * dt0);
      mt2 = (dt1) / (dt * dt0);
    }
    put(j1, f0 * mt0 + f1 * mt1 + f2 * mt2);
    if (j2 == tl) break;
    ++j2;
    if (scheme == 2) {
      j = vpre2[j2];
      j1 = vpre1[j2];
    } else {
      j = j1;
      j1 = vpre1[j2];
    }
    f2 = val(j2);
    f0 = val(j);
    f1 = val(j1);
    dt = time[j2] - time[j];
    dt1 = time[j1] - time[j];
    dt0 = time[j2] - time[j1];
  }
  if (scheme == 2) {
    mt0 = 0.0;
    mt1 = -1.0 / (time[j2] - time[j1]);
    mt2 = 1.0 / (time[j2] - time[j1]);
  } else {
    mt0 = (dt0) / (dt1 * dt);
    mt1 = -(dt) / (dt1 * dt0);
    mt2 = (dt + dt0) / (dt * dt0);
  }
  put(j2, f0 * mt0 + f1 * mt1 + f2 * mt2);
}

__global__ void k_combine_full(const int64_t* __restrict__ rowptr, const int* __restrict__ col,
                               const double* __restrict__ C, const double* __restrict__ B,
                               const uint8_t* __restrict__ bound, int n, double mult, double* __restrict__ A) {
  const int row = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (row >= n) return;
  const bool brow = bound[row];
  for (int64_t q = rowptr[row] + lane; q < rowptr[row + 1]; q += 32) {
    const int j = col[q];
    double v = C[q] * mult + B[q];
    if (j == row) v += v * 1e-12;
    A[q] = (brow || bound[j]) ? 0.0 : v;
  }
}

__global__ void k_spmv(const int64_t* __restrict__ rowptr, const int* __restrict__ col,
                       const double* __restrict__ A, const double* __restrict__ x, int n, int npls,
                       double* __restrict__ y) {
  const int row = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (row >= n) return;
  const int64_t b = rowptr[row], e = rowptr[row + 1];
  for (int p = 0; p < npls; ++p) {
    const double* xp = x + (int64_t)p * n;
    double acc = 0.0;
    for (int64_t q = b + lane; q < e; q += 32) acc = fma(A[q], xp[col[q]], acc);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if (lane == 0) y[row + (int64_t)p * n] = acc;
  }
}

// Block partial sums of a . b per column into work[col * kDotBlocks + block].
__device__ __forceinline__ void block_reduce_store(double v, double* out) {
  __shared__ double red[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if (lane == 0) red[warp] = v;
  __syncthreads();
  if (warp == 0) {
    v = (lane < (int)(blockDim.x >> 5)) ? red[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) *out = v;
  }
  __syncthreads();
}

__global__ void k_dot_partial(const double* __restrict__ a, const double* __restrict__ b, int n, int npls,
                              double* __restrict__ work) {
  for (int p = 0; p < npls; ++p) {
    const double* ap = a + (int64_t)p * n;
    const double* bp = b + (int64_t)p * n;
    double v = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
      v = fma(ap[i], bp[i], v);
    block_reduce_store(v, work + (int64_t)p * kDotBlocks + blockIdx.x);
  }
}

__global__ void k_dot_final(const double* __restrict__ work, int npls, double* __restrict__ out) {
  const int p = blockIdx.x;
  double v = 0.0;
  for (int i = threadIdx.x; i < kDotBlocks; i += blockDim.x) v += work[(int64_t)p * kDotBlocks + i];
  __shared__ double red[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if (lane == 0) red[warp] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    if (p < npls) out[p] = t;
  }
}

__global__ void k_pcg_step(const double* __restrict__ rz, const double* __restrict__ pq, double* __restrict__ x,
                           double* __restrict__ r, const double* __restrict__ p, const double* __restrict__ q, int n,
                           int npls, double* __restrict__ work) {
  for (int c = 0; c < npls; ++c) {
    const double alpha = (pq[c] != 0.0) ? rz[c] / pq[c] : 0.0;
    const int64_t o = (int64_t)c * n;
    double v = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
      x[o + i] = fma(alpha, p[o + i], x[o + i]);
      const double ri = fma(-alpha, q[o + i], r[o + i]);
      r[o + i] = ri;
      v = fma(ri, ri, v);
    }
    block_reduce_store(v, work + (int64_t)c * kDotBlocks + blockIdx.x);
  }
}

__global__ void k_pcg_dir(double* __restrict__ rz, const double* __restrict__ rz_new, const double* __restrict__ z,
                          double* __restrict__ p, int n, int npls) {
  for (int c = 0; c < npls; ++c) {
    const double beta = (rz[c] != 0.0) ? rz_new[c] / rz[c] : 0.0;
    const int64_t o = (int64_t)c * n;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
      p[o + i] = fma(beta, p[o + i], z[o + i]);
  }
}

__global__ void k_copy_scalars(double* __restrict__ dst, const double* __restrict__ src, int n) {
  if (threadIdx.x < n) dst[threadIdx.x] = src[threadIdx.x];
}

}  // namespace

void launch_combine_full(const int64_t* rowptr, const int* col, const double* Cval, const double* Bval,
                         const uint8_t* bound, int n, double mult, double* Aval, cudaStream_t s) {
  const int64_t threads = (int64_t)n * 32;
  k_combine_full<<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(rowptr, col, Cval, Bval, bound, n, mult, Aval);
}

void launch_spmv(const int64_t* rowptr, const int* col, const double* Aval, const double* x, int n, int npls,
                 double* y, cudaStream_t s) {
  const int64_t threads = (int64_t)n * 32;
  k_spmv<<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(rowptr, col, Aval, x, n, npls, y);
}

void launch_dots(const double* a, const double* b, int n, int npls, double* work, double* out, cudaStream_t s) {
  k_dot_partial<<<kDotBlocks, 256, 0, s>>>(a, b, n, npls, work);
  k_dot_final<<<npls, 256, 0, s>>>(work, npls, out);
}

void launch_pcg_step(const double* rz, const double* pq, double* x, double* r, const double* p, const double* q,
                     int n, int npls, double* work, double* rr, cudaStream_t s) {
  k_pcg_step<<<kDotBlocks, 256, 0, s>>>(rz, pq, x, r, p, q, n, npls, work);
  k_dot_final<<<npls, 256, 0, s>>>(work, npls, rr);
}

void launch_pcg_dir(double* rz, const double* rz_new, const double* z, double* p, int n, int npls, cudaStream_t s) {
  k_pcg_dir<<<kDotBlocks, 256, 0, s>>>(rz, rz_new, z, p, n, npls);
  k_copy_scalars<<<1, 64, 0, s>>>(rz, rz_new, npls);
}

void launch_assemble(const ElemDev& e, const int* elems, int nelems, const int64_t* rowptr,
                     const int* col, double* Cval, double* Bval, cudaStream_t s) {
  if (nelems <= 0) return;
  const int64_t work = (int64_t)nelems * 144;
  k_assemble<<<(unsigned)((work + 255) / 256), 256, 0, s>>>(e, elems, nelems, rowptr, col, Cval, Bval);
}

void launch_combine(const double* Cval, const double* Bval, const int64_t* src, const uint8_t* diag,
                    int64_t nnz, double mult, double* out, cudaStream_t s) {
  if (nnz <= 0) return;
  const unsigned g = (unsigned)std::min<int64_t>((nnz + 255) / 256, 148 * 64);
  k_combine<<<g, 256, 0, s>>>(Cval, Bval, src, diag, nnz, mult, out);
}

void launch_history_rhs(const int64_t* rowptr, const int* col, const double* Cval, const double* u1,
                        const double* u2, double m1c, double m2c, const double* S, double coef,
                        const uint8_t* bound, int n, int npls, double* rhs, cudaStream_t s) {
  if (npls > 1) {
    const int64_t threads = (int64_t)n * 32;
    k_history_rhs_multi<<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(rowptr, col, Cval, u1, u2, m1c, m2c, S,
                                                                          coef, bound, n, npls, rhs);
  } else {
    const int64_t threads = (int64_t)n * kRhsLanes;
    k_history_rhs<<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(rowptr, col, Cval, u1, u2, m1c, m2c, S, coef,
                                                                    bound, n, npls, rhs);
  }
}

void launch_normal_field(const float* f, const int* idx, const double* len, int nanom, int n, int npls, double* En,
                         cudaStream_t s) {
  const int64_t t = (int64_t)nanom * npls;
  if (t <= 0) return;
  k_normal_field<<<(unsigned)((t + 255) / 256), 256, 0, s>>>(f, idx, len, nanom, n, npls, En);
}

void launch_anomaly_rhs(const int64_t* rowptr, const int* col, const double* Cds, const double* En,
                        const uint8_t* bound, int n, int npls, double* rhs, cudaStream_t s) {
  const int64_t threads = (int64_t)n * 32;
  k_anomaly_rhs<<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(rowptr, col, Cds, En, bound, n, npls, rhs);
}

void launch_receivers(const int64_t* rowptr, const int* col, const double* val, const int* src,
                      int nrows, const double* u, int64_t ld, double* out, cudaStream_t s) {
  if (nrows <= 0) return;
  const int64_t threads = (int64_t)nrows * 32;
  k_receivers<<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(rowptr, col, val, src, nrows, u, ld, out);
}

void launch_time_diff(const double* series, int nt, int nser, int t0, const double* time,
                      const int* vpre1, const int* vpre2, int scheme, double sign, double* out,
                      cudaStream_t s) {
  if (nser <= 0 || nt < 3) return;
  k_time_diff<<<(nser + 127) / 128, 128, 0, s>>>(series, nt, nser, t0, time, vpre1, vpre2, scheme, sign, out);
}

}  // namespace tdem
