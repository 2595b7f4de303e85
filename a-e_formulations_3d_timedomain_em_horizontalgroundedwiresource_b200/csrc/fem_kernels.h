// FEM kernels of the transient solve: element assembly, system combine, history
// right-hand side, receiver evaluation and time differencing.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace tdem {

// Element data for assembly (device arrays).
struct ElemDev {
  const int* ed;        // 12 edge ids per element
  const double* h;      // hx, hy, hz per element
  const double* sigma;  // conductivity per element
  const double* inv_mu; // 1 / mu per element
};

// Adds sigma * C_e and B_e / mu of the elements in `elems` (one colour: no two
// share an edge) into the full symmetric CSR values Cval / Bval (Bval may be null:
// mass term only).
void launch_assemble(const ElemDev& e, const int* elems, int nelems, const int64_t* rowptr,
                     const int* col, double* Cval, double* Bval, cudaStream_t s);

// A = mult * C + B on the analysed lower-triangle entries of the interior system;
// diagonal entries are scaled by (1 + 1e-12) as the reference does
// (CalcNonstat3DLine/time_approx.cpp:987-994).  src[q] is the full-CSR index of
// entry q, diag[q] != 0 marks diagonal entries.
void launch_combine(const double* Cval, const double* Bval, const int64_t* src, const uint8_t* diag,
                    int64_t nnz, double mult, double* out, cudaStream_t s);

// History right-hand side for npls columns (column-major, leading dimension n):
//   rhs = C * (m1 * u1 + m2 * u2) + coef * S, zero on Dirichlet rows
// (CalcNonstat3DLine/time_approx.cpp:1018-1081).
void launch_history_rhs(const int64_t* rowptr, const int* col, const double* Cval, const double* u1,
                        const double* u2, double m1, double m2, const double* S, double coef,
                        const uint8_t* bound, int n, int npls, double* rhs, cudaStream_t s);

// Receiver values: out[row] = sum_j R[row, j] * u[j, src[row]] for every operator row.
// Primary-secondary source of one time layer.  The normal field f (float, V/m,
// nanom values per source, source-major) of the anomalous edges idx becomes edge
// degrees of freedom En = f * len * 0.5 (the other entries of En stay as they are,
// zero); then rhs += C_dsigma * En on the rows that are not Dirichlet edges.
void launch_normal_field(const float* f, const int* idx, const double* len, int nanom, int n, int npls, double* En,
                         cudaStream_t s);
void launch_anomaly_rhs(const int64_t* rowptr, const int* col, const double* Cds, const double* En,
                        const uint8_t* bound, int n, int npls, double* rhs, cudaStream_t s);

void launch_receivers(const int64_t* rowptr, const int* col, const double* val, const int* src,
                      int nrows, const double* u, int64_t ld, double* out, cudaStream_t s);

// A = mult * C + B on every entry of the full CSR, with the diagonal scaled by
// (1 + 1e-12); rows and columns of Dirichlet edges are left out (their values
// are set to 0), so A restricted to the interior equals the factorized matrix.
void launch_combine_full(const int64_t* rowptr, const int* col, const double* Cval, const double* Bval,
                         const uint8_t* bound, int n, double mult, double* Aval, cudaStream_t s);

// y = A x for npls columns (leading dimension n).
void launch_spmv(const int64_t* rowptr, const int* col, const double* Aval, const double* x, int n, int npls,
                 double* y, cudaStream_t s);

// Per-column dot products out[p] = sum_i a[i,p] b[i,p] (deterministic two-pass
// reduction; `work` holds kDotBlocks * npls doubles).
constexpr int kDotBlocks = 296;
void launch_dots(const double* a, const double* b, int n, int npls, double* work, double* out, cudaStream_t s);

// Preconditioned-CG vector updates with per-column scalars held on the device:
//   pcg_step:  alpha = rz / pq;  x += alpha p;  r -= alpha q;  rr = r . r
//   pcg_dir:   beta = rz_new / rz;  p = z + beta p;  rz = rz_new
void launch_pcg_step(const double* rz, const double* pq, double* x, double* r, const double* p, const double* q,
                     int n, int npls, double* work, double* rr, cudaStream_t s);
void launch_pcg_dir(double* rz, const double* rz_new, const double* z, double* p, int n, int npls, cudaStream_t s);

// Time differencing of receiver series (CalcNonstat3DLine/give_out_vec_loop.cpp:240-615,
// 3-point variant CalcNonstat3DLine (3-point)/give_out_vec_loop.cpp).  series is
// nt x nser (time-major); vpre1 / vpre2 give the earlier layers used at each layer
// (absolute layer numbers); t0 is the first layer of the series.  scheme 2 uses
// two-point interior differences, scheme 3 three-point ones.  out = sign * d/dt.
void launch_time_diff(const double* series, int nt, int nser, int t0, const double* time,
                      const int* vpre1, const int* vpre2, int scheme, double sign, double* out,
                      cudaStream_t s);

}  // namespace tdem
