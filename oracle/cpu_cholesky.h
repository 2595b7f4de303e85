// CPU FP64 sparse Cholesky used by the oracle -- TEST INFRASTRUCTURE ONLY.
//
// Nothing in the product links this file.  It serves two purposes:
//   * the direct solver of the CPU restatement of the transient solve
//     (oracle/tdem_oracle.cpp), and
//   * the solver behind the pardiso_64 shim (oracle/pardiso_shim.cpp) that lets
//     the reference's own CalcNonstat3DLine / CalcStat3D_3T_A be compiled from
//     source on Linux.  The reference calls MKL PARDISO with mtype = 2 (real SPD)
//     and phases 12 / 33 / -1 (CalcNonstat3DLine/pardiso.cpp:69-126); MKL is not
//     available, so this is a restatement of a generic supernodal multifrontal
//     Cholesky, not of PARDISO's internals.
//
// Method: nested-dissection ordering (coordinate bisection with one-sided vertex
// separators when vertex coordinates are known, breadth-first level-set
// bisection otherwise), the dissection tree used as the assembly tree (one front
// per leaf block / separator), dense partial Cholesky of each front, FP64
// throughout.  Dense kernels come from the OpenBLAS bundled with numpy when its
// path is given in TDEM_ORACLE_BLAS (dlopen), else from plain loops.
#pragma once
#include <cstdint>
#include <vector>

namespace oracle {

struct Front {
  int c0 = 0, c1 = 0;          // pivot columns [c0, c1) in permuted numbering
  std::vector<int> rows;       // rows below the pivot block (permuted, sorted, >= c1)
  int parent = -1;
  std::vector<int> children;
  std::vector<int> rel;        // positions of `rows` inside the parent front
  int64_t lofs = 0;            // offset of this front's (m x k) column block in L
  // original entries: value index, local row, local col (local row >= local col)
  std::vector<int64_t> a_idx;
  std::vector<int> a_r, a_c;
  int m() const { return (c1 - c0) + (int)rows.size(); }
  int k() const { return c1 - c0; }
};

class SparseCholesky {
 public:
  // Pattern of a symmetric matrix given by its upper triangle in CSR form with
  // 0-based indices (row i holds columns j >= i, diagonal included).  coords
  // (n x 3, optional) are vertex positions for the geometric ordering.
  int analyze(int n, const int64_t* ptr, const int64_t* ind, const double* coords,
              int nthreads);
  // Numeric factorization; val follows the analyzed pattern.  Returns 0 or the
  // 1-based permuted column at which a non-positive pivot appeared.
  int factor(const double* val);
  // x = A^-1 b for nrhs column-major right-hand sides of length n.
  void solve(int nrhs, const double* b, double* x) const;

  int n = 0;
  int nthreads = 1;
  int64_t nnz_l = 0;        // stored entries of L (dense front blocks)
  double flops = 0.0;       // factorization flops (multiply-add = 2)
  std::vector<int> perm;    // perm[old] = new
  std::vector<int> iperm;   // iperm[new] = old
  std::vector<Front> fronts;  // postorder: children before parents
  std::vector<double> L;
  int64_t pattern_hash = 0;
  int64_t nnz_a = 0;

 private:
  std::vector<std::vector<int>> subtrees_;  // independent subtrees (postorder lists)
  std::vector<int> top_;                    // fronts above the subtrees (postorder)
  void build_schedule();
};

// Loads dense kernels from TDEM_ORACLE_BLAS if set (idempotent).
bool blas_available();

}  // namespace oracle
