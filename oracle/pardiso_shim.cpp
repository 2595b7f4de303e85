// pardiso_64 stand-in for building the reference from source -- TEST INFRASTRUCTURE ONLY.
//
// The reference solves every sparse SPD system through MKL's C-ABI entry
// pardiso_64 (CalcNonstat3DLine/pardiso.cpp:69-126: mtype = 2, iparm all zero,
// phase 12 = analysis + numeric factorization of an upper-triangular 1-based
// CSR matrix, phase 33 = solve for nrhs column-major right-hand sides,
// phase -1 = release).  MKL is not installed here, so this file exports a
// pardiso_64 with those semantics backed by oracle::SparseCholesky, letting the
// unmodified reference link on Linux.  Only the phases and arguments the
// reference uses are supported; anything else sets error = -1.
//
// The handle lives in pt[0].  When the environment variable TDEM_ORACLE_COORDS
// is set and the matrix size equals the edge count in tsize3d_.dat (or the node
// count in xyz.dat), vertex coordinates read from the working directory steer
// the nested-dissection ordering; otherwise a graph ordering is used.  The
// analysis is reused while the sparsity pattern is unchanged.  TDEM_ORACLE_THREADS
// sets the thread count (default: all cores).
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "cpu_cholesky.h"

namespace {
struct Handle {
  oracle::SparseCholesky chol;
  bool analyzed = false;
};

std::vector<double> load_coords(int64_t n) {
  std::vector<double> out;
  if (!getenv("TDEM_ORACLE_COORDS")) return out;
  FILE* f = fopen("xyz.dat", "rb");
  if (!f) return out;
  fseek(f, 0, SEEK_END);
  long bytes = ftell(f);
  fseek(f, 0, SEEK_SET);
  std::vector<double> xyz(bytes / 8);
  size_t got = fread(xyz.data(), 8, xyz.size(), f);
  fclose(f);
  if (got != xyz.size()) return out;
  const int64_t nodes = (int64_t)xyz.size() / 3;
  if (n == nodes) return xyz;
  std::ifstream ts("tsize3d_.dat");
  int64_t dummy = 0, nedges = -1;
  if (!(ts >> dummy >> nedges) || nedges != n) return out;
  FILE* fe = fopen("nodesforedges.dat", "rb");
  if (!fe) return out;
  std::vector<int32_t> nfe(2 * n);
  got = fread(nfe.data(), 4, nfe.size(), fe);
  fclose(fe);
  if ((int64_t)got != 2 * n) return out;
  out.resize(3 * n);
  for (int64_t e = 0; e < n; ++e) {
    const int64_t a = nfe[2 * e] - 1, b = nfe[2 * e + 1] - 1;
    if (a < 0 || b < 0 || a >= nodes || b >= nodes) return {};
    for (int k = 0; k < 3; ++k) out[3 * e + k] = 0.5 * (xyz[3 * a + k] + xyz[3 * b + k]);
  }
  return out;
}

int thread_count() {
  if (const char* t = getenv("TDEM_ORACLE_THREADS")) return std::max(1, atoi(t));
  unsigned h = std::thread::hardware_concurrency();
  return h ? (int)h : 1;
}
}  // namespace

namespace {
// Optional per-call wall-clock log (TDEM_ORACLE_TIMING=<file>): one line
// "phase n nrhs t_begin t_end" in seconds since the first call, used to split a
// reference run into set-up, factorization and per-step time.
double now_rel() {
  static const auto t0 = std::chrono::steady_clock::now();
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}
struct CallLog {
  long long phase, n, nrhs;
  double t0;
  ~CallLog() {
    if (const char* f = getenv("TDEM_ORACLE_TIMING")) {
      if (FILE* fp = fopen(f, "a")) {
        fprintf(fp, "%lld %lld %lld %.6f %.6f\n", phase, n, nrhs, t0, now_rel());
        fclose(fp);
      }
    }
  }
};
}  // namespace

extern "C" void pardiso_64(void* pt, const int64_t* /*maxfct*/, const int64_t* /*mnum*/,
                           const int64_t* mtype, const int64_t* phase, const int64_t* n,
                           const void* a, const int64_t* ia, const int64_t* ja, int64_t* /*perm*/,
                           const int64_t* nrhs, int64_t* /*iparm*/, const int64_t* /*msglvl*/,
                           void* b, void* x, int64_t* error) {
  CallLog log_{*phase, *n, nrhs ? *nrhs : 0, now_rel()};
  void** ptv = (void**)pt;
  Handle* h = (Handle*)ptv[0];
  *error = 0;
  if (*phase == -1) {
    delete h;
    ptv[0] = nullptr;
    return;
  }
  if (*mtype != 2) { *error = -1; return; }
  if (*phase == 12 || *phase == 11 || *phase == 22) {
    if (!h) { h = new Handle(); ptv[0] = h; }
    const int64_t nn = *n;
    // 1-based upper CSR -> 0-based
    std::vector<int64_t> ptr(nn + 1), ind(ia[nn] - 1);
    for (int64_t i = 0; i <= nn; ++i) ptr[i] = ia[i] - 1;
    for (int64_t q = 0; q < (int64_t)ind.size(); ++q) ind[q] = ja[q] - 1;
    if (*phase != 22) {
      // re-analyse only when the pattern changed
      oracle::SparseCholesky probe;
      bool same = false;
      if (h->analyzed && h->chol.n == nn && h->chol.nnz_a == ptr[nn]) {
        uint64_t hh = 1469598103934665603ull ^ (uint64_t)nn;
        for (int64_t i = 0; i <= nn; ++i) hh = (hh ^ (uint64_t)ptr[i]) * 1099511628211ull;
        for (int64_t q = 0; q < ptr[nn]; ++q) hh = (hh ^ (uint64_t)ind[q]) * 1099511628211ull;
        same = ((int64_t)hh == h->chol.pattern_hash);
      }
      if (!same) {
        std::vector<double> xyz = load_coords(nn);
        h->chol = oracle::SparseCholesky();
        if (h->chol.analyze((int)nn, ptr.data(), ind.data(), xyz.empty() ? nullptr : xyz.data(),
                            thread_count()) != 0) {
          *error = -1;
          return;
        }
        h->analyzed = true;
      }
    }
    if (*phase == 12 || *phase == 22) {
      int e = h->chol.factor((const double*)a);
      if (e) *error = -4;  // zero / negative pivot
    }
    return;
  }
  if (*phase == 33) {
    if (!h || !h->analyzed) { *error = -1; return; }
    h->chol.solve((int)*nrhs, (const double*)b, (double*)x);
    return;
  }
  *error = -1;
}

extern "C" void mkl_set_num_threads(int) {}
