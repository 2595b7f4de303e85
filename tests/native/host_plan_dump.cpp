// Test driver (CPU): runs the host half of a solve (TransientSolve::plan, no device)
// on argv[1] with formulation argv[2] (0 = A, 1 = E) and writes what it built for the
// device, for the Python test to compare with the numpy oracle:
//   <argv[3]>.S    source vectors, n x npls doubles (column-major)
//   <argv[3]>.u0   initial field, n x npls doubles
//   <argv[3]>.rb / .re   receiver operators: int64 nrec, nrows, nnz; int64 rowptr[nrows + 1];
//                        int32 col[nnz]; double val[nnz]; int32 src[nrows]
// and prints "ok <n> <npls>".  With argv[1] = "--merged": host_plan_dump --merged <0|1>
// <out prefix> <dir>...  plans the directories as one merged run (plan_merged).
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "driver.h"
using namespace tdem;

static bool dump_vec(const std::string& fn, const std::vector<double>& v) {
  FILE* f = fopen(fn.c_str(), "wb");
  if (!f) return false;
  const bool ok = fwrite(v.data(), 8, v.size(), f) == v.size();
  return fclose(f) == 0 && ok;
}

static bool dump_op(const std::string& fn, const ReceiverOperator& r) {
  FILE* f = fopen(fn.c_str(), "wb");
  if (!f) return false;
  const int64_t head[3] = {r.nrec, (int64_t)r.rowptr.size() - 1, (int64_t)r.col.size()};
  bool ok = fwrite(head, 8, 3, f) == 3;
  ok = ok && fwrite(r.rowptr.data(), 8, r.rowptr.size(), f) == r.rowptr.size();
  ok = ok && fwrite(r.col.data(), 4, r.col.size(), f) == r.col.size();
  ok = ok && fwrite(r.val.data(), 8, r.val.size(), f) == r.val.size();
  ok = ok && fwrite(r.src.data(), 4, r.src.size(), f) == r.src.size();
  return fclose(f) == 0 && ok;
}

int main(int argc, char** argv) {
  const bool merged = argc > 1 && std::string(argv[1]) == "--merged";
  if (argc < (merged ? 5 : 4)) {
    printf("usage: host_plan_dump <dir> <0|1> <out prefix> | --merged <0|1> <out prefix> <dir>...\n");
    return 2;
  }
  // both forms hold <0|1> and <out prefix> in argv[2] and argv[3]
  TransientSolve ts;
  RunOptions opt;
  opt.scheme = 2;
  opt.formulation = std::atoi(argv[2]);
  const std::string out = argv[3];
  const std::string e = merged ? ts.plan_merged(std::vector<std::string>(argv + 4, argv + argc), opt)
                               : ts.plan(argv[1], opt);
  if (!e.empty()) {
    printf("plan: %s\n", e.c_str());
    return 1;
  }
  if (!dump_vec(out + ".S", ts.planned_sources()) || !dump_vec(out + ".u0", ts.planned_initial_field()) ||
      !dump_op(out + ".rb", ts.planned_receivers_b()) || !dump_op(out + ".re", ts.planned_receivers_e())) {
    printf("write failed\n");
    return 1;
  }
  printf("ok %d %d\n", ts.model().n_edges, ts.model().npls);
  return 0;
}
