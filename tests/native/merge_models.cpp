// Test driver (CPU): merging of model directories that differ only in sources and
// receivers (the serving loop's batched time steps).  argv[1..n-1]: directories of
// one mesh; argv[n]: a directory with another mesh.  Checks the merged model
// (sources and receivers in order, per-source receiver ranges shifted), the initial
// field read per directory, the host plan of the merged directories (TransientSolve
// ::plan_merged, no device) and the refusal of a different mesh; with --expect, the
// refusal of two directories with the given message.
#include <cstdio>
#include <string>
#include <vector>

#include "driver.h"
#include "model.h"
using namespace tdem;

// --expect <dir a> <dir b> <error>: merging a and b must fail with exactly <error>
static int expect(const char* a, const char* b, const char* want) {
  std::vector<Model> parts(2);
  std::string e;
  if (!(e = load_model(a, parts[0])).empty() || !(e = load_model(b, parts[1])).empty()) {
    printf("load: %s\n", e.c_str());
    return 1;
  }
  Model m;
  e = merge_models(parts, m);
  if (e != want) {
    printf("expected '%s', got '%s'\n", want, e.c_str());
    return 1;
  }
  printf("ok refused: %s\n", e.c_str());
  return 0;
}

int main(int argc, char** argv) {
  if (argc == 5 && std::string(argv[1]) == "--expect") return expect(argv[2], argv[3], argv[4]);
  if (argc < 4) { printf("usage\n"); return 2; }
  std::vector<std::string> dirs(argv + 1, argv + argc - 1);
  std::vector<Model> parts(dirs.size());
  for (size_t i = 0; i < dirs.size(); ++i) {
    std::string e = load_model(dirs[i], parts[i]);
    if (!e.empty()) { printf("load: %s\n", e.c_str()); return 1; }
  }
  Model m;
  std::string e = merge_models(parts, m);
  if (!e.empty()) { printf("merge: %s\n", e.c_str()); return 1; }
  int np = 0, nb = 0, ne = 0;
  for (size_t i = 0; i < parts.size(); ++i) {
    const Model& p = parts[i];
    for (int s = 0; s < p.npls; ++s) {
      if (m.wires[np + s] != p.wires[s]) { printf("wire order\n"); return 1; }
      if (m.rec_b_ig[np + s] != nb + p.rec_b_ig[s] || m.rec_b_ig[np + s + 1] != nb + p.rec_b_ig[s + 1] ||
          m.rec_e_ig[np + s] != ne + p.rec_e_ig[s] || m.rec_e_ig[np + s + 1] != ne + p.rec_e_ig[s + 1]) {
        printf("receiver ranges\n");
        return 1;
      }
    }
    for (size_t k = 0; k < p.rec_b.size(); ++k)
      if (m.rec_b[nb + k] != p.rec_b[k]) { printf("receiver order\n"); return 1; }
    // the part's initial field, read from its own directory on the merged mesh
    std::vector<double> u_own, u_merged;
    if (!(e = load_initial_field(p, true, u_own)).empty() ||
        !(e = load_initial_field(m, dirs[i], p.npls, true, u_merged)).empty()) {
      printf("initial field: %s\n", e.c_str());
      return 1;
    }
    if (u_own != u_merged) { printf("initial field differs\n"); return 1; }
    np += p.npls;
    nb += (int)p.rec_b.size();
    ne += (int)p.rec_e.size();
  }
  if (m.npls != np || (int)m.rec_b.size() != nb || (int)m.rec_e.size() != ne) { printf("counts\n"); return 1; }
  // host plan of the merged directories
  TransientSolve ts;
  RunOptions opt;
  opt.formulation = 0;
  opt.scheme = 3;
  std::vector<std::array<int, 3>> info;
  if (!(e = ts.plan_merged(dirs, opt, &info)).empty()) { printf("plan_merged: %s\n", e.c_str()); return 1; }
  if (info.size() != dirs.size() || ts.model().npls != np || ts.device_bytes_needed() <= 0) {
    printf("plan_merged result\n");
    return 1;
  }
  for (size_t i = 0; i < parts.size(); ++i)
    if (info[i][0] != parts[i].npls || info[i][1] != (int)parts[i].rec_b.size() ||
        info[i][2] != (int)parts[i].rec_e.size()) {
      printf("part info\n");
      return 1;
    }
  // another mesh is refused
  Model other, bad;
  if (!(e = load_model(argv[argc - 1], other)).empty()) { printf("load: %s\n", e.c_str()); return 1; }
  std::vector<Model> mixed{parts[0], other};
  e = merge_models(mixed, bad);
  if (e != "the meshes differ") { printf("mismatch not found: '%s'\n", e.c_str()); return 1; }
  printf("ok %d sources\n", np);
  return 0;
}
