// Test driver (CPU): the library's host routine for the E-formulation's
// primary-secondary source values, for the steps given on the command line
// (it t1 t2 three_point ...), written as doubles to argv[2].
#include "model.h"
#include <cstdio>
#include <cstdlib>
using namespace tdem;
int main(int argc, char** argv) {
  Model m;
  std::string e = load_model(argv[1], m);
  if (!e.empty()) { printf("load: %s\n", e.c_str()); return 1; }
  NormalField nf;
  e = init_normal_field(m, true, nf);
  if (!e.empty()) { printf("init: %s\n", e.c_str()); return 1; }
  FILE* out = fopen(argv[2], "wb");
  for (int a = 3; a + 3 < argc + 1; a += 4) {
    int it = atoi(argv[a]), t1 = atoi(argv[a + 1]), t2 = atoi(argv[a + 2]), three = atoi(argv[a + 3]);
    std::vector<double> v;
    e = normal_field_rate(m, nf, it, t1, t2, three != 0, v);
    if (!e.empty()) { printf("rate: %s\n", e.c_str()); return 1; }
    fwrite(v.data(), 8, v.size(), out);
  }
  fclose(out);
  printf("ok n=%d npls=%d nanom=%zu\n", m.n_edges, m.npls, nf.idx.size());
}
