// Test driver (CPU): the library's element colouring for assembly on the model in
// argv[1]; checks that no two elements of one colour share an edge, that every
// element is listed once, ascending inside its colour, and that each element has
// the lowest colour its earlier neighbours leave free (the greedy rule).
#include "model.h"
#include <cstdio>
#include <set>
using namespace tdem;
int main(int argc, char** argv) {
  Model m;
  std::string e = load_model(argv[1], m);
  if (!e.empty()) { printf("load: %s\n", e.c_str()); return 1; }
  std::vector<int> order, cstart;
  if (!(e = element_colouring(m, order, cstart)).empty()) { printf("colour: %s\n", e.c_str()); return 1; }
  const int ncol = (int)cstart.size() - 1;
  if ((int)order.size() != m.n_elem || cstart[ncol] != m.n_elem) { printf("count\n"); return 1; }
  std::vector<int> color(m.n_elem, -1);
  for (int c = 0; c < ncol; ++c)
    for (int k = cstart[c]; k < cstart[c + 1]; ++k) {
      if (color[order[k]] != -1) { printf("twice\n"); return 1; }
      if (k > cstart[c] && order[k] <= order[k - 1]) { printf("not ascending\n"); return 1; }
      color[order[k]] = c;
    }
  std::vector<std::vector<int>> owner(m.n_edges);
  for (int el = 0; el < m.n_elem; ++el)
    for (int j = 0; j < 12; ++j) owner[m.ed[el][j]].push_back(el);
  for (int el = 0; el < m.n_elem; ++el) {
    std::set<int> taken;
    for (int j = 0; j < 12; ++j)
      for (int o : owner[m.ed[el][j]]) {
        if (o != el && color[o] == color[el]) { printf("conflict\n"); return 1; }
        if (o < el) taken.insert(color[o]);
      }
    int c = 0;
    while (taken.count(c)) ++c;
    if (c != color[el]) { printf("not greedy\n"); return 1; }
  }
  printf("ok %d colours\n", ncol);
  return 0;
}
