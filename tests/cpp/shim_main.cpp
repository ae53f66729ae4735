// Drop-in check of include/vine/cspp.hpp: the reference's call sequence
// (main.cu:61-81) against the 3-vertex known-answer graph.
#include <cstdio>
#include <vector>

#include "vine/cspp.hpp"

int main() {
  Graph<c_edge> g;
  g.from_arcs(3, {0, 1, 0}, {1, 2, 2}, {5, 7, 20}, {2, 3, 1});
  g.adj_to_csr();
  if (g.make_gpu_graph() != 0) {
    std::printf("graph: %s\n", vine_last_error());
    return 2;
  }
  std::vector<c_label> src{c_label(0), c_label(0), c_label(0)};
  std::vector<int> sinks{2, 2, 2};
  std::vector<c_constraint<c_label>> C{c_constraint<c_label>(100), c_constraint<c_label>(4),
                                       c_constraint<c_label>(0)};
  cspp<c_label, c_edge> solver(&g, 3, src, sinks, C);
  int rc = solver.solve();
  bool ok = rc == 0 && solver.found_l[0] && solver.cost_l[0] == 12 && solver.delay_l[0] == 5 &&
            solver.size_of_result_l[0] == 3 && solver.path_l[0][1] == 1 && solver.found_l[1] &&
            solver.cost_l[1] == 20 && solver.size_of_result_l[1] == 2 && !solver.found_l[2];
  std::printf("%s rc=%d costs %g %g found %d %d %d\n", ok ? "OK" : "FAIL", rc, solver.cost_l[0],
              solver.cost_l[1], solver.found_l[0], solver.found_l[1], solver.found_l[2]);
  return ok ? 0 : 1;
}
