// Host-only check of the drop-in graph model (no device work): reads a graph
// with read_graph, builds the CSR with adj_to_csr and prints it as
// "N M" then the row pointers, then one "head len delay eid" line per slot.
#include <cstdio>

#include "vine/cspp.hpp"

int main(int argc, char **argv) {
  if (argc < 3) return 3;
  Graph<c_edge> g;
  if (read_graph(argv[1], &g, atoi(argv[2])) != 0) return 2;
  if (g.adj_to_csr() != 0) return 2;
  printf("%d %d\n", g.N, g.M);
  for (int i = 0; i <= g.N; ++i) printf("%d\n", g._count_row[i]);
  for (int j = 0; j < g.M; ++j)
    printf("%d %.1f %.1f %d\n", g._vid_col[j], g._len[j], g._delay[j], g._eid_col[j]);
  return 0;
}
