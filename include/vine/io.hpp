// vine/io.hpp -- the reference's graph / query readers and error macro, for
// callers of vine/cspp.hpp (included from there).
//
//   read_graph(file, g, graph_type)   include/io.hpp:22-93
//   task::read_query / load_query     include/task.hpp:27-76
//   cuda_err_chk(expr)                include/util.hpp:14-20
//
// Same file formats and the same effect on the Graph's members (v_l, e_l, N,
// M) as the reference's readers, written here so that a reference caller
// needs no header of the reference.  Differences: the type-1 reader numbers
// edges from 0 (the reference's counter was never initialised), a missing or
// malformed file returns VINE_ERR_IO instead of crashing or exit(0), and
// '%' comment lines before the header are skipped.
#ifndef VINE_IO_HPP_
#define VINE_IO_HPP_

#include <cstdio>
#include <tuple>
#include <vector>

#include "../vine.h"

// graph_type 1: "n<sep>m<sep>" then m rows "src snk weight delay", each
//   added in both directions (edge ids 2i and 2i+1);
// graph_type 2 (COLA road graphs): "N" then lines "u: v w c v w c ... -1".
template <class Graph_t>
int read_graph(const char *file_name, Graph_t *g, int graph_type) {
  using myVertex = typename Graph_t::MyV;
  FILE *f = std::fopen(file_name, "r");
  if (!f) return VINE_ERR_IO;
  int c = std::fgetc(f);
  while (c == '%') {  // comment lines
    while (c != '\n' && c != EOF) c = std::fgetc(f);
    c = std::fgetc(f);
  }
  if (c != EOF) std::ungetc(c, f);
  int n = 0;
  if (std::fscanf(f, "%d", &n) != 1 || n < 1) {
    std::fclose(f);
    return VINE_ERR_IO;
  }
  g->v_l.clear();
  g->v_l.reserve(n);
  g->N = n;
  g->e_l.clear();
  for (int i = 0; i < n; i++) g->v_l.push_back(myVertex(i));
  if (graph_type == 1) {
    char sep;
    int m = 0;
    if (std::fscanf(f, "%c", &sep) != 1 || std::fscanf(f, "%d", &m) != 1 || m < 0) {
      std::fclose(f);
      return VINE_ERR_IO;
    }
    if (std::fscanf(f, "%c", &sep) < 0) sep = '\n';  // separator after m (may be absent)
    g->e_l.reserve((size_t)2 * m);
    int src, snk, w, d, id = 0;
    while (std::fscanf(f, "%d", &src) == 1) {
      if (std::fscanf(f, "%d %d %d", &snk, &w, &d) != 3 || src < 0 || src >= n || snk < 0 ||
          snk >= n) {
        std::fclose(f);
        return VINE_ERR_IO;
      }
      g->e_l.push_back(new Edge(id));
      g->e_l.back()->assign(id, src, snk, (float)w, (float)d);
      g->v_l[src].assign(g->e_l[id], g);
      ++id;
      g->e_l.push_back(new Edge(id));
      g->e_l.back()->assign(id, snk, src, (float)w, (float)d);
      g->v_l[snk].assign(g->e_l[id], g);
      ++id;
    }
  } else {
    int u, v, w, cc, m = 0;
    while (std::fscanf(f, "%d:", &u) == 1) {
      if (u < 0 || u >= n) {
        std::fclose(f);
        return VINE_ERR_IO;
      }
      while (std::fscanf(f, "%d", &v) == 1) {
        if (v == -1) break;
        if (std::fscanf(f, "%d %d", &w, &cc) != 2 || v < 0 || v >= n) {
          std::fclose(f);
          return VINE_ERR_IO;
        }
        g->e_l.push_back(new Edge(m));
        g->e_l.back()->assign(m, u, v, (float)w, (float)cc);
        g->v_l[u].assign(g->e_l[m++], g);
      }
    }
  }
  g->M = (int)g->e_l.size();
  std::fclose(f);
  return 0;
}

// Query lists (include/task.hpp:10-77).
class task {
 public:
  int ntask = 0;
  std::vector<int> source_l_;
  std::vector<int> sink_l_;
  std::vector<int> delay_l_;
  std::vector<int> hop_l_;
  std::vector<int> cost_l_;

  task() {}
  task(int n) : ntask(n) {}

  // graph_type 1: a header line, then rows "id,src,snk,delay,hop,cost";
  // otherwise rows "u v cost_lower cost_upper cost_limit" (budget = cost_limit).
  int read_query(const char *file_name, int graph_type) {
    FILE *f = std::fopen(file_name, "r");
    if (!f) return VINE_ERR_IO;
    if (graph_type == 1) {
      char line[4096];
      if (!std::fgets(line, sizeof(line), f)) {
        std::fclose(f);
        return VINE_ERR_IO;
      }
      int id, src, snk, delay, hop, cost;
      while (std::fscanf(f, "%d ,%d ,%d ,%d ,%d ,%d", &id, &src, &snk, &delay, &hop, &cost) == 6) {
        source_l_.push_back(src);
        sink_l_.push_back(snk);
        delay_l_.push_back(delay);
        hop_l_.push_back(hop);
        cost_l_.push_back(cost);
      }
    } else {
      read_cola(f);
    }
    std::fclose(f);
    ntask = (int)source_l_.size();
    return 0;
  }

  // COLA query files (include/task.hpp:61-76).
  int load_query(const char *file_name) {
    FILE *f = std::fopen(file_name, "r");
    if (!f) return VINE_ERR_IO;
    read_cola(f);
    std::fclose(f);
    ntask = (int)source_l_.size();
    return 0;
  }

 private:
  void read_cola(FILE *f) {
    int u, v, lo, hi, limit;
    while (std::fscanf(f, "%d %d %d %d %d\n", &u, &v, &lo, &hi, &limit) == 5) {
      source_l_.push_back(u);
      sink_l_.push_back(v);
      delay_l_.push_back(limit);
    }
  }
};

// Prints a CUDA error and carries on, as the reference's macro does.
#ifndef cuda_err_chk
template <typename Code>
inline void vine_err_chk(Code code, const char *file, int line) {
  if ((int)code != 0) std::fprintf(stderr, "GPUassert: error %d %s %d\n", (int)code, file, line);
}
#define cuda_err_chk(ans) \
  { vine_err_chk((ans), __FILE__, __LINE__); }
#endif

#endif  // VINE_IO_HPP_
