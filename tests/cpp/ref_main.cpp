// A caller written the way the reference's main.cu drives its query path
// (main.cu:17-83): a config file names the graph format, graph file, query
// file and task count; read_graph fills the adjacency model, adj_to_csr and
// an edge list build the CSR, make_gpu_graph uploads it, and cspp::solve runs
// the queries.  Only the includes differ from the reference's caller (this
// one header instead of comm.hpp / task.hpp / label.hpp / constraint.hpp).
// After solve() it prints one line per task: "task found cost delay nvertices
// v0 v1 ...", which the reference's caller had no way to print.
#include <stdio.h>
#include <iostream>
#include <vector>
#include <cuda_runtime.h>

#include "vine/cspp.hpp"

static Graph<c_edge> *g;

int pre_process_task(task *tasks, int N) {  // keep vertices in range (main.cu:19-26)
  for (int i = 0; i < tasks->ntask; i++) {
    tasks->source_l_[i] %= N;
    tasks->sink_l_[i] %= N;
  }
  return 0;
}

c_edge *create_edge_list(Graph<c_edge> *g) {  // per edge id weights (main.cu:28-36)
  c_edge *l = (c_edge *)malloc(sizeof(c_edge) * g->M);
  for (int i = 0; i < g->M; i++) {
    l[i].len = g->e_l[i]->len;
    l[i].delay = g->e_l[i]->delay;
  }
  return l;
}

int main(int argc, char *argv[]) {
  using Constraint = c_constraint<c_label>;
  using Graph = Graph<c_edge>;
  int graph_type, ntask;
  char graph_f[255], query_f[255];
  FILE *conf = fopen(argc > 1 ? argv[1] : "../inputs/config", "r");
  if (!conf || fscanf(conf, "%d", &graph_type) != 1 || fscanf(conf, "%254s", graph_f) != 1 ||
      fscanf(conf, "%254s", query_f) != 1 || fscanf(conf, "%d", &ntask) != 1) {
    printf("config unreadable\n");
    return 3;
  }
  fclose(conf);

  cudaSetDevice(0);
  g = new Graph();
  task *tasks = new task();
  if (read_graph(graph_f, g, graph_type) != 0) {
    printf("graph unreadable\n");
    return 3;
  }
  if (graph_type == 1) {
    tasks->read_query(query_f, 1);
    pre_process_task(tasks, g->N);
  } else {
    tasks->load_query(query_f);  // COLA query file
  }
  g->adj_to_csr();
  g->el = create_edge_list(g);
  if (g->make_gpu_graph() != 0) {
    printf("graph upload: %s\n", vine_last_error());
    return 2;
  }

  cspp<c_label, c_edge> *solver;
  std::vector<Constraint> C_l;
  std::vector<c_label> source_state_l;
  for (int i = 0; i < ntask; i++) {
    c_label l(tasks->source_l_[i]);
    source_state_l.push_back(l);
    Constraint c(tasks->delay_l_[i]);
    C_l.push_back(c);
  }
  cuda_err_chk(cudaGetLastError());
  std::cout << "Number of V " << g->N << std::endl;
  std::cout << "Number of E " << g->M << std::endl;
  solver = new cspp<c_label, c_edge>(g, ntask, source_state_l, tasks->sink_l_, C_l);
  cuda_err_chk(cudaGetLastError());
  int rc = solver->solve();
  cuda_err_chk(cudaGetLastError());
  std::cout << "solve " << rc << std::endl;
  for (int i = 0; i < ntask; i++) {
    printf("%d %d %.1f %.1f %d", i, solver->found_l[i], solver->cost_l[i], solver->delay_l[i],
           solver->size_of_result_l[i]);
    for (int k = 0; k < solver->size_of_result_l[i]; k++) printf(" %d", solver->path_l[i][k]);
    printf("\n");
  }
  delete solver;
  return rc == 0 ? 0 : 1;
}
