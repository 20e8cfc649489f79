// Test infrastructure (oracle), not product code.
//
// Driver linked against the reference's own front-end sources
// (code/src/commons/{NFALoader,NFA,node,vasim_helper,nfa_utils,...}.cpp and
// pugixml), compiled by oracle/Makefile into oracle/_ref/ref_frontend. It runs
// the same sequence as the reference CLI (code/src/ngap/main.cu:57-79 and
// ngap::preprocessing, code/src/ngap/ngap.cu:63-91) and writes the resulting
// group graphs the way Graph::ReadNFA reads them (code/src/commons/graph.cu:
// 169-206), so that the product's preprocessing and the Python restatement can
// be checked id-for-id against the reference itself.
//
// usage: ref_frontend <file.anml> <group_num> <out.txt> [max_nfa_size]
#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <vector>

#include "NFA.h"
#include "NFALoader.h"
#include "nfa_utils.h"
#include "node.h"

int main(int argc, char** argv) {
  if (argc < 4) {
    fprintf(stderr, "usage: %s <file.anml> <group_num> <out.txt> [max_nfa_size]\n", argv[0]);
    return 2;
  }
  int group_num = atoi(argv[2]);
  int max_size = argc > 4 ? atoi(argv[4]) : -1;
  NFA* nfa = load_nfa_from_file(argv[1]);
  nfa->mark_cc_id();
  std::vector<NFA*> ccs = nfa_utils::split_nfa_by_ccs(*nfa);
  for (auto cc : ccs) {
    cc->calc_scc();
    cc->topo_sort();
  }
  int total_ccs = (int)ccs.size();
  auto res = nfa_utils::limit_out_degree_on_ccs(ccs, 4, true, false);
  if (max_size != -1) {
    std::vector<NFA*> tmp;
    for (auto cc : ccs)
      if (cc->size() <= max_size) tmp.push_back(cc);
    ccs = tmp;
  }
  auto groups = nfa_utils::group_nfas_by_num(group_num, ccs);
  FILE* f = fopen(argv[3], "w");
  if (!f) return 3;
  fprintf(f, "NGAPREF 1\n");
  fprintf(f, "groups %d ccs_total %d ccs_failed %d\n", (int)groups.size(), total_ccs, res.second);
  for (size_t g = 0; g < groups.size(); g++) {
    NFA* gn = groups[g];
    int V = gn->size();
    std::vector<std::pair<int, int>> edges;
    std::vector<int> aas, starts;
    fprintf(f, "group %d V %d\n", (int)g, V);
    for (int i = 0; i < V; i++) {
      Node* n = gn->get_node_by_int_id(i);
      unsigned w[8] = {0};
      for (int s = 0; s < 256; s++)
        if (n->symbol_set.test(s)) w[s / 32] |= 1u << (s % 32);
      int attrs = 0;
      if (n->is_start_always_enabled()) {
        attrs |= 1;
        aas.push_back(i);
      }
      if (n->is_start() && !n->is_start_always_enabled()) starts.push_back(i);
      if (n->is_report()) attrs |= 2;
      fprintf(f, "n %d", i);
      for (int k = 0; k < 8; k++) fprintf(f, " %08x", w[k]);
      fprintf(f, " %d %s\n", attrs, n->str_id.c_str());
      for (auto& to : gn->adj[n->str_id]) edges.emplace_back(i, gn->get_node_by_str_id(to)->sid);
    }
    std::sort(edges.begin(), edges.end());
    for (auto& e : edges) fprintf(f, "e %d %d\n", e.first, e.second);
    fprintf(f, "aas");
    for (int a : aas) fprintf(f, " %d", a);
    fprintf(f, "\nstart");
    for (int s : starts) fprintf(f, " %d", s);
    fprintf(f, "\n");
  }
  fclose(f);
  return 0;
}
