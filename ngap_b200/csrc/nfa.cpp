// NFA preprocessing that fixes report ids.
//
// Reference steps reproduced (all in code/src/commons/ unless noted):
//   NFA.cpp:188-227          mark_cc_id: CCs of the undirected graph, numbered
//                            in order of their lowest node id;
//   nfa_utils.cpp:54-91      split_nfa_by_ccs: CC-local ids in global id order;
//   nfa_utils.cpp:507-635    limit_out_degree_on_nfa: repeatedly pick, among
//                            nodes with out-degree > limit scanned from the
//                            highest id down, the first with the smallest
//                            out-degree (get_indegree_of_node returns the
//                            out-degree, NFA.cpp:518-521), delete it and
//                            re-add it as clones "_dup_p" of <= limit
//                            successors each (clone 0 keeps the id, the others
//                            are appended), self-loops kept on every clone;
//                            give up after 2*|CC| iterations;
//   nfa_utils.cpp:637-680    limit_out_degree_on_ccs: failed CCs are dropped;
//   code/src/ngap/ngap.cu:77-91  max_nfa_size filter;
//   nfa_utils.cpp:382-424    group_nfas_by_num: contiguous CC ranges, bound
//                            arithmetic in float;
//   nfa_utils.cpp:466-486    merge_nfas: group ids = concatenation order.
// Nodes are handled by integer handles instead of string ids; adjacency and
// predecessor lists keep the reference's insertion order, which decides which
// successors each clone receives.
#include "nfa.h"

#include <algorithm>
#include <climits>

namespace ngap {

namespace {

struct CcGraph {
  std::vector<int> attr;                   // handle -> ANML node index
  std::vector<std::vector<int>> adj, from;  // handle -> ordered handle lists
  std::vector<int> by_int;                 // integer id -> handle
  int V = 0;

  int new_handle(int a) {
    attr.push_back(a);
    adj.emplace_back();
    from.emplace_back();
    return (int)attr.size() - 1;
  }
  int add_node(int a) {  // NFA::addNode(n): id = V++
    int h = new_handle(a);
    by_int.push_back(h);
    V++;
    return h;
  }
  void add_edge(int f, int t) {  // NFA::addEdge, deduplicated
    auto& a = adj[f];
    if (std::find(a.begin(), a.end(), t) == a.end()) a.push_back(t);
    auto& b = from[t];
    if (std::find(b.begin(), b.end(), f) == b.end()) b.push_back(f);
  }
};

void erase_first(std::vector<int>& v, int x) {
  auto it = std::find(v.begin(), v.end(), x);
  if (it != v.end()) v.erase(it);
}

bool limit_out_degree(CcGraph& cc, int limit) {
  const int orig_size = cc.V;
  int iteration = 0;
  while (true) {
    iteration++;
    int pick = -1, pick_int = -1;
    size_t min_deg = SIZE_MAX;
    for (int i = cc.V - 1; i >= 0; i--) {
      int h = cc.by_int[i];
      size_t d = cc.adj[h].size();
      if (d > (size_t)limit && d < min_deg) {
        min_deg = d;
        pick = h;
        pick_int = i;
      }
    }
    if (pick < 0) break;

    std::vector<int> from_nodes = cc.from[pick];
    std::vector<int> to_nodes = cc.adj[pick];
    // NFA::remove_node_unsafe (NFA.cpp:542-591)
    {
      std::vector<int> fr = cc.from[pick];
      for (int fn : fr) erase_first(cc.adj[fn], pick);
      std::vector<int> to = cc.adj[pick];
      for (int t : to) erase_first(cc.from[t], pick);
      cc.adj[pick].clear();
      cc.from[pick].clear();
    }
    bool self_loop = std::find(to_nodes.begin(), to_nodes.end(), pick) != to_nodes.end();
    if (self_loop) {
      erase_first(to_nodes, pick);
      erase_first(from_nodes, pick);
    }
    int p = 0;
    size_t t = 0;
    while (t < to_nodes.size()) {
      int h;
      if (p == 0) {
        h = cc.new_handle(cc.attr[pick]);
        cc.by_int[pick_int] = h;
      } else {
        h = cc.add_node(cc.attr[pick]);
      }
      int L = limit;
      if (self_loop) {
        L = limit - 1;
        cc.add_edge(h, h);
      }
      for (int kk = 0; kk < L && t + kk < to_nodes.size(); kk++) cc.add_edge(h, to_nodes[t + kk]);
      for (int f : from_nodes) cc.add_edge(f, h);
      p++;
      t += L;
    }
    if (iteration >= orig_size * 2) return false;
  }
  return true;
}

}  // namespace

int build_groups(const AnmlNfa& nfa, const GroupOpts& opts, GroupSet& out) {
  out = GroupSet();
  const int V = (int)nfa.nodes.size();
  if (V == 0) {
    set_error("the NFA has no states");
    return NGAP_E_INVALID;
  }
  if (opts.group_num <= 0) {
    set_error("group_num must be positive (got %d)", opts.group_num);
    return NGAP_E_INVALID;
  }
  // --- connected components (undirected), numbered by lowest member id.
  std::vector<std::vector<int>> und(V);
  for (int i = 0; i < V; i++)
    for (int t : nfa.adj[i]) {
      und[i].push_back(t);
      und[t].push_back(i);
    }
  std::vector<int> cc_of(V, -1);
  int num_cc = 0;
  std::vector<int> stack;
  for (int i = 0; i < V; i++) {
    if (cc_of[i] >= 0) continue;
    cc_of[i] = num_cc;
    stack.push_back(i);
    while (!stack.empty()) {
      int x = stack.back();
      stack.pop_back();
      for (int y : und[x])
        if (cc_of[y] < 0) {
          cc_of[y] = num_cc;
          stack.push_back(y);
        }
    }
    num_cc++;
  }
  out.num_ccs_total = num_cc;
  // --- split into CCs; local id = rank by global id.
  std::vector<CcGraph> ccs(num_cc);
  std::vector<int> local(V);
  for (int i = 0; i < V; i++) local[i] = ccs[cc_of[i]].add_node(i);
  for (int i = 0; i < V; i++) {
    CcGraph& cc = ccs[cc_of[i]];
    for (int t : nfa.adj[i]) cc.add_edge(local[i], local[t]);
  }
  // --- out-degree limiting; failed CCs are dropped.
  std::vector<int> kept;
  for (int c = 0; c < num_cc; c++) {
    if (limit_out_degree(ccs[c], opts.degree_limit)) {
      kept.push_back(c);
    } else {
      out.num_ccs_failed++;
      if (opts.remove_degree && opts.quit_degree) {
        set_error("CC %d cannot be limited to out-degree %d (quit when degree > %d)", c,
                  opts.degree_limit, opts.degree_limit);
        return NGAP_E_DEGREE;
      }
    }
  }
  if (opts.max_nfa_size != -1) {
    std::vector<int> k2;
    for (int c : kept) {
      if (ccs[c].V <= opts.max_nfa_size) k2.push_back(c);
      else out.num_ccs_too_big++;
    }
    kept.swap(k2);
  }
  const int cc_num = (int)kept.size();
  if (cc_num == 0) {
    set_error("no connected component is left after degree limiting and size filtering");
    return NGAP_E_INVALID;
  }
  // --- contiguous grouping (float bound arithmetic as in the reference).
  int group_num = opts.group_num;
  if (group_num > cc_num) group_num = cc_num;
  std::vector<std::vector<int>> members;
  {
    float per_group = 1.0f * (float)cc_num / (float)group_num;
    float bound = per_group;
    std::vector<int> cur;
    for (int i = 0; i < cc_num; i++) {
      if (!cur.empty() && (float)(i + 1) > bound && (int)members.size() + 1 < group_num) {
        bound += per_group;
        members.push_back(cur);
        cur.clear();
      }
      cur.push_back(kept[i]);
    }
    if (!cur.empty()) members.push_back(cur);
  }
  out.group_num = (int)members.size();
  // --- merge each group: ids in CC order, then CC-local id order.
  for (auto& mem : members) {
    GroupGraph g;
    int total = 0;
    for (int c : mem) total += ccs[c].V;
    g.V = total;
    g.bits.assign((size_t)total * 8, 0);
    g.attrs.assign(total, 0);
    g.orig_node.resize(total);
    std::vector<std::pair<int32_t, int32_t>> edges;
    int base = 0;
    for (int c : mem) {
      CcGraph& cc = ccs[c];
      g.cc_begin.push_back(base);
      std::vector<int> gid(cc.attr.size(), -1);
      for (int i = 0; i < cc.V; i++) gid[cc.by_int[i]] = base + i;
      for (int i = 0; i < cc.V; i++) {
        int h = cc.by_int[i];
        int s = base + i;
        const AnmlNode& nd = nfa.nodes[cc.attr[h]];
        g.orig_node[s] = cc.attr[h];
        for (int w = 0; w < 8; w++) g.bits[(size_t)s * 8 + w] = nd.symbols.w[w];
        if (nd.start == kStartAllInput) {
          g.attrs[s] |= 1;
          g.aas.push_back(s);
        }
        if (nd.start == kStartOfData) g.starts.push_back(s);
        if (nd.report) g.attrs[s] |= 2;
        for (int t : cc.adj[h]) edges.emplace_back(s, gid[t]);
      }
      base += cc.V;
    }
    g.cc_begin.push_back(base);
    std::sort(edges.begin(), edges.end());
    g.E = (int32_t)edges.size();
    g.cols.resize(edges.size());
    g.row_offsets.assign((size_t)g.V + 1, 0);
    for (size_t e = 0; e < edges.size(); e++) {
      g.cols[e] = edges[e].second;
      g.row_offsets[edges[e].first + 1]++;
    }
    for (int v = 0; v < g.V; v++) g.row_offsets[v + 1] += g.row_offsets[v];
    out.groups.push_back(std::move(g));
  }
  return NGAP_OK;
}

}  // namespace ngap
