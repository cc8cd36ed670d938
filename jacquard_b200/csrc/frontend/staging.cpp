// Major-stage splitting at global logic levels (restates the algorithm of
// src/staging.rs:93-236: a slice keeps the endpoints whose logic level is at
// most the split; nodes at or below the split that still feed logic above it
// become staged IO pins, written to the state by this slice and read back by
// the next one through the "current cycle" global read).
#include "frontend.hpp"

#include <algorithm>

namespace jq {

// Iterative DFS topological order of the cone of `roots`, stopping at staged
// inputs (src/aig.rs:3125-3179).
static void topo_cone(const AIG &g, const std::vector<uint32_t> &roots,
                      const std::vector<uint8_t> *stop, std::vector<uint32_t> &order,
                      std::vector<uint32_t> &mark, uint32_t gen) {
  std::vector<uint32_t> stk;
  stk.reserve(1024);
  for (uint32_t r : roots) {
    if (mark[r] == gen) continue;
    stk.push_back(r << 1);
    while (!stk.empty()) {
      uint32_t it = stk.back();
      stk.pop_back();
      uint32_t u = it >> 1;
      if (it & 1) {
        order.push_back(u);
        continue;
      }
      if (mark[u] == gen) continue;
      mark[u] = gen;
      stk.push_back(u << 1 | 1);
      if (g.kind[u] == DRV_AND && !(stop && (*stop)[u])) {
        uint32_t b = g.fb[u] >> 1, a = g.fa[u] >> 1;
        if (b && mark[b] != gen) stk.push_back(b << 1);
        if (a && mark[a] != gen) stk.push_back(a << 1);
      }
    }
  }
}

static StagedAIG from_split(const AIG &g, const std::vector<uint32_t> &unrealized,
                            const std::vector<uint8_t> &pi, bool has_pi,
                            uint64_t split) {
  std::vector<uint32_t> roots;
  for (uint32_t e : unrealized) g.for_each_endpoint_input(e, [&](uint32_t p) { roots.push_back(p); });
  std::vector<uint32_t> mark(g.num_pins + 1, 0), order;
  topo_cone(g, roots, has_pi ? &pi : nullptr, order, mark, 1);
  std::vector<uint32_t> fanouts(g.num_pins + 1, 0);
  std::vector<uint32_t> level(g.num_pins + 1, 0);
  for (uint32_t i : order) {
    if (has_pi && pi[i]) continue;
    if (g.kind[i] == DRV_AND) {
      uint32_t a = g.fa[i] >> 1, b = g.fb[i] >> 1;
      if (a) { fanouts[a]++; level[i] = std::max(level[i], level[a] + 1); }
      if (b) { fanouts[b]++; level[i] = std::max(level[i], level[b] + 1); }
    }
  }
  std::vector<uint32_t> ep_level(unrealized.size(), 0);
  for (size_t k = 0; k < unrealized.size(); ++k)
    g.for_each_endpoint_input(unrealized[k], [&](uint32_t p) {
      fanouts[p]++;
      ep_level[k] = std::max(ep_level[k], level[p]);
    });
  std::vector<uint8_t> at_split(g.num_pins + 1, 0);
  for (uint32_t i : order) {
    if (level[i] > split) continue;
    at_split[i] = 1;
    if (has_pi && pi[i]) continue;
    if (g.kind[i] == DRV_AND) {
      uint32_t a = g.fa[i] >> 1, b = g.fb[i] >> 1;
      if (a && --fanouts[a] == 0) at_split[a] = 0;
      if (b && --fanouts[b] == 0) at_split[b] = 0;
    }
  }
  StagedAIG st;
  st.has_staged_inputs = has_pi;
  if (has_pi) st.is_staged_input = pi;
  for (size_t k = 0; k < unrealized.size(); ++k) {
    if (ep_level[k] > split) continue;
    st.endpoints.push_back(unrealized[k]);
    g.for_each_endpoint_input(unrealized[k], [&](uint32_t p) {
      if (--fanouts[p] == 0) at_split[p] = 0;
    });
  }
  for (uint32_t i : order)
    if (at_split[i] && !(has_pi && pi[i])) st.staged_outputs.push_back(i);
  return st;
}

std::vector<StagedAIG> build_staged_aigs(const AIG &g,
                                         const std::vector<uint32_t> &level_split) {
  std::vector<StagedAIG> ret;
  std::vector<uint32_t> unrealized(g.num_endpoint_groups());
  for (size_t i = 0; i < unrealized.size(); ++i) unrealized[i] = (uint32_t)i;
  std::vector<uint8_t> pi(g.num_pins + 1, 0);
  bool has_pi = false;
  uint32_t last = 0;
  for (uint32_t cur : level_split) {
    if (cur <= last) continue;
    StagedAIG st = from_split(g, unrealized, pi, has_pi, cur - last);
    std::vector<uint8_t> done(g.num_endpoint_groups(), 0);
    for (uint32_t e : st.endpoints) done[e] = 1;
    std::vector<uint32_t> rest;
    for (uint32_t e : unrealized)
      if (!done[e]) rest.push_back(e);
    unrealized.swap(rest);
    for (uint32_t p : st.staged_outputs) pi[p] = 1;
    has_pi = true;
    bool finished = st.staged_outputs.empty();
    ret.push_back(std::move(st));
    last = cur;
    if (finished) return ret;
  }
  ret.push_back(from_split(g, unrealized, pi, has_pi, UINT64_MAX));
  return ret;
}

}  // namespace jq
