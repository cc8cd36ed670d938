// Seeded synthetic gate-level designs in the aigpdk cell set, built directly as
// an AIG.  Stands in for the reference's benchmark netlists, which are not
// available: the shapes follow the synthetic configurations the benchmark is
// quoted on (levelized random AND logic, DFFs whose D pins are chosen nodes,
// optional clustered locality, single-port SRAM macros, a reset input).
//
// Semantics of the sequential cells follow the reference's AIG construction:
//   * a plain DFF has en_iv = the clock's posedge flag (src/aig.rs:2028-2060);
//   * a synchronous reset gates D with the inverted reset input;
//   * SRAM macros use the `$__RAMGEM_SYNC_` port set (src/aig.rs:95-108) with
//     the upper address bits tied to 0 for macros narrower than 8192 words.
#include "aig.hpp"
#include "frontend.hpp"

#include <algorithm>
#include <stdexcept>

namespace jq {

namespace {
struct SplitMix64 {
  uint64_t s;
  explicit SplitMix64(uint64_t seed) : s(seed) {}
  uint64_t next() {
    uint64_t z = (s += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
  }
  uint32_t below(uint32_t n) { return (uint32_t)((next() >> 11) % n); }
  double unit() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
};
}  // namespace

AIG generate_design(const GenParams &p, GenInfo *info) {
  if (p.n_clusters == 0 || p.nodes_per_cluster == 0 || p.depth == 0)
    throw std::invalid_argument("empty design");
  SplitMix64 rng(p.seed * 0x2545F4914F6CDD1Dull + 0x1234567ull);
  AIG g;
  const uint32_t C = p.n_clusters;

  // ---- level-0 sources: clock flag, primary inputs, DFF Q, SRAM read bits
  uint32_t clk = g.add_pin(DRV_CLKFLAG, 0);
  std::vector<uint32_t> pis;
  for (uint32_t i = 0; i < p.n_pi; ++i) pis.push_back(g.add_pin(DRV_INPUT, i));
  uint32_t rst = 0;
  if (p.with_reset) {
    if (p.n_pi == 0) throw std::invalid_argument("reset needs an input");
    rst = pis[0];
  }
  std::vector<std::vector<uint32_t>> pool(C);  // per-cluster level-0 pins
  std::vector<uint32_t> dff_cluster(p.n_dff);
  g.dffs.resize(p.n_dff);
  for (uint32_t i = 0; i < p.n_dff; ++i) {
    uint32_t c = (uint32_t)((uint64_t)i * C / std::max(1u, p.n_dff));
    dff_cluster[i] = c;
    g.dffs[i].q = g.add_pin(DRV_DFF, i);
    pool[c].push_back(g.dffs[i].q);
  }
  g.srams.resize(p.n_sram);
  std::vector<uint32_t> sram_cluster(p.n_sram);
  for (uint32_t s = 0; s < p.n_sram; ++s) {
    uint32_t c = (uint32_t)((uint64_t)s * C / std::max(1u, p.n_sram));
    sram_cluster[s] = c;
    for (int k = 0; k < 32; ++k) {
      g.srams[s].r_data[k] = g.add_pin(DRV_SRAM, s);
      pool[c].push_back(g.srams[s].r_data[k]);
    }
  }
  for (uint32_t c = 0; c < C; ++c)
    for (uint32_t pi : pis)
      if (!p.with_reset || pi != rst) pool[c].push_back(pi);
  for (uint32_t c = 0; c < C; ++c)
    if (pool[c].empty()) pool[c].push_back(clk);

  // ---- levelized AND logic, allocated level-major so pins stay topological
  // levels[c][L] = AND pins of cluster c at level L (L >= 1)
  std::vector<std::vector<std::vector<uint32_t>>> levels(
      C, std::vector<std::vector<uint32_t>>(p.depth + 1));
  auto pick_source = [&](uint32_t c, uint32_t L) -> uint32_t {
    uint32_t cc = c;
    if (C > 1 && rng.unit() >= p.intra_frac) {
      cc = rng.below(C - 1);
      if (cc >= c) ++cc;
    }
    uint32_t lo = L > p.fanin_window ? L - p.fanin_window : 0;
    for (int tries = 0; tries < 64; ++tries) {
      uint32_t lv = lo + rng.below(L - lo);
      const std::vector<uint32_t> &v = lv == 0 ? pool[cc] : levels[cc][lv];
      if (!v.empty()) return v[rng.below((uint32_t)v.size())];
    }
    return pool[cc][rng.below((uint32_t)pool[cc].size())];
  };
  uint64_t made = 0;
  for (uint32_t L = 1; L <= p.depth; ++L) {
    for (uint32_t c = 0; c < C; ++c) {
      // spread nodes_per_cluster over depth levels as evenly as possible
      uint32_t n_here = (uint32_t)(((uint64_t)p.nodes_per_cluster * L) / p.depth -
                                   ((uint64_t)p.nodes_per_cluster * (L - 1)) / p.depth);
      auto &out = levels[c][L];
      out.reserve(n_here);
      uint32_t guard = 0;
      while (out.size() < n_here && guard < n_here * 64 + 64) {
        ++guard;
        // the first fanin comes from the previous level so that the level is
        // exact; the second from the fan-in window
        uint32_t a = (L == 1) ? pick_source(c, 1) : [&] {
          if (C > 1 && rng.unit() >= p.intra_frac) {
            uint32_t cc = rng.below(C - 1);
            if (cc >= c) ++cc;
            const auto &v = levels[cc][L - 1];
            if (!v.empty()) return v[rng.below((uint32_t)v.size())];
          }
          const auto &v = levels[c][L - 1];
          if (!v.empty()) return v[rng.below((uint32_t)v.size())];
          return pick_source(c, L);
        }();
        uint32_t b = pick_source(c, L);
        if (a == b) continue;
        uint32_t aiv = a << 1 | (uint32_t)(rng.next() & 1);
        uint32_t biv = b << 1 | (uint32_t)(rng.next() & 1);
        uint32_t before = g.num_pins;
        uint32_t r = g.add_and(aiv, biv);
        if (g.num_pins == before) continue;  // structural duplicate: resample
        out.push_back(r >> 1);
        ++made;
      }
    }
  }

  // ---- DFF data / enable
  uint32_t rst_n = rst ? (rst << 1 | 1) : 1;
  for (uint32_t i = 0; i < p.n_dff; ++i) {
    uint32_t c = dff_cluster[i];
    uint32_t L = 1 + rng.below(p.depth);
    uint32_t src;
    const auto &v = levels[c][L];
    src = v.empty() ? pick_source(c, p.depth) : v[rng.below((uint32_t)v.size())];
    uint32_t d_iv = src << 1 | (uint32_t)(rng.next() & 1);
    if (p.with_reset) d_iv = g.add_and(d_iv, rst_n);
    g.dffs[i].d_iv = d_iv;
    g.dffs[i].en_iv = clk << 1;
  }
  // ---- SRAM ports: one shared read/write address (single port), write
  // enable replicated over the 32 bit-enables, random data nets.
  auto rand_net = [&](uint32_t c) -> uint32_t {
    uint32_t L = 1 + rng.below(p.depth);
    const auto &v = levels[c][L];
    uint32_t n = v.empty() ? pick_source(c, p.depth) : v[rng.below((uint32_t)v.size())];
    return n << 1 | (uint32_t)(rng.next() & 1);
  };
  for (uint32_t s = 0; s < p.n_sram; ++s) {
    RAMBlock &r = g.srams[s];
    uint32_t c = sram_cluster[s];
    for (int k = 0; k < SRAM_ADDR_BITS; ++k) {
      uint32_t a = (k < (int)p.sram_addr_bits) ? rand_net(c) : 0;
      r.r_addr_iv[k] = a;
      r.w_addr_iv[k] = a;
    }
    r.r_en_iv = clk << 1;
    uint32_t we = g.add_and(rand_net(c), clk << 1);
    for (int k = 0; k < 32; ++k) {
      r.w_en_iv[k] = we;
      r.w_data_iv[k] = rand_net(c);
    }
  }
  // ---- primary outputs: distinct nodes
  std::unordered_map<uint32_t, int> seen;
  uint32_t guard = 0;
  while (g.primary_outputs.size() < p.n_po && guard < p.n_po * 64 + 64) {
    ++guard;
    uint32_t c = rng.below(C);
    uint32_t iv = rand_net(c);
    if (seen.count(iv >> 1)) continue;
    seen[iv >> 1] = 1;
    g.primary_outputs.push_back(iv);
  }
  if (info) {
    info->num_and = 0;
    for (uint32_t q = 1; q <= g.num_pins; ++q) info->num_and += g.kind[q] == DRV_AND;
    info->clock_flag_pin = clk;
    info->reset_pin = rst;
  }
  (void)made;
  return g;
}

std::vector<uint8_t> AIG::x_capable_pins(int *iterations) const {
  // src/aig.rs:3277-3366: DFF Q and SRAM read bits are X sources; forward cone
  // through AND gates in pin (topological) order; DFF fixpoint.
  std::vector<uint8_t> x(num_pins + 1, 0);
  for (const DFF &d : dffs) x[d.q] = 1;
  for (const RAMBlock &r : srams)
    for (int k = 0; k < 32; ++k)
      if (r.r_data[k] != NONE && r.r_data[k] != 0) x[r.r_data[k]] = 1;
  int it = 0;
  for (;;) {
    for (uint32_t p = 1; p <= num_pins; ++p) {
      if (x[p] || kind[p] != DRV_AND) continue;
      if (x[fa[p] >> 1] || x[fb[p] >> 1]) x[p] = 1;
    }
    bool changed = false;
    for (const DFF &d : dffs) {
      if (x[d.d_iv >> 1] && !x[d.q]) {
        x[d.q] = 1;
        changed = true;
      }
    }
    ++it;
    if (!changed) break;
  }
  if (iterations) *iterations = it;
  return x;
}

}  // namespace jq
