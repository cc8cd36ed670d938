// Boomerang stage packer: turns a partition's logic cone into a sequence of
// 13-level boomerang stages (the 8192 -> 1 tree the kernel evaluates).
//
// The tree layout and its rules are the reference's (src/pe.rs:32-44,
// src/flatten.rs:984-1076): hier[l] has 8192 >> l slots; slot (l, j) reads
// (l-1, j) as input "a" and (l-1, j + len(l)) as input "b"; a slot either
// passes "a" through or is the AND gate whose fanins sit in those two slots;
// every slot at level >= 1 is visible to the next stage and to the writeout
// hooks, which capture whole 32-slot words.  The placement algorithm below is
// this project's own (the reference's greedy, src/pe.rs:70-660, recomputes
// reverse levels after every placement and is quadratic): per stage it
//   A. places critical-path trees top-down into free subtrees with exact
//      level-1 slot accounting and a duplication filter;
//   B. fills level 1 with the mandatory work: endpoints ready for writeout
//      (packed into as few 32-slot words as possible), height-1 gates, and
//      pass-throughs that carry live values to the next stage;
//   and backs off the tree budget until B fits.
#include "frontend.hpp"

#include <algorithm>
#include <numeric>

namespace jq {

namespace {

constexpr int L = BOOM_STAGES;
inline uint32_t lvl_len(int l) { return 8192u >> l; }

struct Cone {
  std::vector<uint32_t> pin;  // local -> global
  std::vector<int32_t> fa, fb;
  std::vector<uint8_t> leaf, tgt;
  std::vector<uint32_t> cs, cons;  // consumer CSR
};

// Reserved writeout words for SRAM groups and duplicate activations: the
// quantity checked by Partition::quick_reject (src/pe.rs:662-720) and used
// by the flattener (src/flatten.rs:535-540).
struct Reserve {
  uint32_t srams = 0, dups = 0;
};

Reserve count_reserved(const AIG &g, const StagedAIG &st,
                       const std::vector<uint32_t> &eps) {
  Reserve r;
  std::vector<std::pair<uint32_t, uint32_t>> acts;  // (pin, activation key)
  size_t nso = st.staged_outputs.size();
  size_t npo = g.primary_outputs.size(), nd = g.dffs.size();
  for (uint32_t e : eps) {
    if (e < nso) {
      acts.push_back({st.staged_outputs[e], 2});
      continue;
    }
    size_t o = st.endpoints[e - nso];
    if (o < npo) {
      uint32_t iv = g.primary_outputs[o];
      if (iv <= 1) continue;
      acts.push_back({iv >> 1, 2 | (iv & 1)});
    } else if (o < npo + nd) {
      const DFF &d = g.dffs[o - npo];
      if (d.d_iv <= 1) continue;
      acts.push_back({d.d_iv >> 1, d.en_iv << 1 | (d.d_iv & 1)});
    } else {
      r.srams++;
    }
  }
  std::sort(acts.begin(), acts.end());
  acts.erase(std::unique(acts.begin(), acts.end()), acts.end());
  for (size_t i = 1; i < acts.size(); ++i)
    if (acts[i].first == acts[i - 1].first) r.dups++;
  return r;
}

}  // namespace

bool build_partition(const AIG &g, const StagedAIG &st,
                     const std::vector<uint32_t> &endpoints, Partition &out,
                     const PackOptions &opt) {
  out.endpoints = endpoints;
  out.stages.clear();
  Reserve rv = count_reserved(g, st, endpoints);
  uint32_t reserved = rv.srams + (rv.dups + 31) / 32;
  if (reserved >= MAX_WRITEOUTS || rv.srams * 4 + rv.dups > MAX_WRITEOUTS) return false;
  const uint32_t wo_budget = MAX_WRITEOUTS - reserved;

  // ---------------- cone in topological order (leaves first by DFS postorder)
  std::vector<uint32_t> targets;
  for (uint32_t e : endpoints) st.for_each_input(g, e, [&](uint32_t p) { targets.push_back(p); });
  std::sort(targets.begin(), targets.end());
  targets.erase(std::unique(targets.begin(), targets.end()), targets.end());
  Cone C;
  std::unordered_map<uint32_t, int32_t> loc;
  loc.reserve(targets.size() * 8);
  {
    std::vector<std::pair<uint32_t, int>> stk;
    for (uint32_t t : targets) {
      if (loc.count(t)) continue;
      stk.push_back({t, 0});
      while (!stk.empty()) {
        auto [u, ph] = stk.back();
        stk.pop_back();
        if (ph == 1) {
          if (loc.count(u)) continue;
          int32_t id = (int32_t)C.pin.size();
          loc[u] = id;
          C.pin.push_back(u);
          bool lf = st.is_leaf(g, u);
          C.leaf.push_back(lf);
          C.tgt.push_back(0);
          if (lf) {
            C.fa.push_back(-1);
            C.fb.push_back(-1);
          } else {
            C.fa.push_back(loc.at(g.fa[u] >> 1));
            C.fb.push_back(loc.at(g.fb[u] >> 1));
          }
          continue;
        }
        if (loc.count(u)) continue;
        stk.push_back({u, 1});
        if (!st.is_leaf(g, u)) {
          uint32_t b = g.fb[u] >> 1, a = g.fa[u] >> 1;
          if (!loc.count(b)) stk.push_back({b, 0});
          if (!loc.count(a)) stk.push_back({a, 0});
        }
      }
    }
  }
  const int n = (int)C.pin.size();
  for (uint32_t t : targets) C.tgt[loc.at(t)] = 1;
  out.targets = (uint32_t)targets.size();
  out.cone_ands = 0;
  for (int i = 0; i < n; ++i) out.cone_ands += !C.leaf[i];
  {
    std::vector<uint32_t> deg(n + 1, 0);
    for (int i = 0; i < n; ++i)
      if (!C.leaf[i]) { deg[C.fa[i]]++; deg[C.fb[i]]++; }
    C.cs.assign(n + 1, 0);
    for (int i = 0; i < n; ++i) C.cs[i + 1] = C.cs[i] + deg[i];
    C.cons.assign(C.cs[n], 0);
    std::vector<uint32_t> fill(C.cs.begin(), C.cs.end() - 1);
    for (int i = 0; i < n; ++i)
      if (!C.leaf[i]) {
        C.cons[fill[C.fa[i]]++] = i;
        C.cons[fill[C.fb[i]]++] = i;
      }
  }

  // ---------------- stage loop state
  std::vector<uint8_t> done(n), in_input(n), pend(n);
  for (int i = 0; i < n; ++i) {
    done[i] = C.leaf[i];
    in_input[i] = C.leaf[i];
    pend[i] = C.tgt[i];
  }
  uint32_t total_wo = 0;
  std::vector<uint8_t> need(n), need2(n), done_now(n), vis(n), l1(n), inW(n);
  std::vector<int32_t> height(n), rlev(n);
  std::vector<uint32_t> c1(n);
  std::vector<uint8_t> used[L + 1], blocked[L + 1];
  std::vector<uint32_t> cursor(L + 1);
  std::vector<int32_t> mark(n, -1);
  int mark_gen = 0;

  for (int stage_i = 0;; ++stage_i) {
    bool any_pend = false;
    for (int i = 0; i < n; ++i) any_pend |= pend[i] != 0;
    if (!any_pend) break;
    if (stage_i >= opt.max_stages) return false;

    // need / height / rlev / c1 relative to this stage's inputs
    for (int i = n - 1; i >= 0; --i) {
      bool nd = pend[i];
      for (uint32_t k = C.cs[i]; k < C.cs[i + 1] && !nd; ++k) {
        int c = C.cons[k];
        if (!done[c] && need[c]) nd = true;
      }
      need[i] = nd;
      if (nd && done[i] && !in_input[i]) return false;  // lost a live value
    }
    for (int i = 0; i < n; ++i) {
      if (done[i] || !need[i]) { height[i] = 0; c1[i] = 1; continue; }
      int a = C.fa[i], b = C.fb[i];
      int ha = done[a] ? 0 : height[a], hb = done[b] ? 0 : height[b];
      height[i] = 1 + std::max(ha, hb);
      if (height[i] == 1) {
        c1[i] = 1;
      } else {
        // level-1 slots used when i sits at its own height h: each fanin is
        // either an input (pass-through chain: one level-1 slot) or an
        // uncomputed node whose own expansion starts at or below h-1.
        c1[i] = (done[a] ? 1 : c1[a]) + (done[b] ? 1 : c1[b]);
        if (c1[i] > 8192) c1[i] = 8192;
      }
    }
    for (int i = n - 1; i >= 0; --i) {
      if (done[i] || !need[i]) { rlev[i] = -1; continue; }
      int r = pend[i] ? 0 : -1;
      for (uint32_t k = C.cs[i]; k < C.cs[i + 1]; ++k) {
        int c = C.cons[k];
        if (!done[c] && need[c]) r = std::max(r, rlev[c] + 1);
      }
      rlev[i] = r;
    }
    std::vector<int32_t> cand;
    for (int i = 0; i < n; ++i)
      if (!done[i] && need[i] && height[i] >= 2 && height[i] <= L) cand.push_back(i);
    std::sort(cand.begin(), cand.end(), [&](int a, int b) {
      if (rlev[a] != rlev[b]) return rlev[a] > rlev[b];
      if (height[a] != height[b]) return height[a] > height[b];
      return a < b;
    });

    BoomStage S;
    bool built = false;
    // tree budget on level-1 slots; halved until phase B fits (none for
    // flat stages)
    int budget = opt.flat ? 0 : 4096;
    for (int attempt = 0; attempt < 8 && !built; ++attempt) {
      for (int l = 0; l <= L; ++l) {
        S.hier[l].assign(lvl_len(l), NONE);
        used[l].assign(lvl_len(l), 0);
        blocked[l].assign(lvl_len(l), 0);
        cursor[l] = 0;
      }
      S.write_outs.clear();
      std::fill(done_now.begin(), done_now.end(), 0);
      std::fill(vis.begin(), vis.end(), 0);
      uint32_t used1 = 0;

      // ---- phase A: trees
      std::vector<int32_t> dstk;
      auto place = [&](auto &&self, int x, int l, uint32_t j) -> void {
        S.hier[l][j] = C.pin[x];
        used[l][j] = 1;
        if (l == 0) return;
        vis[x] = 1;
        if (l == 1) used1++;
        if (done[x] || height[x] < l) {
          self(self, x, l - 1, j);
        } else {
          done_now[x] = 1;
          self(self, C.fa[x], l - 1, j);
          self(self, C.fb[x], l - 1, j + lvl_len(l));
        }
      };
      if (budget > 0) {
        for (int x : cand) {
          if (done_now[x]) continue;
          int h = height[x];
          if (used1 + c1[x] > (uint32_t)budget) continue;
          // duplication filter: distinct new gates this tree computes
          ++mark_gen;
          uint32_t distinct = 0;
          dstk.clear();
          dstk.push_back(x);
          while (!dstk.empty() && 4 * distinct + 8 < c1[x]) {
            int u = dstk.back();
            dstk.pop_back();
            if (done[u] || mark[u] == mark_gen) continue;
            mark[u] = mark_gen;
            if (!done_now[u]) distinct++;
            dstk.push_back(C.fa[u]);
            dstk.push_back(C.fb[u]);
          }
          if (distinct == 0 || c1[x] > 4 * distinct + 8) continue;
          // first free subtree at level h
          uint32_t &cur = cursor[h];
          while (cur < lvl_len(h) && (used[h][cur] || blocked[h][cur])) ++cur;
          if (cur >= lvl_len(h)) continue;
          uint32_t j = cur;
          place(place, x, h, j);
          // ancestors of the root now have a used descendant
          uint32_t jj = j;
          for (int l = h + 1; l <= L; ++l) {
            jj = jj % lvl_len(l);
            blocked[l][jj] = 1;
          }
        }
      }

      // ---- phase B: level-1 work
      for (int i = n - 1; i >= 0; --i) {
        if (done[i] || done_now[i]) { need2[i] = 0; continue; }
        bool nd = pend[i];
        for (uint32_t k = C.cs[i]; k < C.cs[i + 1] && !nd; ++k) {
          int c = C.cons[k];
          if (!done[c] && !done_now[c] && need2[c]) nd = true;
        }
        need2[i] = nd;
      }
      std::vector<int32_t> W, L1, carry;
      for (int i = 0; i < n; ++i) {
        l1[i] = (!done[i] && !done_now[i] && need2[i] && height[i] == 1);
        if (l1[i]) L1.push_back(i);
      }
      for (int i = 0; i < n; ++i) {
        inW[i] = pend[i] && (in_input[i] || l1[i]);
        if (inW[i]) W.push_back(i);
      }
      for (int i = 0; i < n; ++i) {
        if (!in_input[i] || vis[i] || inW[i]) continue;
        bool na = false;
        for (uint32_t k = C.cs[i]; k < C.cs[i + 1] && !na; ++k) {
          int c = C.cons[k];
          if (!done[c] && !done_now[c] && !l1[c] && need2[c]) na = true;
        }
        if (na) carry.push_back(i);
      }
      uint32_t free1 = 0;
      for (uint32_t j = 0; j < 4096; ++j) free1 += !used[1][j];
      size_t demand = W.size() + (L1.size() - std::count_if(L1.begin(), L1.end(), [&](int x) { return inW[x]; })) + carry.size();
      if (demand > free1) {
        budget = budget / 2;
        if (attempt >= 6) budget = 0;
        continue;
      }
      // writeout groups: fullest-free first
      std::vector<std::pair<int, int>> grp;  // (-free, g)
      for (int gi = 0; gi < 128; ++gi) {
        int f = 0;
        for (int k = 0; k < 32; ++k) f += !used[1][gi * 32 + k];
        if (f) grp.push_back({-f, gi});
      }
      std::sort(grp.begin(), grp.end());
      auto put1 = [&](int x, uint32_t j) {
        if (inW[x] && !l1[x]) {
          // pass-through of an input
          S.hier[1][j] = C.pin[x];
          S.hier[0][j] = C.pin[x];
          used[1][j] = used[0][j] = 1;
        } else if (l1[x]) {
          S.hier[1][j] = C.pin[x];
          S.hier[0][j] = C.pin[C.fa[x]];
          S.hier[0][j + 4096] = C.pin[C.fb[x]];
          used[1][j] = used[0][j] = used[0][j + 4096] = 1;
          done_now[x] = 1;
        } else {
          S.hier[1][j] = C.pin[x];
          S.hier[0][j] = C.pin[x];
          used[1][j] = used[0][j] = 1;
        }
        vis[x] = 1;
      };
      size_t wi = 0;
      std::vector<uint16_t> wos;
      for (auto &pg : grp) {
        if (wi >= W.size()) break;
        int gi = pg.second;
        bool any = false;
        for (int k = 0; k < 32 && wi < W.size(); ++k) {
          uint32_t j = gi * 32 + k;
          if (used[1][j]) continue;
          put1(W[wi++], j);
          any = true;
        }
        if (any) wos.push_back((uint16_t)(128 + gi));
      }
      uint32_t j1 = 0;
      auto next_free = [&]() {
        while (j1 < 4096 && used[1][j1]) ++j1;
        return j1;
      };
      bool ok = true;
      for (int x : L1) {
        if (inW[x]) continue;
        uint32_t j = next_free();
        if (j >= 4096) { ok = false; break; }
        put1(x, j);
      }
      for (int x : carry) {
        if (!ok) break;
        uint32_t j = next_free();
        if (j >= 4096) { ok = false; break; }
        put1(x, j);
      }
      if (!ok) {
        budget = budget / 2;
        if (attempt >= 6) budget = 0;
        continue;
      }
      // ---- final stage: write out tree-computed endpoints in place
      bool last = true;
      for (int i = 0; i < n && last; ++i)
        if (need2[i] && !done[i] && !done_now[i]) last = false;
      std::vector<int32_t> tree_tgts;
      for (int i = 0; i < n; ++i)
        if (pend[i] && !inW[i]) tree_tgts.push_back(i);
      std::vector<uint16_t> extra;
      if (last && !tree_tgts.empty()) {
        // greedy cover of the pending endpoints by visible 32-slot words
        std::unordered_map<uint32_t, int> tid;
        for (int x : tree_tgts) tid[C.pin[x]] = x;
        std::vector<std::vector<int>> word_t(256);
        for (int l = 1; l <= L; ++l)
          for (uint32_t j = 0; j < lvl_len(l); ++j) {
            uint32_t p = S.hier[l][j];
            if (p == NONE) continue;
            auto it = tid.find(p);
            if (it == tid.end()) continue;
            uint32_t pos = lvl_len(l) + j;
            word_t[pos >> 5].push_back(it->second);
          }
        std::vector<uint8_t> cov(n, 0);
        size_t left = tree_tgts.size();
        while (left) {
          int best = -1, bc = 0;
          for (int w = 0; w < 256; ++w) {
            int c = 0;
            for (int x : word_t[w]) c += !cov[x];
            if (c > bc) { bc = c; best = w; }
          }
          if (best < 0) break;
          extra.push_back((uint16_t)best);
          for (int x : word_t[best])
            if (!cov[x]) { cov[x] = 1; --left; }
        }
        if (left != 0 || total_wo + wos.size() + extra.size() > wo_budget) extra.clear();
        else
          for (int x : tree_tgts) inW[x] = 1;
      }
      for (uint16_t w : extra) wos.push_back(w);
      if (total_wo + wos.size() > wo_budget) return false;
      total_wo += (uint32_t)wos.size();
      S.write_outs = wos;
      built = true;
    }
    if (!built) return false;

    // stage-0 inputs must fit the global read (256 threads x 32 bits)
    if (stage_i == 0) {
      std::vector<uint32_t> ins;
      for (uint32_t p : S.hier[0])
        if (p != NONE) ins.push_back(p);
      std::sort(ins.begin(), ins.end());
      ins.erase(std::unique(ins.begin(), ins.end()), ins.end());
      if (ins.size() > 7168) return false;
    }
    // commit
    bool progress = false;
    for (int i = 0; i < n; ++i) {
      if (done_now[i] && !done[i]) { done[i] = 1; progress = true; }
      if (inW[i] && pend[i]) { pend[i] = 0; progress = true; }
      in_input[i] = vis[i];
    }
    out.stages.push_back(std::move(S));
    if (!progress) return false;
  }
  // A partition whose endpoints need no logic at all (constant-D DFFs,
  // constant outputs) has no stages; the flattener emits nothing for it.
  return true;
}

}  // namespace jq
