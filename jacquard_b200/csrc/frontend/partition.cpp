// Endpoint partitioner for one major stage.
//
// The reference partitions endpoints with a RepCut hypergraph handed to
// mt-kahypar (src/repcut.rs:58-272, src/sim/setup.rs:520-601), then merges
// partitions greedily (src/pe.rs:855-1070).  mt-kahypar is a third-party
// library that is not available here, so this file implements its own
// locality partitioner with the same contract -- every endpoint lands in
// exactly one partition whose logic fits the boomerang resources:
//   1. endpoints are ordered by a breadth-first walk over "shares a shallow
//      cone gate" adjacency, so endpoints computed from the same logic sit
//      next to each other;
//   2. the order is cut into chunks bounded by cone size and endpoint count;
//   3. each chunk is packed; a chunk that does not fit is split in half and
//      retried (the reference's halving loop, src/sim/setup.rs:540-580);
//   4. neighbouring small partitions are merged when the merged one still
//      packs without more stages (src/pe.rs:855-1070's acceptance rule).
// Balanced mode (target_parts) replaces step 2 with the smallest cone bound
// that cuts the stage into at most target_parts chunks, packs flat stages,
// and, given a cost model, refines the cut (step 3b) before merging within
// the bound.
#include "frontend.hpp"

#include <algorithm>
#include <cmath>
#include <atomic>
#include <deque>
#include <stdexcept>
#include <thread>

namespace jq {

namespace {

template <class F>
void parallel_for(size_t n, int threads, F &&f) {
  if (threads <= 1 || n <= 1) {
    for (size_t i = 0; i < n; ++i) f(i);
    return;
  }
  std::atomic<size_t> next{0};
  std::vector<std::thread> th;
  for (int t = 0; t < threads; ++t)
    th.emplace_back([&] {
      for (;;) {
        size_t i = next.fetch_add(1);
        if (i >= n) break;
        f(i);
      }
    });
  for (auto &t : th) t.join();
}

}  // namespace

std::vector<Partition> partition_stage(const AIG &g, const StagedAIG &st,
                                       const PartitionOptions &opt) {
  const size_t ne = st.num_endpoint_groups();
  int threads = opt.num_threads > 0 ? opt.num_threads
                                     : (int)std::max(1u, std::thread::hardware_concurrency());
  std::vector<Partition> result;
  if (ne == 0) return result;

  // ---- 1. shallow cone gates per endpoint (depth <= 4, at most 24 gates)
  const int DEPTH = 4;
  const size_t CAP = 24;
  std::vector<std::vector<uint32_t>> shallow(ne);
  parallel_for(ne, threads, [&](size_t e) {
    std::vector<std::pair<uint32_t, int>> q;
    st.for_each_input(g, e, [&](uint32_t p) {
      if (!st.is_leaf(g, p)) q.push_back({p, 0});
    });
    auto &out = shallow[e];
    for (size_t h = 0; h < q.size() && out.size() < CAP; ++h) {
      auto [u, d] = q[h];
      if (std::find(out.begin(), out.end(), u) != out.end()) continue;
      out.push_back(u);
      if (d + 1 >= DEPTH) continue;
      uint32_t a = g.fa[u] >> 1, b = g.fb[u] >> 1;
      if (!st.is_leaf(g, a)) q.push_back({a, d + 1});
      if (!st.is_leaf(g, b)) q.push_back({b, d + 1});
    }
  });
  // inverted index gate -> endpoints (skip gates shared too widely)
  std::unordered_map<uint32_t, std::vector<uint32_t>> inv;
  inv.reserve(ne * 8);
  for (size_t e = 0; e < ne; ++e)
    for (uint32_t u : shallow[e]) {
      auto &v = inv[u];
      if (v.size() < 64) v.push_back((uint32_t)e);
    }
  // ---- BFS order
  std::vector<uint32_t> order;
  order.reserve(ne);
  std::vector<uint8_t> seen(ne, 0);
  std::deque<uint32_t> dq;
  for (size_t s0 = 0; s0 < ne; ++s0) {
    if (seen[s0]) continue;
    seen[s0] = 1;
    dq.push_back((uint32_t)s0);
    while (!dq.empty()) {
      uint32_t e = dq.front();
      dq.pop_front();
      order.push_back(e);
      for (uint32_t u : shallow[e]) {
        auto it = inv.find(u);
        if (it == inv.end()) continue;
        for (uint32_t f : it->second)
          if (!seen[f]) { seen[f] = 1; dq.push_back(f); }
      }
    }
  }

  PackOptions po;
  po.flat = opt.target_parts != 0;  // balanced mode targets the batched kernel
  uint64_t cone_bound = 0;  // balanced mode: the largest chunk cost allowed
  // Steps 2 and 3 for a balanced-cut cost of cone ANDs + SRAM weight +
  // input_w16 / 16 per distinct chunk input (the global read of the batched
  // kernel loads one slot per input; 0 outside balanced mode).
  auto cut_and_pack = [&](uint64_t input_w16) {
  std::vector<std::vector<uint32_t>> chunks;
  // ---- 2. chunking by cone size / endpoint bits
  {
    std::vector<uint32_t> mark(g.num_pins + 1, 0);
    uint32_t gen = 1;
    std::vector<uint32_t> stk;
    // AND gates of endpoint e's cone not yet marked `gen` (marks them);
    // `leaves` receives the cone's inputs (stage inputs: staged signals,
    // DFF / SRAM outputs, primary inputs) not yet marked
    uint64_t leaves = 0;
    auto grow = [&](uint32_t e) {
      uint64_t add = 0;
      leaves = 0;
      stk.clear();
      st.for_each_input(g, e, [&](uint32_t p) { stk.push_back(p); });
      while (!stk.empty()) {
        uint32_t u = stk.back();
        stk.pop_back();
        if (mark[u] == gen) continue;
        mark[u] = gen;
        if (st.is_leaf(g, u)) {
          leaves++;
          continue;
        }
        add++;
        stk.push_back(g.fa[u] >> 1);
        stk.push_back(g.fb[u] >> 1);
      }
      return add;
    };
    auto endpoint_bits = [&](uint32_t e) {
      uint64_t eb = 0;
      st.for_each_input(g, e, [&](uint32_t) { eb++; });
      return eb;
    };
    // Balanced mode weighs an SRAM endpoint as this many AND gates: the
    // batched kernel's SRAM port (staging, transposes, the row read and write
    // of every stream) adds about 2.5k SM cycles to a work item, the time of
    // about 1.2k gates at level 1.
    constexpr uint64_t SRAM_CONE_WEIGHT = 1200;
    const size_t nso = st.staged_outputs.size();
    const size_t npo = g.primary_outputs.size(), nd = g.dffs.size();
    auto weight = [&](uint32_t e) -> uint64_t {
      return e >= nso && st.endpoints[e - nso] >= npo + nd ? SRAM_CONE_WEIGHT : 0;
    };
    // Balanced: a chunk is closed before the endpoint whose cone would take
    // it past `bound`, so no chunk of several endpoints exceeds it.  Returns
    // the number of chunks (stored into `out` when given).
    auto cut_balanced = [&](uint64_t bound, std::vector<std::vector<uint32_t>> *out) {
      size_t n = 0;
      std::vector<uint32_t> cur;
      uint64_t cone = 0, bits = 0;
      ++gen;
      for (uint32_t e : order) {
        const uint64_t eb = endpoint_bits(e);
        bool close = !cur.empty() && bits + eb > opt.target_endpoint_bits;
        uint64_t add = 0;
        if (!close) {
          add = grow(e) + weight(e);
          add += (input_w16 * leaves) >> 4;
          close = !cur.empty() && cone + add > bound;
        }
        if (close) {
          ++n;
          if (out) out->push_back(cur);
          cur.clear();
          cone = bits = 0;
          ++gen;
          add = grow(e) + weight(e);
          add += (input_w16 * leaves) >> 4;
        }
        cur.push_back(e);
        cone += add;
        bits += eb;
      }
      if (!cur.empty()) {
        ++n;
        if (out) out->push_back(cur);
      }
      ++gen;
      return n;
    };
    if (opt.target_parts) {
      // the smallest bound that cuts the stage into at most target_parts
      // chunks (binary search; the whole stage as one chunk is the top)
      uint64_t lo = 1, hi = 0;
      ++gen;
      for (uint32_t e : order) {
        hi += grow(e) + weight(e);
        hi += (input_w16 * leaves) >> 4;
      }
      hi = std::max<uint64_t>(hi, 1);
      while (lo < hi) {
        const uint64_t mid = lo + (hi - lo) / 2;
        if (cut_balanced(mid, nullptr) <= opt.target_parts) hi = mid;
        else lo = mid + 1;
      }
      cone_bound = lo;
      cut_balanced(lo, &chunks);
    } else {
      std::vector<uint32_t> cur;
      uint64_t cone = 0, bits = 0;
      for (uint32_t e : order) {
        const uint64_t eb = endpoint_bits(e);
        if (!cur.empty() && (bits + eb > opt.target_endpoint_bits)) {
          chunks.push_back(cur);
          cur.clear();
          cone = bits = 0;
          ++gen;
        }
        const uint64_t add = grow(e);
        cur.push_back(e);
        cone += add;
        bits += eb;
        if (cone >= opt.target_cone) {
          chunks.push_back(cur);
          cur.clear();
          cone = bits = 0;
          ++gen;
        }
      }
      if (!cur.empty()) chunks.push_back(cur);
    }
  }

  // ---- 3. pack; split failures in half
  std::vector<Partition> good;
  while (!chunks.empty()) {
    std::vector<Partition> built(chunks.size());
    std::vector<uint8_t> ok(chunks.size(), 0);
    parallel_for(chunks.size(), threads, [&](size_t i) {
      ok[i] = build_partition(g, st, chunks[i], built[i], po);
    });
    std::vector<std::vector<uint32_t>> retry;
    for (size_t i = 0; i < chunks.size(); ++i) {
      if (ok[i]) {
        good.push_back(std::move(built[i]));
        continue;
      }
      if (chunks[i].size() == 1)
        throw std::runtime_error("a single endpoint does not fit one partition; use finer level splits");
      size_t h = chunks[i].size() / 2;
      retry.push_back(std::vector<uint32_t>(chunks[i].begin(), chunks[i].begin() + h));
      retry.push_back(std::vector<uint32_t>(chunks[i].begin() + h, chunks[i].end()));
    }
    chunks.swap(retry);
  }

  return good;
  };

  std::vector<Partition> good;
  if (opt.target_parts && opt.cost_model && opt.cost_model->valid()) {
    // ---- 3b. learned choice of the cut.  All partitions of a stage run at
    // once, so the stage lasts as long as its slowest item.  The stage is
    // cut with several weights of chunk inputs against cone gates, and the
    // cut whose slowest partition the cost model predicts fastest is kept
    // (a cut with more than target_parts partitions needs a second round of
    // items and is taken only when every cut does).
    double best = 0;
    size_t best_n = 0;
    uint64_t best_bound = 0;
    for (uint64_t w16 : {0, 4, 8, 16, 32}) {
      std::vector<Partition> cand = cut_and_pack(w16);
      std::vector<double> pred(cand.size());
      parallel_for(cand.size(), threads, [&](size_t i) {
        float f[NFEAT];
        partition_features(g, st, cand[i], opt.xpins, f);
        pred[i] = (double)opt.cost_model->predict(f);  // log cycles
      });
      const double worst = pred.empty() ? 0.0 : *std::max_element(pred.begin(), pred.end());
      const size_t n = cand.size();
      const bool over = n > opt.target_parts, best_over = best_n > opt.target_parts;
      const bool take = good.empty() || (over != best_over ? !over
                                         : over ? n < best_n : worst < best - 1e-6);
      if (take) {
        good = std::move(cand);
        best = worst;
        best_n = n;
        best_bound = cone_bound;
      }
    }
    cone_bound = best_bound;
  } else {
    good = cut_and_pack(opt.target_parts ? opt.input_weight16 : 0);
  }

  // ---- 4. merge neighbours (in endpoint order) when it costs no stages
  for (int pass = 0; pass < opt.merge_passes && good.size() > 1; ++pass) {
    std::vector<Partition> merged;
    // candidate pairs (i, i+1) evaluated in parallel, accepted greedily
    size_t np = good.size();
    std::vector<Partition> trial(np);
    std::vector<uint8_t> tok(np, 0);
    parallel_for(np - 1, threads, [&](size_t i) {
      std::vector<uint32_t> eps = good[i].endpoints;
      eps.insert(eps.end(), good[i + 1].endpoints.begin(), good[i + 1].endpoints.end());
      Partition p;
      if (!build_partition(g, st, eps, p, po)) return;
      if (opt.target_parts && p.cone_ands > cone_bound) return;  // keep the balance
      bool accept;
      if (opt.cost_model && opt.cost_model->valid()) {
        // learned rule: merge when the predicted kernel time of the merged
        // partition is below the two it replaces
        float fa[NFEAT], fb[NFEAT], fm[NFEAT];
        partition_features(g, st, good[i], opt.xpins, fa);
        partition_features(g, st, good[i + 1], opt.xpins, fb);
        partition_features(g, st, p, opt.xpins, fm);
        const double ca = std::exp((double)opt.cost_model->predict(fa));
        const double cb = std::exp((double)opt.cost_model->predict(fb));
        const double cm = std::exp((double)opt.cost_model->predict(fm));
        accept = cm < ca + cb;
      } else {
        accept = p.stages.size() <= std::max(good[i].stages.size(), good[i + 1].stages.size());
      }
      if (accept) {
        trial[i] = std::move(p);
        tok[i] = 1;
      }
    });
    for (size_t i = 0; i < np;) {
      if (i + 1 < np && tok[i]) {
        merged.push_back(std::move(trial[i]));
        i += 2;
      } else {
        merged.push_back(std::move(good[i]));
        i += 1;
      }
    }
    bool changed = merged.size() != good.size();
    good.swap(merged);
    if (!changed) break;
  }
  return good;
}

}  // namespace jq
