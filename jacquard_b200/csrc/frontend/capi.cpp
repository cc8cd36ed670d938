// extern "C" surface of the script front end (host only; no CUDA).
// Declared in include/jacquard_frontend.h.
#include <cstring>
#include <memory>
#include <stdexcept>

#include "frontend.hpp"

#include <algorithm>
#include "../../../include/jacquard_frontend.h"

using namespace jq;

namespace {
struct Design {
  AIG g;
  GenInfo info;
  uint32_t n_inputs = 0;  // input pins added by the builder
};
CostModel unpack_model(const float *m) {
  CostModel cm;
  const int NF = NFEAT, H = 128;
  cm.w1.assign(m, m + H * NF);
  m += H * NF;
  cm.b1.assign(m, m + H);
  m += H;
  cm.w2.assign(m, m + H * H);
  m += H * H;
  cm.b2.assign(m, m + H);
  m += H;
  cm.w3.assign(m, m + H);
  m += H;
  cm.b3 = *m++;
  cm.mean.assign(m, m + NF);
  m += NF;
  cm.inv_std.assign(m, m + NF);
  return cm;
}
struct Script {
  FlatScript s;
  std::vector<StagedAIG> stageds;
  std::vector<std::vector<Partition>> parts;
  std::vector<uint32_t> dff_d, dff_en, dff_q, po;
};
void set_err(char *err, size_t n, const std::string &m) {
  if (!err || !n) return;
  std::strncpy(err, m.c_str(), n - 1);
  err[n - 1] = 0;
}
}  // namespace

extern "C" {

void *jqf_generate(const jqf_gen_params *p, uint64_t *num_and) {
  try {
    GenParams gp;
    gp.seed = p->seed;
    gp.n_clusters = p->n_clusters;
    gp.nodes_per_cluster = p->nodes_per_cluster;
    gp.depth = p->depth;
    gp.fanin_window = p->fanin_window;
    gp.intra_frac = p->intra_frac;
    gp.n_dff = p->n_dff;
    gp.n_pi = p->n_pi;
    gp.n_po = p->n_po;
    gp.n_sram = p->n_sram;
    gp.sram_addr_bits = p->sram_addr_bits;
    gp.with_reset = p->with_reset;
    auto *d = new Design;
    d->g = generate_design(gp, &d->info);
    if (num_and) *num_and = d->info.num_and;
    return d;
  } catch (...) {
    return nullptr;
  }
}

void jqf_free_design(void *d) { delete static_cast<Design *>(d); }

// ---- AIG builder for designs read from a gate-level netlist.  Sources
// (inputs, clock flags, DFF Q pins) can be added at any time; AND gates are
// structurally hashed and constant-folded (src/aig.rs:327-345), so pins stay
// in topological order.
void *jqf_builder_new(void) {
  try {
    return new Design;
  } catch (...) {
    return nullptr;
  }
}

uint32_t jqf_builder_input(void *b) {
  auto *d = static_cast<Design *>(b);
  return d->g.add_pin(DRV_INPUT, d->n_inputs++);
}

uint32_t jqf_builder_clock_flag(void *b) {
  return static_cast<Design *>(b)->g.add_pin(DRV_CLKFLAG, 0);
}

uint32_t jqf_builder_dff(void *b) {
  auto *d = static_cast<Design *>(b);
  uint32_t i = (uint32_t)d->g.dffs.size();
  d->g.dffs.emplace_back();
  d->g.dffs[i].q = d->g.add_pin(DRV_DFF, i);
  return d->g.dffs[i].q;
}

int jqf_builder_set_dff(void *b, uint32_t index, uint32_t d_iv, uint32_t en_iv) {
  auto *d = static_cast<Design *>(b);
  if (index >= d->g.dffs.size() || (d_iv >> 1) > d->g.num_pins || (en_iv >> 1) > d->g.num_pins)
    return -1;
  d->g.dffs[index].d_iv = d_iv;
  d->g.dffs[index].en_iv = en_iv;
  return 0;
}

uint32_t jqf_builder_and(void *b, uint32_t a_iv, uint32_t b_iv) {
  auto *d = static_cast<Design *>(b);
  if ((a_iv >> 1) > d->g.num_pins || (b_iv >> 1) > d->g.num_pins) return NONE;
  const uint32_t before = d->g.num_pins;
  const uint32_t r = d->g.add_and(a_iv, b_iv);
  d->info.num_and += d->g.num_pins - before;
  return r;
}

int64_t jqf_builder_output(void *b, uint32_t iv) {
  auto *d = static_cast<Design *>(b);
  if ((iv >> 1) > d->g.num_pins) return -1;
  auto &po = d->g.primary_outputs;
  for (size_t i = 0; i < po.size(); ++i)
    if (po[i] == iv) return (int64_t)i;
  po.push_back(iv);
  return (int64_t)po.size() - 1;
}

int jqf_builder_finish(void *b, uint32_t clock_flag_pin, uint32_t reset_pin) {
  auto *d = static_cast<Design *>(b);
  for (const DFF &f : d->g.dffs)
    if (f.q == 0) return -1;
  d->info.clock_flag_pin = clock_flag_pin;
  d->info.reset_pin = reset_pin;
  return 0;
}

int jqf_design_info(void *dp, jqf_design_info_t *out) {
  auto *d = static_cast<Design *>(dp);
  out->num_pins = d->g.num_pins;
  out->num_and = d->info.num_and;
  out->num_dffs = d->g.dffs.size();
  out->num_pos = d->g.primary_outputs.size();
  out->num_srams = d->g.srams.size();
  out->clock_flag_pin = d->info.clock_flag_pin;
  out->reset_pin = d->info.reset_pin;
  return 0;
}

// which: 0 kind(u8) 1 fa 2 fb 3 dff_d 4 dff_en 5 dff_q 6 po 7 sram (flattened
// RAMBlock u32 records of JQF_SRAM_RECORD_WORDS words)
int64_t jqf_design_array(void *dp, int which, void *dst, size_t cap) {
  auto *d = static_cast<Design *>(dp);
  const AIG &g = d->g;
  std::vector<uint32_t> tmp;
  const void *src = nullptr;
  size_t bytes = 0;
  switch (which) {
    case 0: src = g.kind.data(); bytes = g.kind.size(); break;
    case 1: src = g.fa.data(); bytes = g.fa.size() * 4; break;
    case 2: src = g.fb.data(); bytes = g.fb.size() * 4; break;
    case 3: for (auto &x : g.dffs) tmp.push_back(x.d_iv); break;
    case 4: for (auto &x : g.dffs) tmp.push_back(x.en_iv); break;
    case 5: for (auto &x : g.dffs) tmp.push_back(x.q); break;
    case 6: tmp = g.primary_outputs; break;
    case 7:
      for (auto &r : g.srams) {
        tmp.insert(tmp.end(), r.r_addr_iv, r.r_addr_iv + SRAM_ADDR_BITS);
        tmp.push_back(r.r_en_iv);
        tmp.insert(tmp.end(), r.r_data, r.r_data + 32);
        tmp.insert(tmp.end(), r.w_addr_iv, r.w_addr_iv + SRAM_ADDR_BITS);
        tmp.insert(tmp.end(), r.w_en_iv, r.w_en_iv + 32);
        tmp.insert(tmp.end(), r.w_data_iv, r.w_data_iv + 32);
      }
      break;
    default: return -1;
  }
  if (!src) { src = tmp.data(); bytes = tmp.size() * 4; }
  if (dst && cap >= bytes) std::memcpy(dst, src, bytes);
  return (int64_t)bytes;
}

int jqf_set_delays(void *dp, const uint32_t *rise, const uint32_t *fall, size_t n) {
  auto *d = static_cast<Design *>(dp);
  if (n != (size_t)d->g.num_pins + 1) return -1;
  d->g.delay_rise.assign(rise, rise + n);
  d->g.delay_fall.assign(fall, fall + n);
  return 0;
}

void *jqf_build_script(void *dp, const jqf_build_params *bp, char *err, size_t errlen) {
  auto *d = static_cast<Design *>(dp);
  try {
    auto sc = std::make_unique<Script>();
    std::vector<uint32_t> split(bp->level_split, bp->level_split + bp->n_level_split);
    sc->stageds = build_staged_aigs(d->g, split);
    PartitionOptions po;
    if (bp->target_cone) po.target_cone = bp->target_cone;
    if (bp->target_endpoint_bits) po.target_endpoint_bits = bp->target_endpoint_bits;
    po.num_threads = bp->num_threads;
    po.merge_passes = bp->merge_passes;
    po.target_parts = bp->target_parts;
    po.input_weight16 = bp->input_weight16;
    CostModel cm;
    std::vector<uint8_t> xp;
    if (bp->cost_model) {
      cm = unpack_model(bp->cost_model);
      po.cost_model = &cm;
      if (bp->xprop) {
        xp = d->g.x_capable_pins();
        po.xpins = &xp;
      }
    }
    for (auto &st : sc->stageds) sc->parts.push_back(partition_stage(d->g, st, po));
    FlattenOptions fo;
    fo.num_blocks = bp->num_blocks;
    fo.xprop = bp->xprop != 0;
    std::string e;
    if (!flatten_script(d->g, sc->stageds, sc->parts, fo, sc->s, &e)) {
      set_err(err, errlen, "flatten: " + e);
      return nullptr;
    }
    if (!d->g.delay_rise.empty()) inject_timing(sc->s, d->g.delay_rise, d->g.delay_fall);
    size_t words = (size_t)sc->s.reg_io_state_size * (fo.xprop ? 2 : 1);
    std::string v = validate_script(sc->s, words);
    if (!v.empty()) {
      set_err(err, errlen, "validate: " + v);
      return nullptr;
    }
    return sc.release();
  } catch (const std::exception &ex) {
    set_err(err, errlen, ex.what());
    return nullptr;
  }
}

void jqf_free_script(void *s) { delete static_cast<Script *>(s); }

int jqf_script_info(void *sp, jqf_script_info_t *out) {
  auto *sc = static_cast<Script *>(sp);
  const FlatScript &s = sc->s;
  out->num_blocks = s.num_blocks;
  out->num_major_stages = s.num_major_stages;
  out->blocks_data_len = s.blocks_data.size();
  out->reg_io_state_size = s.reg_io_state_size;
  out->sram_storage_size = s.sram_storage_size;
  out->xprop_enabled = s.xprop_enabled;
  out->xprop_state_offset = s.xprop_state_offset;
  out->num_partitions = s.partition_x_capable.size();
  out->num_delay_patches = s.delay_patch_offset.size();
  uint64_t st = 0;
  for (uint32_t n : s.part_num_stages) st += n;
  out->total_boomerang_stages = st;
  return 0;
}

// which: 0 blocks_start(u64) 1 blocks_data(u32) 2 input_map(pairs u32)
// 3 output_map(pairs) 4 staged_io_map(pairs) 5 partition_x_capable(u8)
// 6 part_num_stages(u32) 7 dff_data_pos(u32) 8 input_layout(u32)
// 9 stage/block/partition triples (u32): (major stage, block, part index)
int64_t jqf_script_array(void *sp, int which, void *dst, size_t cap) {
  auto *sc = static_cast<Script *>(sp);
  const FlatScript &s = sc->s;
  std::vector<uint32_t> tmp;
  std::vector<uint64_t> t64;
  const void *src = nullptr;
  size_t bytes = 0;
  switch (which) {
    case 0:
      for (size_t v : s.blocks_start) t64.push_back(v);
      src = t64.data(); bytes = t64.size() * 8; break;
    case 1: src = s.blocks_data.data(); bytes = s.blocks_data.size() * 4; break;
    case 2: for (auto &kv : s.input_map) { tmp.push_back(kv.first); tmp.push_back(kv.second); } break;
    case 3: for (auto &kv : s.output_map) { tmp.push_back(kv.first); tmp.push_back(kv.second); } break;
    case 4: for (auto &kv : s.staged_io_map) { tmp.push_back(kv.first); tmp.push_back(kv.second); } break;
    case 5: src = s.partition_x_capable.data(); bytes = s.partition_x_capable.size(); break;
    case 6: tmp = s.part_num_stages; break;
    case 7: tmp = s.dff_data_pos; break;
    case 8: tmp = s.input_layout; break;
    case 9:
      for (size_t ms = 0; ms < s.stages_blocks_parts.size(); ++ms)
        for (size_t b = 0; b < s.stages_blocks_parts[ms].size(); ++b)
          for (uint32_t p : s.stages_blocks_parts[ms][b]) {
            tmp.push_back((uint32_t)ms); tmp.push_back((uint32_t)b); tmp.push_back(p);
          }
      break;
    case 10:
      // per partition (major stage order): major stage, #stages, cone ANDs,
      // targets, endpoints
      for (size_t ms = 0; ms < sc->parts.size(); ++ms)
        for (const Partition &p : sc->parts[ms]) {
          tmp.push_back((uint32_t)ms);
          tmp.push_back((uint32_t)p.stages.size());
          tmp.push_back(p.cone_ands);
          tmp.push_back(p.targets);
          tmp.push_back((uint32_t)p.endpoints.size());
        }
      break;
    default: return -1;
  }
  if (!src) { src = tmp.data(); bytes = tmp.size() * 4; }
  if (dst && cap >= bytes) std::memcpy(dst, src, bytes);
  return (int64_t)bytes;
}

// ---- RepCut hypergraph inputs of one staged slice (src/repcut.rs:58-176).
// Fills (each pointer may be null to only get sizes):
//   fanout_start[num_pins + 2], fanouts[]: AND-gate fanouts of every pin,
//     built as src/aig.rs:2640-2669 does (counts, prefix sums, filled from
//     the back in driver order);
//   ep_start[E + 1], ep_pins[]: each endpoint group's input pins
//     (EndpointGroup::for_each_input order, duplicates kept);
//   staged[num_pins + 1]: 1 for the slice's staged inputs (traversal stops);
//   rlevel[num_pins + 1]: 0 for pins without AND fanouts, else 1 + the
//     largest rlevel of a fanout;
//   flevel[num_pins + 1]: 0 for non-AND pins, else 1 + the largest flevel
//     of the AND fanins.
// sizes[0] = number of endpoint groups E, sizes[1] = fanout list length,
// sizes[2] = ep_pins length.
// The reference's results depend on its traversal order (TopoTraverser,
// src/aig.rs:3125-3170) where a staged input and one of its fanins are both
// in a cone.  The traversal is restated to report those cases:
//   supp_start[blocks + 1], supp_edges[]: per block of 4096 endpoints, the
//     fanout-edge indices k (fanouts[k] = staged j, k in i's range) along
//     which i, coming later in the block's post-order, does not take j's set;
//   wsupp[num_pins + 1]: bit 0 / bit 1 when a staged pin comes before its
//     fanin a / b in the all-endpoint post-order, so its weight misses that
//     fanin's.
// sizes[3] = supp_edges length.
static uint32_t repcut_topo(const AIG &g, const std::vector<uint8_t> &stg, const uint32_t *starts,
                            size_t n_start, std::vector<int32_t> &pos,
                            std::vector<uint32_t> &touched) {
  std::vector<uint32_t> stack;
  stack.reserve(n_start + 64);
  for (size_t k = 0; k < n_start; ++k) stack.push_back(starts[k] << 1);
  uint32_t n = 0;
  while (!stack.empty()) {
    const uint32_t item = stack.back();
    stack.pop_back();
    const uint32_t u = item >> 1;
    if (item & 1) {
      pos[u] = (int32_t)n++;
      continue;
    }
    if (pos[u] != -1) continue;
    pos[u] = -2;  // visited, not yet post-ordered
    touched.push_back(u);
    stack.push_back((u << 1) | 1);
    if (g.kind[u] == DRV_AND && !stg[u]) {
      if (g.fb[u] >> 1) stack.push_back((g.fb[u] >> 1) << 1);
      if (g.fa[u] >> 1) stack.push_back((g.fa[u] >> 1) << 1);
    }
  }
  return n;
}

int jqf_repcut_slice(void *dp, const uint32_t *level_split, size_t n_split, uint32_t slice,
                     uint32_t *fanout_start, uint32_t *fanouts, uint32_t *ep_start,
                     uint32_t *ep_pins, uint8_t *staged, uint32_t *rlevel, uint32_t *flevel,
                     uint32_t *supp_start, uint32_t *supp_edges, uint8_t *wsupp,
                     uint64_t *sizes) {
  try {
    auto *d = static_cast<Design *>(dp);
    const AIG &g = d->g;
    std::vector<uint32_t> split(level_split, level_split + n_split);
    std::vector<StagedAIG> st = build_staged_aigs(g, split);
    if (slice >= st.size()) return -1;
    const StagedAIG &sa = st[slice];
    const uint32_t N = g.num_pins;
    std::vector<uint32_t> fs(N + 2, 0);
    for (uint32_t p = 1; p <= N; ++p)
      if (g.kind[p] == DRV_AND) {
        if (g.fa[p] >> 1) fs[g.fa[p] >> 1]++;
        if (g.fb[p] >> 1) fs[g.fb[p] >> 1]++;
      }
    for (uint32_t i = 1; i < N + 2; ++i) fs[i] += fs[i - 1];
    std::vector<uint32_t> fo(fs[N + 1]);
    for (uint32_t p = 0; p <= N; ++p)
      if (g.kind[p] == DRV_AND) {
        if (g.fa[p] >> 1) fo[--fs[g.fa[p] >> 1]] = p;
        if (g.fb[p] >> 1) fo[--fs[g.fb[p] >> 1]] = p;
      }
    const size_t E = sa.num_endpoint_groups();
    std::vector<uint32_t> es(E + 1, 0), ep;
    for (size_t e = 0; e < E; ++e) {
      sa.for_each_input(g, e, [&](uint32_t pin) { ep.push_back(pin); });
      es[e + 1] = (uint32_t)ep.size();
    }
    auto is_staged = [&](uint32_t p) { return sa.has_staged_inputs && sa.is_staged_input[p]; };
    std::vector<uint32_t> rl(N + 1, 0), fl(N + 1, 0);
    for (uint32_t p = N; p >= 1; --p) {
      uint32_t m = 0;
      bool any = false;
      for (uint32_t k = fs[p]; k < fs[p + 1]; ++k) {
        any = true;
        m = std::max(m, rl[fo[k]]);
      }
      rl[p] = any ? m + 1 : 0;
    }
    for (uint32_t p = 1; p <= N; ++p)
      if (g.kind[p] == DRV_AND) fl[p] = 1 + std::max(fl[g.fa[p] >> 1], fl[g.fb[p] >> 1]);
    std::vector<uint8_t> stg(N + 1, 0);
    for (uint32_t p = 0; p <= N; ++p) stg[p] = is_staged(p) ? 1 : 0;
    // per block: edges i -> staged j with i later than j in the post-order
    std::vector<int32_t> pos(N + 1, -1);
    std::vector<uint32_t> touched, ss{0}, se;
    for (size_t b0 = 0; b0 < E; b0 += 4096) {
      const size_t b1 = std::min(E, b0 + 4096);
      touched.clear();
      repcut_topo(g, stg, ep.data() + es[b0], es[b1] - es[b0], pos, touched);
      for (uint32_t j : touched) {
        if (!stg[j] || g.kind[j] != DRV_AND) continue;
        for (uint32_t f : {g.fa[j] >> 1, g.fb[j] >> 1}) {
          if (!f || pos[f] < 0 || pos[f] <= pos[j]) continue;
          for (uint32_t k = fs[f]; k < fs[f + 1]; ++k)
            if (fo[k] == j) se.push_back(k);
        }
      }
      for (uint32_t u : touched) pos[u] = -1;
      ss.push_back((uint32_t)se.size());
    }
    std::vector<uint8_t> ws(N + 1, 0);
    touched.clear();
    repcut_topo(g, stg, ep.data(), ep.size(), pos, touched);
    for (uint32_t j : touched) {
      if (!stg[j] || g.kind[j] != DRV_AND) continue;
      const uint32_t a = g.fa[j] >> 1, b = g.fb[j] >> 1;
      if (a && pos[a] > pos[j]) ws[j] |= 1;
      if (b && pos[b] > pos[j]) ws[j] |= 2;
    }
    if (sizes) {
      sizes[0] = E;
      sizes[1] = fo.size();
      sizes[2] = ep.size();
      sizes[3] = se.size();
    }
    if (supp_start) std::copy(ss.begin(), ss.end(), supp_start);
    if (supp_edges) std::copy(se.begin(), se.end(), supp_edges);
    if (wsupp) std::copy(ws.begin(), ws.end(), wsupp);
    if (fanout_start) std::copy(fs.begin(), fs.end(), fanout_start);
    if (fanouts) std::copy(fo.begin(), fo.end(), fanouts);
    if (ep_start) std::copy(es.begin(), es.end(), ep_start);
    if (ep_pins) std::copy(ep.begin(), ep.end(), ep_pins);
    if (staged)
      for (uint32_t p = 0; p <= N; ++p) staged[p] = is_staged(p) ? 1 : 0;
    if (rlevel) std::copy(rl.begin(), rl.end(), rlevel);
    if (flevel) std::copy(fl.begin(), fl.end(), flevel);
    return (int64_t)st.size();
  } catch (...) {
    return -1;
  }
}

int jqf_script_features(void *dp, void *sp, float *out) {
  auto *d = static_cast<Design *>(dp);
  auto *sc = static_cast<Script *>(sp);
  std::vector<uint8_t> xp;
  if (sc->s.xprop_enabled) xp = d->g.x_capable_pins();
  for (size_t i = 0; i < sc->s.part_ptrs.size(); ++i)
    partition_features(d->g, sc->stageds[sc->s.part_major_stage[i]], *sc->s.part_ptrs[i],
                       sc->s.xprop_enabled ? &xp : nullptr, out + i * NFEAT);
  return 0;
}

int jqf_cost_model_predict(const float *model, const float *features, size_t n, float *out) {
  CostModel cm = unpack_model(model);
  for (size_t i = 0; i < n; ++i) out[i] = cm.predict(features + i * NFEAT);
  return 0;
}

int jqf_validate(const uint64_t *blocks_start, size_t num_blocks, size_t num_major_stages,
                 const uint32_t *blocks_data, size_t blocks_data_len,
                 uint32_t reg_io_state_size, uint32_t sram_storage_size,
                 size_t state_words, char *err, size_t errlen) {
  FlatScript s;
  s.num_blocks = num_blocks;
  s.num_major_stages = num_major_stages;
  s.blocks_start.assign(blocks_start, blocks_start + num_blocks * num_major_stages + 1);
  s.blocks_data.assign(blocks_data, blocks_data + blocks_data_len);
  s.reg_io_state_size = reg_io_state_size;
  s.sram_storage_size = sram_storage_size;
  std::string v = validate_script(s, state_words);
  set_err(err, errlen, v);
  return v.empty() ? 0 : -1;
}

// src/flatten.rs:97-123 (effective setup/hold with clock arrival folded in)
// and :1891-1924 (per-word minimum, 0 = unset).
int jqf_constraint_buffer(uint32_t num_words, uint64_t clock_period_ps, size_t n,
                          const uint16_t *setup_ps, const uint16_t *hold_ps,
                          const int16_t *clock_arrival_ps, const uint32_t *data_state_pos,
                          uint32_t *out_clock_ps, uint32_t *out_words) {
  for (uint32_t i = 0; i < num_words; ++i) out_words[i] = 0;
  for (size_t k = 0; k < n; ++k) {
    if (data_state_pos[k] == 0xffffffffu) continue;
    uint32_t w = data_state_pos[k] / 32;
    if (w >= num_words) continue;
    int32_t su = (int32_t)setup_ps[k] - (int32_t)clock_arrival_ps[k];
    int32_t ho = (int32_t)hold_ps[k] + (int32_t)clock_arrival_ps[k];
    uint16_t es = (uint16_t)(su < 0 ? 0 : (su > 65535 ? 65535 : su));
    uint16_t eh = (uint16_t)(ho < 0 ? 0 : (ho > 65535 ? 65535 : ho));
    uint32_t ex = out_words[w];
    uint16_t os = (uint16_t)(ex >> 16), oh = (uint16_t)(ex & 0xffff);
    uint16_t ns = os == 0 ? es : (os < es ? os : es);
    uint16_t nh = oh == 0 ? eh : (oh < eh ? oh : eh);
    out_words[w] = (uint32_t)ns << 16 | nh;
  }
  *out_clock_ps = clock_period_ps > 0xffffffffull ? 0xffffffffu : (uint32_t)clock_period_ps;
  return 0;
}

// src/flatten.rs:1812-1846 restated on explicit arrays (patch offsets and the
// pins at each offset, CSR), writing into `blocks_data`.
int jqf_inject_delays(uint32_t *blocks_data, size_t blocks_data_len, size_t n_patches,
                      const uint64_t *offsets, const uint32_t *pins_start, const uint32_t *pins,
                      const uint16_t *rise, const uint16_t *fall, size_t n_pins) {
  for (size_t i = 0; i < n_patches; ++i) {
    uint32_t m = 0;
    for (uint32_t k = pins_start[i]; k < pins_start[i + 1]; ++k) {
      uint32_t p = pins[k];
      if (p < n_pins) m = std::max<uint32_t>(m, std::max(rise[p], fall[p]));
    }
    if (offsets[i] < blocks_data_len) blocks_data[offsets[i]] = m > 65535 ? 65535 : m;
  }
  return 0;
}

}  // extern "C"
