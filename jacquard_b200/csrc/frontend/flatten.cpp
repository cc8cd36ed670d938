// Flattener: lays partitions out as the reference's FlattenedScriptV1
// instruction stream.  The format is the kernel ABI, so the layout rules are
// kept identical to the reference (src/flatten.rs:198-258 format doc,
// :343-400 global-read round mapping, :863-1130 per-partition script,
// :1133-1573 block assembly, state/SRAM offsets, X classification); the code
// is this project's own C++.
#include "frontend.hpp"

#include <algorithm>
#include <map>
#include <unordered_map>

namespace jq {

namespace {

inline uint32_t lvl_len(int l) { return 8192u >> l; }

inline void set_bit(uint32_t &v, uint32_t pos, uint32_t bit) {
  if (bit) v |= 1u << pos;
  else v &= ~(1u << pos);
}

// Insertion-ordered map with "insert overwrites value, keeps position"
// semantics (the reference's IndexMap).
template <class K, class V>
struct OrderedMap {
  std::vector<std::pair<K, V>> items;
  std::unordered_map<K, size_t> idx;
  void insert(const K &k, const V &v) {
    auto it = idx.find(k);
    if (it == idx.end()) {
      idx.emplace(k, items.size());
      items.push_back({k, v});
    } else {
      items[it->second].second = v;
    }
  }
  const V *get(const K &k) const {
    auto it = idx.find(k);
    return it == idx.end() ? nullptr : &items[it->second].second;
  }
};

// map_global_read_to_rounds (src/flatten.rs:343-400).
bool map_rounds(const std::vector<std::pair<uint32_t, uint32_t>> &taken,
                std::vector<std::vector<std::pair<uint32_t, uint32_t>>> &rounds) {
  rounds.assign(NT, {});
  if (taken.empty()) return true;
  size_t chunk = taken.size();
  while (chunk >= 1) {
    std::vector<std::pair<size_t, size_t>> slices;  // [begin, end)
    for (size_t b = 0; b < taken.size(); b += chunk)
      slices.push_back({b, std::min(taken.size(), b + chunk)});
    auto pc = [&](const std::pair<size_t, size_t> &s) {
      uint32_t t = 0;
      for (size_t i = s.first; i < s.second; ++i) t += __builtin_popcount(taken[i].second);
      return t;
    };
    std::stable_sort(slices.begin(), slices.end(),
                     [&](const auto &a, const auto &b) { return pc(a) > pc(b); });
    std::vector<std::vector<std::pair<uint32_t, uint32_t>>> rm(NT);
    std::vector<uint32_t> fill(NT, 0);
    size_t j = 0;
    bool fail = false;
    for (auto &s : slices) {
      for (size_t i = s.first; i < s.second && !fail; ++i) {
        uint32_t c = __builtin_popcount(taken[i].second);
        size_t wrap = j;
        while (fill[j] + c > 32) {
          j = (j + 1) % NT;
          if (j == wrap) { fail = true; break; }
        }
        if (fail) break;
        rm[j].push_back(taken[i]);
        fill[j] += c;
        j = (j + 1) % NT;
      }
      if (fail) break;
    }
    if (!fail) {
      rounds.swap(rm);
      return true;
    }
    chunk /= 2;
  }
  return false;
}

struct FPart {
  std::vector<std::vector<uint32_t>> afters;
  std::vector<uint32_t> wos;  // pins of the normal writeouts
  std::unordered_map<uint32_t, uint16_t> pin2pos;
  uint32_t num_srams = 0, num_normal = 0, num_dup = 0, num_writeouts = 0;
  // pin -> ordered (activation key -> position or -1)
  std::vector<std::pair<uint32_t, std::vector<std::pair<uint32_t, int32_t>>>> acts;
  std::unordered_map<uint32_t, size_t> acts_idx;
  uint32_t cnt_dup = 0;
  uint32_t state_start = 0, sram_start = 0;
  std::vector<uint16_t> sd_perm, ck_perm;
  std::vector<uint32_t> sd_inv, sd_set0, ck_inv, ck_set0, d_inv;

  void add_act(uint32_t pin, uint32_t key) {
    auto it = acts_idx.find(pin);
    if (it == acts_idx.end()) {
      acts_idx.emplace(pin, acts.size());
      acts.push_back({pin, {{key, -1}}});
      return;
    }
    auto &v = acts[it->second].second;
    for (auto &kv : v)
      if (kv.first == key) return;
    v.push_back({key, -1});
  }
};

}  // namespace

// src/flatten.rs:466-561 init_afters_writeouts
static void init_part(const AIG &g, const StagedAIG &st, const Partition &p, FPart &fp) {
  for (const BoomStage &s : p.stages) {
    std::vector<uint32_t> after;
    after.reserve(8192);
    after.push_back(NONE);
    for (int l = BOOM_STAGES; l >= 1; --l)
      after.insert(after.end(), s.hier[l].begin(), s.hier[l].end());
    for (uint16_t w : s.write_outs)
      for (int k = 0; k < 32; ++k) fp.wos.push_back(after[w * 32 + k]);
    fp.num_normal += (uint32_t)s.write_outs.size();
    fp.afters.push_back(std::move(after));
  }
  size_t nso = st.staged_outputs.size();
  size_t npo = g.primary_outputs.size(), nd = g.dffs.size();
  for (uint32_t e : p.endpoints) {
    if (e < nso) {
      fp.add_act(st.staged_outputs[e], 2);
      continue;
    }
    size_t o = st.endpoints[e - nso];
    if (o < npo) {
      uint32_t iv = g.primary_outputs[o];
      if (iv <= 1) continue;
      fp.add_act(iv >> 1, 2 | (iv & 1));
    } else if (o < npo + nd) {
      const DFF &d = g.dffs[o - npo];
      if (d.d_iv <= 1) continue;
      fp.add_act(d.d_iv >> 1, d.en_iv << 1 | (d.d_iv & 1));
    } else {
      fp.num_srams++;
    }
  }
  uint32_t dsum = 0;
  for (auto &a : fp.acts) dsum += (uint32_t)a.second.size() - 1;
  fp.num_dup = (dsum + 31) / 32;
  fp.num_writeouts = fp.num_normal + fp.num_srams + fp.num_dup;
  for (size_t i = 0; i < fp.wos.size(); ++i)
    if (fp.wos[i] != NONE) fp.pin2pos[fp.wos[i]] = (uint16_t)i;  // last wins
}

namespace {
struct Perm {
  uint16_t perm;
  uint32_t inv, set0;
};
}  // namespace

static bool query_perm(const FPart &fp, uint32_t pin_iv, Perm &r) {
  if (pin_iv <= 1) {
    r = {0, pin_iv, 1};
    return true;
  }
  auto it = fp.pin2pos.find(pin_iv >> 1);
  if (it == fp.pin2pos.end()) return false;
  r = {it->second, pin_iv & 1, 0};
  return true;
}
static void place_sd(FPart &fp, uint32_t pos, const Perm &p) {
  fp.sd_perm[pos] = p.perm;
  set_bit(fp.sd_inv[pos >> 5], pos & 31, p.inv);
  set_bit(fp.sd_set0[pos >> 5], pos & 31, p.set0);
}
static void place_ck(FPart &fp, uint32_t pos, const Perm &p, uint32_t dinv) {
  fp.ck_perm[pos] = p.perm;
  set_bit(fp.ck_inv[pos >> 5], pos & 31, p.inv);
  set_bit(fp.ck_set0[pos >> 5], pos & 31, p.set0);
  set_bit(fp.d_inv[pos >> 5], pos & 31, dinv);
}

// src/flatten.rs:602-661 get_or_place_output_with_activation
static bool get_or_place(FPart &fp, uint32_t pin_iv, uint32_t clken_iv, uint32_t &out,
                         std::string *err) {
  auto it = fp.acts_idx.find(pin_iv >> 1);
  if (it == fp.acts_idx.end()) { if (err) *err = "activation missing"; return false; }
  auto &v = fp.acts[it->second].second;
  uint32_t key = clken_iv << 1 | (pin_iv & 1);
  size_t ai = 0;
  for (; ai < v.size(); ++ai)
    if (v[ai].first == key) break;
  if (ai == v.size()) { if (err) *err = "activation key missing"; return false; }
  if (v[ai].second >= 0) { out = (uint32_t)v[ai].second; return true; }
  Perm ck;
  if (!query_perm(fp, clken_iv, ck)) { if (err) *err = "clock enable not written out"; return false; }
  auto op = fp.pin2pos.find(pin_iv >> 1);
  if (op == fp.pin2pos.end()) { if (err) *err = "endpoint pin not written out"; return false; }
  uint32_t origpos = op->second;
  uint32_t r;
  if (ai == 0) {
    place_ck(fp, origpos, ck, pin_iv & 1);
    r = origpos;
  } else {
    fp.cnt_dup++;
    uint32_t dup_pos = (fp.num_writeouts - fp.num_srams) * 32 - fp.cnt_dup;
    uint32_t dup_perm_pos = (fp.num_srams * 4 + fp.num_dup) * 32 - fp.cnt_dup;
    if (dup_perm_pos >= 8192) { if (err) *err = "duplicate overflow"; return false; }
    place_sd(fp, dup_perm_pos, Perm{(uint16_t)origpos, 0, 0});
    place_ck(fp, dup_pos, ck, pin_iv & 1);
    r = dup_pos;
  }
  v[ai].second = (int32_t)r;
  out = r;
  return true;
}

bool flatten_script(const AIG &g, const std::vector<StagedAIG> &stageds,
                    const std::vector<std::vector<Partition>> &parts_in,
                    const FlattenOptions &opt, FlatScript &out, std::string *err) {
  out = FlatScript();
  const size_t nb = opt.num_blocks;
  out.num_blocks = nb;
  out.num_major_stages = stageds.size();
  out.input_layout = g.input_layout();
  OrderedMap<uint32_t, uint32_t> input_map, output_map, staged_io_map;
  for (size_t i = 0; i < out.input_layout.size(); ++i)
    input_map.insert(out.input_layout[i], (uint32_t)i);
  const uint32_t const_zero_pos = (uint32_t)out.input_layout.size();
  uint32_t states_start = (uint32_t)((out.input_layout.size() + 31) / 32);
  if (const_zero_pos == states_start * 32) states_start += 1;
  uint32_t sum_state = states_start, sum_sram = 0;

  // drop partitions without stages (constant-only endpoints); they still
  // contribute their constant mappings below.
  std::vector<std::vector<const Partition *>> parts(stageds.size());
  std::vector<std::vector<const Partition *>> zero_parts(stageds.size());
  for (size_t s = 0; s < stageds.size(); ++s)
    for (const Partition &p : parts_in[s])
      (p.stages.empty() ? zero_parts[s] : parts[s]).push_back(&p);

  std::vector<std::vector<FPart>> fparts(stageds.size());
  for (size_t s = 0; s < stageds.size(); ++s) {
    auto &P = parts[s];
    // masonry layout onto blocks (src/flatten.rs:1206-1226), parts sorted by
    // decreasing #stages, executor fixed cost 3
    std::stable_sort(P.begin(), P.end(), [](const Partition *a, const Partition *b) {
      return a->stages.size() > b->stages.size();
    });
    std::vector<std::vector<uint32_t>> bp(nb);
    std::vector<size_t> cost(nb, 0);
    const size_t fixed = 3;
    for (size_t i = 0; i < P.size() && i < nb; ++i) {
      bp[i].push_back((uint32_t)i);
      cost[i] = P[i]->stages.size() + fixed;
    }
    for (size_t i = nb; i < P.size(); ++i) {
      size_t put = std::min_element(cost.begin(), cost.end()) - cost.begin();
      bp[put].push_back((uint32_t)i);
      cost[put] += P[i]->stages.size() + fixed;
    }
    auto &F = fparts[s];
    F.resize(P.size());
    for (size_t i = 0; i < P.size(); ++i) init_part(g, stageds[s], *P[i], F[i]);
    for (auto &blk : bp)
      for (uint32_t pid : blk) {
        F[pid].state_start = sum_state;
        sum_state += F[pid].num_writeouts;
        F[pid].sram_start = sum_sram;
        sum_sram += F[pid].num_srams * SRAM_WORDS;
      }
    // make_inputs_outputs (src/flatten.rs:663-858)
    size_t nso = stageds[s].staged_outputs.size();
    size_t npo = g.primary_outputs.size(), ndf = g.dffs.size();
    for (const Partition *zp : zero_parts[s]) {
      for (uint32_t e : zp->endpoints) {
        if (e < nso) continue;
        size_t o = stageds[s].endpoints[e - nso];
        if (o < npo) {
          if (g.primary_outputs[o] <= 1) output_map.insert(g.primary_outputs[o], 0);
        } else if (o < npo + ndf) {
          const DFF &d = g.dffs[o - npo];
          if (d.d_iv <= 1) input_map.insert(d.q, const_zero_pos);
        }
      }
    }
    for (size_t pid = 0; pid < P.size(); ++pid) {
      FPart &fp = F[pid];
      fp.sd_perm.assign(8192, 0);
      fp.sd_inv.assign(NT, 0);
      fp.sd_set0.assign(NT, 0xffffffffu);
      fp.ck_perm.assign(8192, 0);
      fp.ck_inv.assign(NT, 0);
      fp.ck_set0.assign(NT, 0xffffffffu);
      fp.d_inv.assign(NT, 0);
      fp.cnt_dup = 0;
      uint32_t cur_sram = 0;
      for (uint32_t e : P[pid]->endpoints) {
        uint32_t pos;
        if (e < nso) {
          uint32_t idx = stageds[s].staged_outputs[e];
          if (!get_or_place(fp, idx << 1, 1, pos, err)) return false;
          staged_io_map.insert(idx, fp.state_start * 32 + pos);
          continue;
        }
        size_t o = stageds[s].endpoints[e - nso];
        if (o < npo) {
          uint32_t iv = g.primary_outputs[o];
          if (iv <= 1) { output_map.insert(iv, 0); continue; }
          if (!get_or_place(fp, iv, 1, pos, err)) return false;
          output_map.insert(iv, fp.state_start * 32 + pos);
        } else if (o < npo + ndf) {
          const DFF &d = g.dffs[o - npo];
          if (d.d_iv <= 1) { input_map.insert(d.q, const_zero_pos); continue; }
          if (!get_or_place(fp, d.d_iv, d.en_iv, pos, err)) return false;
          output_map.insert(d.d_iv, fp.state_start * 32 + pos);
          input_map.insert(d.q, fp.state_start * 32 + pos);
        } else {
          const RAMBlock &ram = g.srams[o - npo - ndf];
          uint32_t local = fp.num_writeouts - fp.num_srams + cur_sram;
          uint32_t glob = fp.state_start + local;
          Perm ren;
          if (!query_perm(fp, ram.r_en_iv, ren)) { if (err) *err = "sram r_en not written out"; return false; }
          for (int k = 0; k < 32; ++k) {
            uint32_t d = ram.r_data[k];
            if (d == NONE) continue;
            input_map.insert(d, glob * 32 + k);
            output_map.insert(d << 1, glob * 32 + k);
            place_ck(fp, local * 32 + k, ren, 0);
          }
          uint32_t st0 = cur_sram * 128;
          for (int k = 0; k < SRAM_ADDR_BITS; ++k) {
            Perm pr, pw;
            if (!query_perm(fp, ram.r_addr_iv[k], pr) || !query_perm(fp, ram.w_addr_iv[k], pw)) {
              if (err) *err = "sram address not written out";
              return false;
            }
            place_sd(fp, st0 + k, pr);
            place_sd(fp, st0 + 16 + k, pw);
          }
          for (int k = 0; k < 32; ++k) {
            Perm pe, pd;
            if (!query_perm(fp, ram.w_en_iv[k], pe) || !query_perm(fp, ram.w_data_iv[k], pd)) {
              if (err) *err = "sram write port not written out";
              return false;
            }
            place_sd(fp, st0 + 32 + k, pe);
            place_sd(fp, st0 + 64 + k, pd);
          }
          cur_sram++;
        }
      }
      if ((fp.cnt_dup + 31) / 32 != fp.num_dup) { if (err) *err = "duplicate count mismatch"; return false; }
    }
    out.stages_blocks_parts.push_back({});
    for (auto &blk : bp) out.stages_blocks_parts.back().push_back(blk);
  }

  // ---- per-partition scripts (src/flatten.rs:863-1130) and block assembly
  std::vector<std::vector<uint8_t>> xflag(stageds.size());
  std::vector<uint8_t> xpins;
  if (opt.xprop) xpins = g.x_capable_pins();
  for (size_t s = 0; s < stageds.size(); ++s) {
    auto &P = parts[s];
    auto &F = fparts[s];
    std::vector<std::vector<uint32_t>> scripts(P.size());
    std::vector<std::vector<std::pair<size_t, std::vector<uint32_t>>>> patches(P.size());
    for (size_t pid = 0; pid < P.size(); ++pid) {
      const Partition &p = *P[pid];
      FPart &fp = F[pid];
      std::vector<uint32_t> &sc = scripts[pid];
      sc.reserve(256 + 512 * 4 + 5120 * (p.stages.size() + 2));
      sc.push_back((uint32_t)p.stages.size());
      sc.push_back(0);
      sc.push_back(fp.num_writeouts);
      sc.push_back(fp.state_start);
      sc.push_back(fp.num_srams);
      sc.push_back(fp.sram_start);
      sc.push_back(0);
      sc.push_back(fp.num_dup);
      while (sc.size() < 128) sc.push_back(0);
      uint32_t last_wo = NONE;
      for (size_t j = 0; j < p.stages.size(); ++j)
        for (uint16_t wo : p.stages[j].write_outs) {
          uint32_t cur = (uint32_t)j << 8 | wo;
          if (last_wo == NONE) last_wo = cur;
          else { sc.push_back(last_wo | cur << 16); last_wo = NONE; }
        }
      if (last_wo != NONE) sc.push_back(last_wo | 0xffffu << 16);
      if (sc.size() > 256) { if (err) *err = "too many writeout hooks"; return false; }
      while (sc.size() < 256) sc.push_back(0xffffffffu);
      // global read of stage-0 inputs
      std::map<uint32_t, uint32_t> taken;
      auto pos_of = [&](uint32_t pin, bool &staged, uint32_t &pos) -> bool {
        if (const uint32_t *q = input_map.get(pin)) { staged = false; pos = *q; return true; }
        if (const uint32_t *q = staged_io_map.get(pin)) { staged = true; pos = *q; return true; }
        return false;
      };
      for (uint32_t pin : p.stages[0].hier[0]) {
        if (pin == NONE) continue;
        bool stg;
        uint32_t pos;
        if (!pos_of(pin, stg, pos)) { if (err) *err = "stage-0 input not in the state"; return false; }
        uint32_t key = (pos >> 5) | (stg ? 0x80000000u : 0u);
        taken[key] |= 1u << (pos & 31);
      }
      std::vector<std::pair<uint32_t, uint32_t>> tv(taken.begin(), taken.end());
      std::vector<std::vector<std::pair<uint32_t, uint32_t>>> rounds;
      if (!map_rounds(tv, rounds)) { if (err) *err = "global read does not fit"; return false; }
      uint32_t R = 0;
      for (auto &v : rounds) R = std::max(R, (uint32_t)v.size());
      sc[6] = R;
      size_t gp = sc.size();
      sc.resize(gp + 2 * (size_t)R * NT, 0);
      for (uint32_t i = 0; i < NT; ++i)
        for (size_t r = 0; r < rounds[i].size(); ++r) {
          sc[gp + NT * 2 * r + i * 2] = rounds[i][r].first;
          sc[gp + NT * 2 * r + i * 2 + 1] = rounds[i][r].second;
        }
      // (staged, word<<5|bit) -> local bit position; bits enter LSB-last
      std::unordered_map<uint64_t, uint16_t> op2lp;
      for (uint32_t i = 0; i < NT; ++i) {
        uint32_t bit_id = 0;
        for (auto it = rounds[i].rbegin(); it != rounds[i].rend(); ++it) {
          bool stg = (it->first >> 31) != 0;
          for (int k = 31; k >= 0; --k)
            if ((it->second >> k) & 1) {
              uint64_t key = (uint64_t)stg << 32 | (uint32_t)((it->first << 5) | (uint32_t)k);
              op2lp[key] = (uint16_t)(i * 32 + bit_id);
              bit_id++;
            }
        }
      }
      std::unordered_map<uint32_t, uint16_t> last_pos;
      for (uint32_t pin : p.stages[0].hier[0]) {
        if (pin == NONE) continue;
        bool stg = false;
        uint32_t pos = 0;
        pos_of(pin, stg, pos);
        last_pos[pin] = op2lp.at((uint64_t)stg << 32 | pos);
      }
      for (size_t bs = 0; bs < p.stages.size(); ++bs) {
        const BoomStage &S = p.stages[bs];
        std::vector<uint16_t> perm(8192, 0);
        for (uint32_t j = 0; j < 8192; ++j) {
          uint32_t pin = S.hier[0][j];
          if (pin == NONE) continue;
          auto it = last_pos.find(pin);
          if (it == last_pos.end()) { if (err) *err = "stage input not produced by previous stage"; return false; }
          perm[j] = it->second;
        }
        std::vector<uint32_t> xa(NT, 0), xb(NT, 0), ob(NT, 0);
        std::vector<std::vector<uint32_t>> tpins(NT);
        for (int hi = 1; hi <= BOOM_STAGES; ++hi) {
          uint32_t hl = lvl_len(hi);
          for (uint32_t j = 0; j < hl; ++j) {
            uint32_t o = S.hier[hi][j];
            if (o == NONE) continue;
            uint32_t posn = hl + j;
            tpins[posn >> 5].push_back(o);
            uint32_t a = S.hier[hi - 1][j], b = S.hier[hi - 1][j + hl];
            if (o == a) { ob[posn >> 5] |= 1u << (posn & 31); continue; }
            if (g.kind[o] != DRV_AND || (g.fa[o] >> 1) != a || (g.fb[o] >> 1) != b) {
              if (err) *err = "boomerang slot is neither pass-through nor its AND";
              return false;
            }
            if (g.fa[o] & 1) xa[posn >> 5] |= 1u << (posn & 31);
            if (g.fb[o] & 1) xb[posn >> 5] |= 1u << (posn & 31);
          }
        }
        for (int k = 0; k < 4; ++k)
          for (uint32_t i = k * 8; i < 8192; i += 32)
            for (int q = 0; q < 8; q += 2) sc.push_back((uint32_t)perm[i + q] | (uint32_t)perm[i + q + 1] << 16);
        for (uint32_t i = 0; i < NT; ++i) {
          sc.push_back(xa[i]);
          sc.push_back(xb[i]);
          sc.push_back(ob[i]);
          size_t off = sc.size();
          sc.push_back(0);  // padding: gate delay, patched by inject_timing
          if (!tpins[i].empty()) patches[pid].push_back({off, std::move(tpins[i])});
        }
        last_pos.clear();
        const auto &after = fp.afters[bs];
        for (uint32_t i = 0; i < 8192; ++i)
          if (after[i] != NONE) last_pos[after[i]] = (uint16_t)i;
      }
      for (int k = 0; k < 4; ++k)
        for (uint32_t i = k * 8; i < 8192; i += 32)
          for (int q = 0; q < 8; q += 2) sc.push_back((uint32_t)fp.sd_perm[i + q] | (uint32_t)fp.sd_perm[i + q + 1] << 16);
      for (uint32_t i = 0; i < NT; ++i) {
        sc.push_back(fp.sd_inv[i]);
        sc.push_back(fp.sd_set0[i]);
        sc.push_back(0);
        sc.push_back(0);
      }
      for (int k = 0; k < 4; ++k)
        for (uint32_t i = k * 8; i < 8192; i += 32)
          for (int q = 0; q < 8; q += 2) sc.push_back((uint32_t)fp.ck_perm[i + q] | (uint32_t)fp.ck_perm[i + q + 1] << 16);
      for (uint32_t i = 0; i < NT; ++i) {
        sc.push_back(fp.ck_inv[i]);
        sc.push_back(fp.ck_set0[i]);
        sc.push_back(fp.d_inv[i]);
        sc.push_back(0);
      }
    }
    // X capability: any pin of the partition X-capable
    if (opt.xprop) {
      xflag[s].assign(P.size(), 0);
      for (size_t pid = 0; pid < P.size(); ++pid) {
        bool x = false;
        for (const BoomStage &S : P[pid]->stages) {
          for (int l = 0; l <= BOOM_STAGES && !x; ++l)
            for (uint32_t pin : S.hier[l])
              if (pin != NONE && pin < xpins.size() && xpins[pin]) { x = true; break; }
          if (x) break;
        }
        xflag[s][pid] = x;
      }
    }
    // assemble blocks
    const auto &bp = out.stages_blocks_parts[s];
    for (size_t b = 0; b < nb; ++b) {
      out.blocks_start.push_back(out.blocks_data.size());
      if (bp[b].empty()) {
        std::vector<uint32_t> dummy(NT, 0);
        dummy[1] = 1;
        out.blocks_data.insert(out.blocks_data.end(), dummy.begin(), dummy.end());
        continue;
      }
      size_t last_st = 0;
      for (uint32_t pid : bp[b]) {
        last_st = out.blocks_data.size();
        size_t base = last_st;
        out.blocks_data.insert(out.blocks_data.end(), scripts[pid].begin(), scripts[pid].end());
        for (auto &pp : patches[pid]) {
          out.delay_patch_offset.push_back(base + pp.first);
          out.delay_patch_pins_start.push_back((uint32_t)out.delay_patch_pins.size());
          out.delay_patch_pins.insert(out.delay_patch_pins.end(), pp.second.begin(), pp.second.end());
        }
      }
      out.blocks_data[last_st + 1] = 1;
    }
  }
  out.delay_patch_pins_start.push_back((uint32_t)out.delay_patch_pins.size());
  out.blocks_start.push_back(out.blocks_data.size());
  out.blocks_data.insert(out.blocks_data.end(), NT * 8, 0);
  out.reg_io_state_size = sum_state;
  out.sram_storage_size = sum_sram;
  out.input_map = input_map.items;
  out.output_map = output_map.items;
  out.staged_io_map = staged_io_map.items;

  // ---- X-propagation classification and metadata words 8/9
  // (src/flatten.rs:1419-1543).  The inter-partition fixpoint looks each
  // stage's input pins up in the output map the way the reference does,
  // i.e. using the pin number as the map key.
  out.xprop_enabled = opt.xprop;
  out.xprop_state_offset = sum_state;
  if (opt.xprop) {
    struct Range { uint32_t lo, hi; size_t s, pid; };
    for (;;) {
      std::vector<Range> xr;
      for (size_t s = 0; s < stageds.size(); ++s)
        for (size_t pid = 0; pid < parts[s].size(); ++pid)
          if (xflag[s][pid]) xr.push_back({fparts[s][pid].state_start,
                                           fparts[s][pid].state_start + fparts[s][pid].num_writeouts, s, pid});
      std::sort(xr.begin(), xr.end(), [](const Range &a, const Range &b) { return a.lo < b.lo; });
      auto in_x = [&](uint32_t w) {
        auto it = std::upper_bound(xr.begin(), xr.end(), w, [](uint32_t v, const Range &r) { return v < r.lo; });
        if (it == xr.begin()) return false;
        --it;
        return w >= it->lo && w < it->hi;
      };
      bool changed = false;
      for (size_t s = 0; s < stageds.size(); ++s)
        for (size_t pid = 0; pid < parts[s].size(); ++pid) {
          if (xflag[s][pid]) continue;
          bool hit = false;
          for (const BoomStage &S : parts[s][pid]->stages) {
            for (uint32_t pin : S.hier[0]) {
              if (pin == NONE) continue;
              const uint32_t *q = output_map.get(pin);
              if (q && in_x(*q >> 5)) { hit = true; break; }
            }
            if (hit) break;
          }
          if (hit) { xflag[s][pid] = 1; changed = true; }
        }
      if (!changed) break;
    }
  }
  for (size_t s = 0; s < stageds.size(); ++s) {
    const auto &bp = out.stages_blocks_parts[s];
    for (size_t b = 0; b < nb; ++b) {
      size_t off = out.blocks_start[s * nb + b];
      for (uint32_t pid : bp[b]) {
        out.part_ptrs.push_back(parts[s][pid]);
        out.part_major_stage.push_back((uint32_t)s);
        uint8_t x = opt.xprop ? xflag[s][pid] : 0;
        if (opt.xprop) {
          out.blocks_data[off + 8] = x;
          out.blocks_data[off + 9] = out.xprop_state_offset;
        }
        out.partition_x_capable.push_back(x);
        out.part_num_stages.push_back(out.blocks_data[off]);
        size_t ns = out.blocks_data[off], R = out.blocks_data[off + 6];
        off += NT + 2 * R * NT + ns * 5120 + 2 * 5120;
      }
    }
  }
  // DFF data positions (for the constraint buffer)
  out.dff_data_pos.resize(g.dffs.size());
  for (size_t i = 0; i < g.dffs.size(); ++i) {
    const uint32_t *q = output_map.get(g.dffs[i].d_iv);
    out.dff_data_pos[i] = q ? *q : NONE;
  }
  return true;
}

void inject_timing(FlatScript &s, const std::vector<uint32_t> &rise,
                   const std::vector<uint32_t> &fall) {
  // src/flatten.rs:1812-1846: max over the position's pins of max(rise,fall),
  // clamped to u16.
  for (size_t i = 0; i < s.delay_patch_offset.size(); ++i) {
    uint32_t m = 0;
    for (uint32_t k = s.delay_patch_pins_start[i]; k < s.delay_patch_pins_start[i + 1]; ++k) {
      uint32_t p = s.delay_patch_pins[k];
      if (p < rise.size()) m = std::max(m, std::max(rise[p], fall[p]));
    }
    if (m > 65535) m = 65535;
    if (s.delay_patch_offset[i] < s.blocks_data.size()) s.blocks_data[s.delay_patch_offset[i]] = m;
  }
}

}  // namespace jq
