// Partition features and host-side inference of the learned cost model.
#include <cmath>
#include <algorithm>
#include <cstring>

#include "frontend.hpp"

namespace jq {

void partition_features(const AIG &g, const StagedAIG &st, const Partition &p,
                        const std::vector<uint8_t> *xpins, float *f) {
  std::memset(f, 0, sizeof(float) * NFEAT);
  const float ns = (float)p.stages.size();
  uint64_t used = 0, pass = 0, ands = 0, used1 = 0, h0 = 0;
  int maxl = 0;
  bool isx = false;
  std::vector<uint32_t> ins;
  for (size_t si = 0; si < p.stages.size(); ++si) {
    const BoomStage &S = p.stages[si];
    for (uint32_t pin : S.hier[0])
      if (pin != NONE) {
        ++h0;
        if (si == 0) ins.push_back(pin);
        if (xpins && pin < xpins->size() && (*xpins)[pin]) isx = true;
      }
    for (int l = 1; l <= BOOM_STAGES; ++l) {
      const uint32_t len = 8192u >> l;
      for (uint32_t j = 0; j < len; ++j) {
        uint32_t o = S.hier[l][j];
        if (o == NONE) continue;
        ++used;
        if (l == 1) ++used1;
        if (xpins && o < xpins->size() && (*xpins)[o]) isx = true;
        if (o == S.hier[l - 1][j]) ++pass;
        else { ++ands; if (l > maxl) maxl = l; }
      }
    }
  }
  std::sort(ins.begin(), ins.end());
  ins.erase(std::unique(ins.begin(), ins.end()), ins.end());
  uint32_t staged_in = 0;
  for (uint32_t pin : ins)
    if (st.has_staged_inputs && st.is_staged_input[pin]) ++staged_in;
  uint32_t wos = 0;
  for (const BoomStage &S : p.stages) wos += (uint32_t)S.write_outs.size();
  uint32_t n_sram = 0, n_staged_ep = 0;
  size_t nso = st.staged_outputs.size(), npo = g.primary_outputs.size(), nd = g.dffs.size();
  for (uint32_t e : p.endpoints) {
    if (e < nso) { ++n_staged_ep; continue; }
    size_t o = st.endpoints[e - nso];
    if (o >= npo + nd) ++n_sram;
  }
  // distinct pins at level >= 1 over all stages
  std::vector<uint32_t> vis;
  for (const BoomStage &S : p.stages)
    for (int l = 1; l <= BOOM_STAGES; ++l)
      for (uint32_t o : S.hier[l])
        if (o != NONE) vis.push_back(o);
  std::sort(vis.begin(), vis.end());
  vis.erase(std::unique(vis.begin(), vis.end()), vis.end());
  const float R = std::ceil((float)ins.size() / 256.0f);
  f[0] = ns;
  f[1] = (float)p.cone_ands;
  f[2] = (float)p.targets;
  f[3] = (float)p.endpoints.size();
  f[4] = (float)ins.size();
  f[5] = (float)staged_in;
  f[6] = (float)wos;
  f[7] = (float)n_sram;
  f[8] = (float)(p.endpoints.size() - n_sram > p.targets ? p.endpoints.size() - n_sram - p.targets : 0);
  f[9] = isx ? 1.f : 0.f;
  f[10] = (float)used;
  f[11] = (float)pass;
  f[12] = (float)ands;
  f[13] = (float)used1;
  f[14] = (float)maxl;
  f[15] = (float)h0;
  f[16] = (float)ands / (float)std::max<uint32_t>(1, p.cone_ands);
  f[17] = 256.f + 512.f * R + 5120.f * (ns + 2.f);
  f[18] = ns > 0 ? (float)used / (ns * 8191.f) : 0.f;
  f[19] = std::log2(1.f + (float)p.cone_ands);
  f[20] = std::log2(1.f + (float)p.targets);
  f[21] = std::log2(1.f + (float)ins.size());
  f[22] = p.endpoints.empty() ? 0.f : (float)n_staged_ep / (float)p.endpoints.size();
  f[23] = (float)vis.size();
}

static inline float bf16_round(float x) {
  uint32_t u;
  std::memcpy(&u, &x, 4);
  if ((u & 0x7f800000u) == 0x7f800000u) return x;  // inf / nan unchanged
  u += 0x7fffu + ((u >> 16) & 1u);                  // round to nearest even
  u &= 0xffff0000u;
  std::memcpy(&x, &u, 4);
  return x;
}

float CostModel::predict(const float *feat) const {
  float x[NFEAT], h1[128], h2[128];
  for (int i = 0; i < NFEAT; ++i) x[i] = bf16_round((feat[i] - mean[i]) * inv_std[i]);
  for (int o = 0; o < 128; ++o) {
    float a = b1[o];
    for (int i = 0; i < NFEAT; ++i) a += bf16_round(w1[o * NFEAT + i]) * x[i];
    h1[o] = bf16_round(a > 0 ? a : 0);
  }
  for (int o = 0; o < 128; ++o) {
    float a = b2[o];
    for (int i = 0; i < 128; ++i) a += bf16_round(w2[o * 128 + i]) * h1[i];
    h2[o] = bf16_round(a > 0 ? a : 0);
  }
  float y = b3;
  for (int i = 0; i < 128; ++i) y += bf16_round(w3[i]) * h2[i];
  return y;
}

}  // namespace jq
