// RepCut hypergraph build on the device (src/repcut.rs:58-176,
// RCHyperGraph::from_staged_aig: the reference builds it on the host with
// Rayon; it is the front end's documented bottleneck).
//
// For each block of 4096 endpoint groups every pin gets a 4096-bit endpoint
// set (64 words).  It is seeded with the endpoints whose inputs include the
// pin and filled from fanouts to fanins in reverse-level order, one warp per
// pin with two words per lane, within the block's cone (the reference's
// traversal does not descend through the slice's staged inputs).  As each pin's
// block set becomes final it is folded into a per-pin popcount and a 128-bit
// fingerprint (two independent 64-bit hashes, block-salted), so equal
// endpoint sets give equal fingerprints.  Grouping pins by fingerprint gives
// the reference's clusters.  Node and endpoint weights follow the
// reference's f32 arithmetic exactly (round-to-nearest divides and adds, no
// contraction).
#include "sim_common.cuh"

namespace jqk {

constexpr uint32_t RC_WORDS = 64;  // 4096 bits (REPCUT_BITSET_BLOCK_SIZE)

__device__ __forceinline__ uint64_t rc_mix(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

// Seed: endpoint e in [b0, b1) sets its bit on each of its input pins.
__global__ void rc_seed_kernel(const uint32_t *ep_start, const uint32_t *ep_pins, uint32_t b0,
                               uint32_t b1, unsigned long long *sets) {
  const uint32_t e = b0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= b1) return;
  const uint32_t bit = e - b0;
  for (uint32_t k = ep_start[e]; k < ep_start[e + 1]; ++k)
    atomicOr(sets + (size_t)ep_pins[k] * RC_WORDS + bit / 64, 1ull << (bit % 64));
}

// One reverse level of one endpoint block.  A pin is in the block's cone
// when an endpoint of the block has it as an input, or a fanout in the cone
// that is not a staged input reaches it (the traversal does not descend
// through staged inputs).  A cone pin's set is its own endpoints' bits OR
// the sets of its fanouts in the cone, staged ones included, as the
// reference ORs every fanout it has already processed; the edges along which
// the reference's traversal order has not yet processed a staged fanout are
// marked in supp_bits.  Pins outside the cone keep an empty set.  The final block set is folded into the pin's popcount and
// fingerprint.
__global__ void rc_level_kernel(const uint32_t *nodes, uint32_t n, const uint32_t *fanout_start,
                                const uint32_t *fanouts, const uint8_t *staged,
                                const uint32_t *supp_bits, unsigned long long *sets,
                                uint8_t *cone, uint32_t block_index, unsigned long long *fp,
                                uint32_t *popcount) {
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= n) return;
  const uint32_t p = nodes[warp];
  unsigned long long *sp = sets + (size_t)p * RC_WORDS;
  unsigned long long w0 = sp[lane], w1 = sp[lane + 32];
  bool in = __any_sync(0xffffffffu, (w0 | w1) != 0);  // seeded
  for (uint32_t k = fanout_start[p]; k < fanout_start[p + 1]; ++k) {
    const uint32_t j = fanouts[k];
    if (!cone[j]) continue;
    if (!staged[j]) in = true;
    if ((supp_bits[k >> 5] >> (k & 31)) & 1u) continue;  // j not yet processed there
    const unsigned long long *sj = sets + (size_t)j * RC_WORDS;
    w0 |= sj[lane];
    w1 |= sj[lane + 32];
  }
  if (!in) return;  // outside this block's cone: no segment, set stays empty
  sp[lane] = w0;
  sp[lane + 32] = w1;
  if (lane == 0) cone[p] = 1;
  const uint64_t salt = 0x9e3779b97f4a7c15ull * ((uint64_t)block_index * RC_WORDS + 1);
  uint64_t h1 = rc_mix(w0 ^ (salt + lane)) ^ rc_mix(w1 ^ (salt + lane + 32));
  uint64_t h2 = rc_mix(w0 * 0xd6e8feb86659fd93ull + lane + 7 * salt) ^
                rc_mix(w1 * 0xd6e8feb86659fd93ull + lane + 32 + 7 * salt);
  uint32_t pc = __popcll(w0) + __popcll(w1);
#pragma unroll
  for (int d = 16; d >= 1; d >>= 1) {
    h1 ^= __shfl_xor_sync(0xffffffffu, h1, d);
    h2 ^= __shfl_xor_sync(0xffffffffu, h2, d);
    pc += __shfl_xor_sync(0xffffffffu, pc, d);
  }
  if (lane == 0) {
    fp[2 * p] = rc_mix(fp[2 * p] ^ h1 ^ (0x632be59bd9b4e019ull * (block_index + 1)));
    fp[2 * p + 1] = rc_mix(fp[2 * p + 1] + h2 + 0x8cb92ba72f3d8dd7ull * (block_index + 1));
    popcount[p] += pc;
  }
}

// Node weights of one forward level (pins in the cone of every endpoint,
// i.e. with a non-empty set in some block; others stay 0).
__global__ void rc_weight_kernel(const uint32_t *nodes, uint32_t n, const uint8_t *kind,
                                 const uint32_t *fa, const uint32_t *fb,
                                 const uint32_t *fanout_start, const uint32_t *popcount,
                                 const uint8_t *wsupp, float *nw) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t p = nodes[i];
  if (popcount[p] == 0) return;
  float w = 1.0f;
  if (kind[p] == 1) {
    const uint32_t a = fa[p] >> 1, b = fb[p] >> 1;
    // a fanin the reference has not yet weighed contributes its initial 0
    const float wa = (wsupp[p] & 1u) ? 0.0f : nw[a], wb = (wsupp[p] & 2u) ? 0.0f : nw[b];
    if (a) w = __fadd_rn(w, __fdiv_rn(wa, (float)(fanout_start[a + 1] - fanout_start[a])));
    if (b) w = __fadd_rn(w, __fdiv_rn(wb, (float)(fanout_start[b + 1] - fanout_start[b])));
  }
  nw[p] = w;
}

__global__ void rc_mark_kernel(const uint32_t *edges, uint32_t n, uint32_t *bits) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) atomicOr(bits + (edges[i] >> 5), 1u << (edges[i] & 31));
}

__global__ void rc_endpoint_weight_kernel(const uint32_t *ep_start, const uint32_t *ep_pins,
                                          uint32_t E, const float *nw, const uint32_t *nfe,
                                          unsigned long long *weight) {
  const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= E) return;
  float tot = 0.0f;
  for (uint32_t k = ep_start[e]; k < ep_start[e + 1]; ++k) {
    const uint32_t p = ep_pins[k];
    tot = __fadd_rn(tot, __fdiv_rn(nw[p], (float)nfe[p]));
  }
  const float r = __fadd_rn(tot, 0.5f);
  const unsigned long long v = r <= 0.0f ? 0ull : (unsigned long long)r;
  weight[e] = v < 1 ? 1 : v;
}

}  // namespace jqk

using namespace jqk;

extern "C" int jq_repcut_build(uint32_t num_pins, const uint8_t *kind, const uint32_t *fa,
                               const uint32_t *fb, const uint32_t *fanout_start,
                               const uint32_t *fanouts, const uint8_t *staged,
                               uint32_t num_endpoints, const uint32_t *ep_start,
                               const uint32_t *ep_pins, const uint32_t *nfe,
                               const uint32_t *rlevel_nodes, const uint32_t *rlevel_start_host,
                               uint32_t num_rlevels, const uint32_t *flevel_nodes,
                               const uint32_t *flevel_start_host, uint32_t num_flevels,
                               const uint32_t *supp_start_host, const uint32_t *supp_edges,
                               const uint8_t *wsupp, uint32_t num_fanouts, uint32_t *supp_bits,
                               unsigned long long *sets, uint8_t *cone,
                               unsigned long long *fingerprint, uint32_t *popcount,
                               float *node_weight, unsigned long long *endpoint_weight,
                               void *stream) {
  if (!kind || !fa || !fb || !fanout_start || !staged || !ep_start || !nfe || !rlevel_nodes ||
      !rlevel_start_host || !flevel_nodes || !flevel_start_host || !supp_start_host ||
      !wsupp || !supp_bits || !sets || !cone || !fingerprint ||
      !popcount || !node_weight || !endpoint_weight)
    return JQ_ERR_INVALID_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  const size_t pins = (size_t)num_pins + 1;
  if (cudaMemsetAsync(fingerprint, 0, pins * 2 * sizeof(unsigned long long), st) != cudaSuccess ||
      cudaMemsetAsync(popcount, 0, pins * sizeof(uint32_t), st) != cudaSuccess ||
      cudaMemsetAsync(node_weight, 0, pins * sizeof(float), st) != cudaSuccess)
    return JQ_ERR_CUDA;
  const uint32_t blocks = (num_endpoints + 4095) / 4096;
  for (uint32_t bi = 0; bi < blocks; ++bi) {
    const uint32_t b0 = bi * 4096, b1 = b0 + 4096 < num_endpoints ? b0 + 4096 : num_endpoints;
    const size_t nbits = ((size_t)num_fanouts + 31) / 32 + 1;
    if (cudaMemsetAsync(sets, 0, pins * RC_WORDS * sizeof(unsigned long long), st) != cudaSuccess ||
        cudaMemsetAsync(cone, 0, pins, st) != cudaSuccess ||
        cudaMemsetAsync(supp_bits, 0, nbits * sizeof(uint32_t), st) != cudaSuccess)
      return JQ_ERR_CUDA;
    const uint32_t ns = supp_start_host[bi + 1] - supp_start_host[bi];
    if (ns)
      rc_mark_kernel<<<(ns + 255) / 256, 256, 0, st>>>(supp_edges + supp_start_host[bi], ns,
                                                       supp_bits);
    rc_seed_kernel<<<(b1 - b0 + 255) / 256, 256, 0, st>>>(ep_start, ep_pins, b0, b1, sets);
    for (uint32_t l = 0; l < num_rlevels; ++l) {
      const uint32_t s0 = rlevel_start_host[l], n = rlevel_start_host[l + 1] - s0;
      if (!n) continue;
      rc_level_kernel<<<(n + 7) / 8, 256, 0, st>>>(rlevel_nodes + s0, n, fanout_start, fanouts,
                                                     staged, supp_bits, sets, cone, bi,
                                                     fingerprint, popcount);
    }
  }
  for (uint32_t l = 0; l < num_flevels; ++l) {
    const uint32_t s0 = flevel_start_host[l], n = flevel_start_host[l + 1] - s0;
    if (!n) continue;
    rc_weight_kernel<<<(n + 255) / 256, 256, 0, st>>>(flevel_nodes + s0, n, kind, fa, fb,
                                                       fanout_start, popcount, wsupp,
                                                       node_weight);
  }
  if (num_endpoints)
    rc_endpoint_weight_kernel<<<(num_endpoints + 255) / 256, 256, 0, st>>>(
        ep_start, ep_pins, num_endpoints, node_weight, nfe, endpoint_weight);
  return cudaGetLastError() == cudaSuccess ? JQ_OK : JQ_ERR_LAUNCH;
}
