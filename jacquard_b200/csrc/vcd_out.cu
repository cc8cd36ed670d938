// Per-snapshot walks over the resident snapshots of a run, compacted on the
// device in (snapshot, signal) order, so the host only formats results:
// - output transitions for the waveform writers (src/sim/vcd_io.rs:758-946
//   walk every output of every snapshot on the host and keep the changes):
//   each output is encoded (0, 1, or 3 for X) and compared with the previous
//   snapshot's code (2 before the first);
// - set bits for the display / assertion post-scan
//   (src/bin/jacquard.rs:1152-1253 probe every condition bit of every
//   snapshot on the host): a condition fires where its bit is 1.
#include "sim_common.cuh"

namespace jqk {

constexpr int OT = 256;  // threads per block

struct TransParams {
  const uint32_t *states;   // snapshot s of the walk starts at states + (first + s) * stride
  size_t first, num, stride;
  size_t xmask_offset;      // words from a value word to its X word, 0 = no X
  size_t arrival_offset;    // words from a value word to its arrival word, 0 = none
  const uint32_t *out_pos;  // state bit position of each output, or ~0u for a constant
  const uint32_t *out_const;  // value of constant outputs (may be null: 0)
  uint32_t n_out;
  int set_bits;               // 1: report set bits instead of transitions
};

__device__ __forceinline__ uint32_t out_code(const TransParams &P, size_t s, uint32_t j) {
  const uint32_t pos = P.out_pos[j];
  if (pos == 0xffffffffu) return P.out_const ? (P.out_const[j] & 1u) : 0u;
  const uint32_t *snap = P.states + (P.first + s) * P.stride;
  const size_t w = pos >> 5;
  const uint32_t v = (snap[w] >> (pos & 31)) & 1u;
  if (P.xmask_offset && ((snap[P.xmask_offset + w] >> (pos & 31)) & 1u)) return 3u;
  return v;
}

__device__ __forceinline__ bool changed(const TransParams &P, size_t s, uint32_t j, uint32_t &code) {
  code = out_code(P, s, j);
  if (P.set_bits) return code == 1u;
  const uint32_t prev = s == 0 ? 2u : out_code(P, s - 1, j);
  return code != prev;
}

__global__ void __launch_bounds__(OT) trans_count_kernel(TransParams P, uint32_t *counts) {
  for (size_t s = blockIdx.x; s < P.num; s += gridDim.x) {
    uint32_t n = 0;
    for (uint32_t j0 = 0; j0 < P.n_out; j0 += OT) {
      const uint32_t j = j0 + threadIdx.x;
      uint32_t code;
      const bool c = j < P.n_out && changed(P, s, j, code);
      n += (uint32_t)__syncthreads_count(c);
    }
    if (threadIdx.x == 0) counts[s] = n;
  }
}

// Exclusive scan of counts into offsets (one block, chunks of OT), total last.
__global__ void __launch_bounds__(OT) trans_scan_kernel(const uint32_t *counts, size_t n,
                                                        unsigned long long *offsets) {
  __shared__ unsigned long long part[OT];
  unsigned long long carry = 0;
  for (size_t c0 = 0; c0 < n; c0 += OT) {
    const size_t i = c0 + threadIdx.x;
    const unsigned long long v = i < n ? counts[i] : 0ull;
    part[threadIdx.x] = v;
    __syncthreads();
    for (int d = 1; d < OT; d <<= 1) {
      const unsigned long long add = threadIdx.x >= (unsigned)d ? part[threadIdx.x - d] : 0ull;
      __syncthreads();
      part[threadIdx.x] += add;
      __syncthreads();
    }
    if (i < n) offsets[i] = carry + part[threadIdx.x] - v;
    const unsigned long long chunk = part[OT - 1];
    __syncthreads();
    carry += chunk;
  }
  if (threadIdx.x == 0) offsets[n] = carry;
}

__global__ void __launch_bounds__(OT) trans_write_kernel(TransParams P,
                                                         const unsigned long long *offsets,
                                                         uint32_t *trans, uint32_t *arrivals,
                                                         size_t capacity) {
  __shared__ uint32_t warp_n[OT / 32];
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (size_t s = blockIdx.x; s < P.num; s += gridDim.x) {
    unsigned long long base = offsets[s];
    for (uint32_t j0 = 0; j0 < P.n_out; j0 += OT) {
      const uint32_t j = j0 + threadIdx.x;
      uint32_t code = 0;
      const bool c = j < P.n_out && changed(P, s, j, code);
      const uint32_t ball = __ballot_sync(0xffffffffu, c);
      if (lane == 0) warp_n[warp] = __popc(ball);
      __syncthreads();
      uint32_t before = 0, total = 0;
      for (uint32_t w = 0; w < OT / 32; ++w) {
        if (w < warp) before += warp_n[w];
        total += warp_n[w];
      }
      const unsigned long long k = base + before + __popc(ball & ((1u << lane) - 1u));
      if (c && k < capacity) {
        trans[k] = j | (code << 30);
        if (arrivals) {
          const uint32_t pos = P.out_pos[j];
          arrivals[k] = (pos == 0xffffffffu || !P.arrival_offset)
                            ? 0u
                            : (P.states[(P.first + s) * P.stride + P.arrival_offset + (pos >> 5)] &
                               0xffffu);
        }
      }
      base += total;
      __syncthreads();
    }
  }
}

}  // namespace jqk

using namespace jqk;

static int run_walk(TransParams P, uint32_t *counts, unsigned long long *offsets,
                    uint32_t *transitions, uint32_t *arrivals, size_t capacity, size_t *total,
                    void *stream) {
  cudaStream_t st = (cudaStream_t)stream;
  *total = 0;
  if (P.num == 0) return JQ_OK;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const unsigned grid = (unsigned)(P.num < (size_t)sms * 8 ? P.num : (size_t)sms * 8);
  trans_count_kernel<<<grid, OT, 0, st>>>(P, counts);
  trans_scan_kernel<<<1, OT, 0, st>>>(counts, P.num, offsets);
  if (capacity) trans_write_kernel<<<grid, OT, 0, st>>>(P, offsets, transitions, arrivals, capacity);
  if (cudaGetLastError() != cudaSuccess) return JQ_ERR_LAUNCH;
  unsigned long long t = 0;
  if (cudaMemcpyAsync(&t, offsets + P.num, sizeof(t), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return JQ_ERR_CUDA;
  *total = (size_t)t;
  return t > capacity ? JQ_ERR_EVENT_OVERFLOW : JQ_OK;
}

extern "C" int jq_output_transitions(const uint32_t *states, size_t first_snapshot,
                                     size_t num_snapshots, size_t snapshot_words,
                                     size_t xmask_offset, size_t arrival_offset,
                                     const uint32_t *out_pos, const uint32_t *out_const,
                                     uint32_t n_out, uint32_t *counts,
                                     unsigned long long *offsets, uint32_t *transitions,
                                     uint32_t *arrivals, size_t capacity, size_t *total,
                                     void *stream) {
  if (!states || !out_pos || !counts || !offsets || !total || snapshot_words == 0 || n_out == 0 ||
      n_out >= (1u << 30) || (capacity && !transitions))
    return JQ_ERR_INVALID_ARG;
  TransParams P{states, first_snapshot, num_snapshots, snapshot_words, xmask_offset,
                arrival_offset, out_pos, out_const, n_out, 0};
  return run_walk(P, counts, offsets, transitions, arrivals, capacity, total, stream);
}

extern "C" int jq_set_bits(const uint32_t *states, size_t first_snapshot, size_t num_snapshots,
                           size_t snapshot_words, const uint32_t *bit_pos, uint32_t n_bits,
                           uint32_t *counts, unsigned long long *offsets, uint32_t *hits,
                           size_t capacity, size_t *total, void *stream) {
  if (!states || !bit_pos || !counts || !offsets || !total || snapshot_words == 0 || n_bits == 0 ||
      n_bits >= (1u << 30) || (capacity && !hits))
    return JQ_ERR_INVALID_ARG;
  TransParams P{states, first_snapshot, num_snapshots, snapshot_words, 0, 0, bit_pos, nullptr,
                n_bits, 1};
  return run_walk(P, counts, offsets, hits, nullptr, capacity, total, stream);
}
