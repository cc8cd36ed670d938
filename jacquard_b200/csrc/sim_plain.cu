// Plain interpreter kernel for sm_100a: the reference's script semantics
// (csrc/kernel_v1_impl.cuh:32-626), one stimulus stream, persistent over all
// cycles of a launch with a bounded-wait grid barrier between major stages.
//
// Per (cycle, major stage) each CTA walks its partition list:
//   metadata -> global read (bit gather of state words into 256x32 bits) ->
//   boomerang stages (16-pair shuffle, 8192->1 AND tree, writeout hooks) ->
//   SRAM/duplicate permutation + SRAM port -> clock-enable permutation and
//   DFF commit (+X lanes, +u16 arrivals, +setup/hold events).
// Script chunks are streamed with 16-byte read-only loads, double-buffered in
// registers one stage ahead.  State/SRAM reads bypass L1 (written by other
// SMs between barriers).
//
// Stage depth.  An optional table (jq_plain_prepare) gives, per boomerang
// stage of every partition, the deepest tree level whose outputs anything
// reads (a writeout hook or a needed gather of the next stage): 0 when only
// the first AND level (positions 4096..8191) is read, 1 when nothing below
// position 512 is, 2 otherwise.  Levels whose outputs nobody reads are
// skipped with their CTA barriers; the values that are read are computed as
// before.  The shuffled inputs go to their own buffer (s_in), so a stage
// needs one barrier before its first AND level instead of two.
#include "sim_common.cuh"

namespace jqk {

struct PlainParams {
  unsigned num_blocks, num_major_stages;
  const size_t *blocks_start;
  const uint32_t *blocks_data;
  uint32_t *sram, *sram_x;
  size_t num_cycles, state_size;
  uint32_t *states;
  const uint32_t *constraints;  // [clock, words...] or null
  jq_event_buffer *events;
  uint32_t event_cap;
  int32_t arrival_off;
  uint32_t first_cycle;
  uint64_t timeout;
  int slot;
  const uint8_t *depth;         // stage depth codes, or null (every level runs)
  const uint32_t *depth_base;   // first code of each (major stage, block) entry
};

template <bool TRACK>
__device__ __forceinline__ void run_block(const PlainParams &P, const uint32_t *__restrict__ script,
                                          const uint32_t *in, uint32_t *out, uint32_t cycle,
                                          uint32_t *s_meta, uint32_t *s_st, uint32_t *s_stx,
                                          uint32_t *s_wo, uint32_t *s_wox, uint16_t *s_arr,
                                          uint16_t *s_woarr, uint32_t *s_in, uint32_t *s_inx,
                                          const uint8_t *depth) {
  const int t = threadIdx.x;
  const uint32_t clock_ps = TRACK && P.constraints ? __ldg(P.constraints) : 0;
  const uint32_t *cons = P.constraints ? P.constraints + 1 : nullptr;
  size_t off = 0;
  for (;;) {
    s_meta[t] = __ldg(script + off + t);
    __syncthreads();
    const uint32_t ns = s_meta[0];
    if (!ns) break;
    const uint32_t is_last = s_meta[1], num_ios = s_meta[2], io_off = s_meta[3];
    const uint32_t num_srams = s_meta[4], sram_off = s_meta[5], R = s_meta[6];
    const uint32_t num_dup = s_meta[7];
    const bool is_x = s_meta[8] != 0;
    const uint32_t xoff = s_meta[9];
    const uint32_t hw = s_meta[128 + t / 2];
    const uint32_t hook = (t & 1) ? (hw >> 16) : (hw & 0xffffu);
    const uint32_t *gr = script + off + 256;
    const uint32_t *ch = gr + 512 * (size_t)R;

    // prefetch stage 0 (or the SRAM chunk when there are no stages)
    uint4 c0 = ldg4(ch + 4 * t), c1 = ldg4(ch + 1024 + 4 * t), c2 = ldg4(ch + 2048 + 4 * t),
          c3 = ldg4(ch + 3072 + 4 * t), cf = ldg4(ch + 4096 + 4 * t);

    // ---- global read
    uint32_t v = 0, vx = 0;
    for (uint32_t r = 0; r < R; ++r) {
      uint2 im = ldg2(gr + 512 * r + 2 * t);
      uint32_t m = im.y;
      if (m) {
        const uint32_t *base = (im.x >> 31) ? out : in;
        size_t w = im.x & 0x7fffffffu;
        uint32_t val = ldcg(base + w);
        uint32_t xv = is_x ? ldcg(base + xoff + w) : 0u;
        while (m) {
          uint32_t low = m & (0u - m);
          v = (v << 1) | ((val & low) ? 1u : 0u);
          vx = (vx << 1) | ((xv & low) ? 1u : 0u);
          m ^= low;
        }
      }
    }
    s_st[t] = v;
    s_stx[t] = vx;
    __syncthreads();

    // ---- boomerang stages
    for (uint32_t bs = 0; bs < ns; ++bs) {
      const uint32_t *nx = ch + STAGE_WORDS * (bs + 1);
      const uint32_t dcode = depth ? depth[bs] : 2u;
      uint32_t hin = gather16(s_st, c0, c1, c2, c3);
      uint32_t hinx = is_x ? gather16(s_stx, c0, c1, c2, c3) : 0u;
      const uint32_t xa = cf.x, xb = cf.y, ob = cf.z;
      const uint16_t dly = (uint16_t)(cf.w & 0xffffu);
      const bool pass = ob == 0xffffffffu;
      c0 = ldg4(nx + 4 * t);
      c1 = ldg4(nx + 1024 + 4 * t);
      c2 = ldg4(nx + 2048 + 4 * t);
      c3 = ldg4(nx + 3072 + 4 * t);
      cf = ldg4(nx + 4096 + 4 * t);
      s_in[t] = hin;
      s_inx[t] = hinx;
      __syncthreads();  // every gather from s_st done, every input word in s_in
      // level 0: threads 128..255; inputs' arrivals are 0 after the shuffle.
      // Threads below 128 keep their input word at their position: the
      // deeper levels never read it (they read level-0 outputs upwards).
      if (t >= 128) {
        uint32_t r, rx;
        xand(s_in[t - 128], s_inx[t - 128], hin, hinx, xa, xb, ob, r, rx);
        s_st[t] = r;
        if (is_x) s_stx[t] = rx;
        if (TRACK) s_arr[t] = dly;
      } else {
        s_st[t] = hin;
        s_stx[t] = hinx;
        if (TRACK) s_arr[t] = 0;
      }
      __syncthreads();
      // levels 1..3 in shared memory
      if (dcode >= 1) {
#pragma unroll
      for (int hi = 1; hi <= 3; ++hi) {
        const int w = 1 << (7 - hi);
        if (t >= w && t < 2 * w) {
          uint32_t r, rx;
          xand(s_st[t + w], s_stx[t + w], s_st[t + 2 * w], s_stx[t + 2 * w], xa, xb, ob, r, rx);
          s_st[t] = r;
          if (is_x) s_stx[t] = rx;
          if (TRACK) s_arr[t] = arr_step(pass, s_arr[t + w], s_arr[t + 2 * w], dly);
        }
        __syncthreads();
      }
      }
      // levels 4..7 inside warp 0, levels 8..12 bit-level in thread 0
      if (dcode >= 2) {
      if (t < 32) {
        uint32_t cur = s_st[t], curx = s_stx[t];
        uint32_t ca = TRACK ? (uint32_t)s_arr[t] : 0u;
        if (t < 16) ca = 0;  // only lanes 16..31 carry level-3 arrivals
#pragma unroll
        for (int hi = 4; hi <= 7; ++hi) {
          const int w = 1 << (7 - hi);
          uint32_t a = __shfl_down_sync(0xffffffffu, cur, w);
          uint32_t b = __shfl_down_sync(0xffffffffu, cur, 2 * w);
          uint32_t ax = __shfl_down_sync(0xffffffffu, curx, w);
          uint32_t bx = __shfl_down_sync(0xffffffffu, curx, 2 * w);
          uint32_t aa = __shfl_down_sync(0xffffffffu, ca, w);
          uint32_t ba = __shfl_down_sync(0xffffffffu, ca, 2 * w);
          if (t >= w && t < 2 * w) {
            uint32_t r, rx;
            xand(a, ax, b, bx, xa, xb, ob, r, rx);
            cur = r;
            if (is_x) curx = rx;
            ca = arr_step(pass, (uint16_t)aa, (uint16_t)ba, dly);
          }
        }
        uint32_t v1 = __shfl_down_sync(0xffffffffu, cur, 1);
        uint32_t v1x = __shfl_down_sync(0xffffffffu, curx, 1);
        if (t == 0) {
          uint32_t r8 = ((v1 << 16) ^ xa) & ((v1 ^ xb) | ob) & 0xffff0000u;
          uint32_t r9 = ((r8 >> 8) ^ xa) & (((r8 >> 16) ^ xb) | ob) & 0xff00u;
          uint32_t r10 = ((r9 >> 4) ^ xa) & (((r9 >> 8) ^ xb) | ob) & 0xf0u;
          uint32_t r11 = ((r10 >> 2) ^ xa) & (((r10 >> 4) ^ xb) | ob) & 0xcu;
          uint32_t r12 = ((r11 >> 1) ^ xa) & (((r11 >> 2) ^ xb) | ob) & 0x2u;
          cur = r8 | r9 | r10 | r11 | r12;
          if (is_x) {
            uint32_t d, x8, x9, x10, x11, x12;
            xand(v1 << 16, v1x << 16, v1, v1x, xa, xb, ob, d, x8);
            x8 &= 0xffff0000u;
            xand(r8 >> 8, x8 >> 8, r8 >> 16, x8 >> 16, xa, xb, ob, d, x9);
            x9 &= 0xff00u;
            xand(r9 >> 4, x9 >> 4, r9 >> 8, x9 >> 8, xa, xb, ob, d, x10);
            x10 &= 0xf0u;
            xand(r10 >> 2, x10 >> 2, r10 >> 4, x10 >> 4, xa, xb, ob, d, x11);
            x11 &= 0xcu;
            xand(r11 >> 1, x11 >> 1, r11 >> 2, x11 >> 2, xa, xb, ob, d, x12);
            x12 &= 0x2u;
            curx = x8 | x9 | x10 | x11 | x12;
          } else {
            curx = 0;
          }
          ca = 0;  // thread 0's arrival is never advanced
        }
        s_st[t] = cur;
        s_stx[t] = curx;
        if (TRACK) s_arr[t] = (uint16_t)ca;
      }
      __syncthreads();
      }
      if ((hook >> 8) == bs) {
        const uint32_t src = hook & 255u;
        s_wo[t] = s_st[src];
        if (is_x) s_wox[t] = s_stx[src];
        if (TRACK) s_woarr[t] = s_arr[src];
      }
    }
    __syncthreads();

    // ---- SRAM & duplicate permutation (c* hold the SRAM chunk now)
    uint32_t sd = (gather16(s_wo, c0, c1, c2, c3) & ~cf.y) ^ cf.x;
    uint32_t sdx = is_x ? (gather16(s_wox, c0, c1, c2, c3) & ~cf.y) : 0u;
    {
      const uint32_t *ck = ch + STAGE_WORDS * (ns + 1);
      c0 = ldg4(ck + 4 * t);
      c1 = ldg4(ck + 1024 + 4 * t);
      c2 = ldg4(ck + 2048 + 4 * t);
      c3 = ldg4(ck + 3072 + 4 * t);
      cf = ldg4(ck + 4096 + 4 * t);
    }
    __syncthreads();  // every thread has gathered from s_wo before SRAM/dup slots change
    const uint32_t en = __shfl_down_sync(0xffffffffu, sd, 1);
    const uint32_t data = __shfl_down_sync(0xffffffffu, sd, 2);
    const uint32_t datax = __shfl_down_sync(0xffffffffu, sdx, 2);
    if ((uint32_t)t < num_srams * 4 && (t & 3) == 0) {
      const uint32_t i = t >> 2;
      uint32_t *ram = P.sram + sram_off + (size_t)i * SRAM_WORDS;
      const uint32_t ra = sd & 0xffffu, wa = sd >> 16;
      uint32_t r = ldcg(ram + ra), w0 = ldcg(ram + wa);
      uint32_t rx = 0, w0x = 0;
      const bool hx = is_x && P.sram_x != nullptr;
      uint32_t *ramx = hx ? P.sram_x + sram_off + (size_t)i * SRAM_WORDS : nullptr;
      if (hx) {
        rx = ldcg(ramx + ra);
        w0x = ldcg(ramx + wa);
      }
      s_wo[num_ios - num_srams + i] = r;
      ram[wa] = (w0 & ~en) | (data & en);
      if (is_x) {
        s_wox[num_ios - num_srams + i] = rx;
        if (hx) ramx[wa] = (w0x & ~en) | (datax & en);
      }
    } else if ((uint32_t)t >= num_srams * 4 && (uint32_t)t < num_srams * 4 + num_dup) {
      const uint32_t slot = num_ios - num_srams - num_dup + (t - num_srams * 4);
      s_wo[slot] = sd;
      if (is_x) s_wox[slot] = sdx;
    }
    __syncthreads();

    // ---- clock-enable permutation and commit
    uint32_t cp = (gather16(s_wo, c0, c1, c2, c3) & ~cf.y) ^ cf.x;
    uint32_t cpx = is_x ? (gather16(s_wox, c0, c1, c2, c3) & ~cf.y) : 0u;
    if ((uint32_t)t < num_ios) {
      const size_t o = (size_t)io_off + t;
      const uint32_t wv = s_wo[t] ^ cf.z;
      const uint32_t old = ldcg(in + o);
      out[o] = (old & ~cp) | (wv & cp);
      if (is_x) {
        const uint32_t oldx = ldcg(in + xoff + o);
        const uint32_t wx = s_wox[t];
        out[xoff + o] = (oldx & ~cp & ~cpx) | (wx & cp & ~cpx) | cpx;
      }
      if (TRACK) {
        const uint16_t a = s_woarr[t];
        if (P.arrival_off != 0) out[(size_t)(uint32_t)P.arrival_off + o] = (uint32_t)a;
        if (cons != nullptr && cp != 0) {
          const uint32_t c = __ldg(cons + o);
          if (c != 0) {
            const uint16_t su = (uint16_t)(c >> 16), ho = (uint16_t)(c & 0xffffu);
            if (a > 0 && (uint32_t)a + (uint32_t)su > clock_ps)
              push_event(P.events, P.event_cap, 4, (uint32_t)o, cycle,
                         (uint32_t)((int32_t)clock_ps - (int32_t)a - (int32_t)su), a, su);
            if (a < ho)
              push_event(P.events, P.event_cap, 5, (uint32_t)o, cycle,
                         (uint32_t)((int32_t)a - (int32_t)ho), a, ho);
          }
        }
      }
    }
    off += 256 + 512 * (size_t)R + STAGE_WORDS * ((size_t)ns + 2);
    if (depth) depth += ns;
    if (is_last) break;
    __syncthreads();
  }
}

template <bool TRACK>
__global__ void __launch_bounds__(NT, 3) jq_plain_kernel(PlainParams P) {
  __shared__ uint32_t s_meta[NT], s_st[NT], s_stx[NT], s_wo[NT], s_wox[NT], s_in[NT], s_inx[NT];
  __shared__ uint16_t s_arr[NT], s_woarr[NT];
  __shared__ size_t s_start[32];
  const int t = threadIdx.x;
  s_wo[t] = 0;
  s_wox[t] = 0;
  s_stx[t] = 0;
  s_arr[t] = 0;
  s_woarr[t] = 0;
  if (t < (int)P.num_major_stages) s_start[t] = P.blocks_start[(size_t)t * P.num_blocks + blockIdx.x];
  __syncthreads();
  for (size_t c = 0; c < P.num_cycles; ++c) {
    const uint32_t *in = P.states + c * P.state_size;
    uint32_t *out = P.states + (c + 1) * P.state_size;
    for (unsigned ms = 0; ms < P.num_major_stages; ++ms) {
      const uint8_t *dp =
          P.depth ? P.depth + P.depth_base[(size_t)ms * P.num_blocks + blockIdx.x] : nullptr;
      run_block<TRACK>(P, P.blocks_data + s_start[ms], in, out, P.first_cycle + (uint32_t)c,
                       s_meta, s_st, s_stx, s_wo, s_wox, s_arr, s_woarr, s_in, s_inx, dp);
      if (!grid_barrier(P.slot, P.num_blocks, P.timeout)) return;
    }
  }
}

// 16-bit shuffle index q (0..8191) of a boomerang chunk: bit k of thread T
// at chunk[(k>>3)*1024 + T*4 + ((k>>1)&3)], low half for even k
// (src/flatten.rs:984-1076).
__device__ __forceinline__ uint32_t shuffle_src(const uint32_t *chunk, uint32_t q) {
  const uint32_t T = q >> 5, k = q & 31;
  const uint32_t w = chunk[(k >> 3) * 1024 + T * 4 + ((k >> 1) & 3)];
  return ((k & 1) ? (w >> 16) : (w & 0xffffu)) & 8191u;
}

// Boomerang stages per (major stage, block) entry.
__global__ void jq_plain_stage_count_kernel(const size_t *blocks_start, const uint32_t *script,
                                            uint32_t *counts, unsigned entries) {
  const unsigned e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= entries) return;
  size_t off = blocks_start[e];
  uint32_t n = 0;
  for (;;) {
    const uint32_t ns = script[off];
    if (!ns) break;
    n += ns;
    if (script[off + 1]) break;
    off += 256 + 512 * (size_t)script[off + 6] + STAGE_WORDS * ((size_t)ns + 2);
  }
  counts[e] = n;
}

// Stage depth codes of one (major stage, block) entry's partitions (one CTA
// of NT threads per entry).  Walking each partition's stages last to first:
// a tree position is read from outside its stage when a writeout hook of the
// stage covers its word or a needed gather of the next stage names it, and
// it is live when it is read from outside or its parent is live (children
// [2L, 3L) are the a inputs of [L, 2L), [3L, 4L) its b inputs).  A gather of
// a first-level position (4096..8191) is needed when the position is live,
// except the b input when ob forces it to one.  The code is 2 when a
// position below 512 is live, else 1 when one below 4096 is, else 0.
__global__ void __launch_bounds__(NT) jq_plain_depth_kernel(const size_t *blocks_start,
                                                            const uint32_t *script,
                                                            const uint32_t *depth_base,
                                                            uint8_t *depth, unsigned entries) {
  __shared__ uint32_t need[256], ext[256];
  __shared__ uint8_t live[8192];
  __shared__ int any_deep, any_mid;
  const unsigned e = blockIdx.x;
  if (e >= entries) return;
  const uint32_t t = threadIdx.x;
  size_t off = blocks_start[e];
  uint8_t *dp = depth + depth_base[e];
  for (;;) {
    const uint32_t ns = script[off];
    if (!ns) break;
    const uint32_t nio = script[off + 2], R = script[off + 6];
    const uint32_t *ch = script + off + 256 + 512 * (size_t)R;
    need[t] = 0;  // nothing reads the last stage but its hooks
    __syncthreads();
    for (int ci = (int)ns - 1; ci >= 0; --ci) {
      const uint32_t *C = ch + (size_t)ci * STAGE_WORDS;
      ext[t] = need[t];
      if (t == 0) any_deep = any_mid = 0;
      __syncthreads();
      for (uint32_t slot = t; slot < nio; slot += NT) {
        const uint32_t hw = script[off + 128 + slot / 2];
        const uint32_t hook = (slot & 1) ? (hw >> 16) : (hw & 0xffffu);
        if ((hook >> 8) == (uint32_t)ci) ext[hook & 255u] = 0xffffffffu;
      }
      __syncthreads();
      // top-down, one level per pass: position 1, then [2, 4), ..., [4096, 8192)
      if (t == 0) live[0] = 0;
      for (uint32_t M = 1; M <= 4096; M <<= 1) {
        for (uint32_t c = M + t; c < 2 * M; c += NT) {
          uint8_t l = (uint8_t)((ext[c >> 5] >> (c & 31)) & 1u);
          if (M > 1) {
            const uint32_t h = M >> 1;
            l |= live[c < M + h ? c - h : c - M];
          }
          live[c] = l;
        }
        __syncthreads();
      }
      int deep = 0, mid = 0;
      for (uint32_t c = 1 + t; c < 4096; c += NT) {
        if (live[c]) {
          if (c < 512) deep = 1;
          else mid = 1;
        }
      }
      if (deep) any_deep = 1;
      if (mid) any_mid = 1;
      need[t] = 0;
      __syncthreads();
      // the previous stage's positions that this stage's needed gathers read
      for (uint32_t P = 4096 + t; P < 8192; P += NT) {
        if (!live[P]) continue;
        const uint32_t sa = shuffle_src(C, P - 4096);
        atomicOr(&need[sa >> 5], 1u << (sa & 31));
        const bool ob = (C[4096 + 4 * (P >> 5) + 2] >> (P & 31)) & 1u;
        if (!ob) {
          const uint32_t sb = shuffle_src(C, P);
          atomicOr(&need[sb >> 5], 1u << (sb & 31));
        }
      }
      if (t == 0) dp[ci] = any_deep ? 2 : any_mid ? 1 : 0;
      __syncthreads();
    }
    dp += ns;
    if (script[off + 1]) break;
    off += 256 + 512 * (size_t)R + STAGE_WORDS * ((size_t)ns + 2);
  }
}

}  // namespace jqk

// ------------------------------------------------------------------ host side
#include <cstdio>
#include <cstdlib>

using namespace jqk;

namespace {

// Re-arms one slot's barrier and status before a launch (a kernel, so that
// it is captured in CUDA graphs together with the launch).
__global__ void jq_plain_reset_kernel(int slot) {
  g_bar_count[slot] = 0;
  g_status[slot] = 0;
}

int g_max_blocks_cache[64];

// Stage-depth tables of the legacy wrappers, per device: allocated on the
// first call and grown when a larger script comes (the reference's wrappers
// take no workspace), refilled by every call.
struct DepthCache {
  uint8_t *depth = nullptr;
  uint32_t *base = nullptr;
  size_t depth_cap = 0, base_cap = 0;
};
DepthCache g_depth_cache[64];

int plain_prepare(const size_t *blocks_start, const uint32_t *blocks_data, size_t num_blocks,
                  size_t num_major_stages, uint32_t *depth_base, uint8_t *depth,
                  size_t depth_capacity, size_t *num_stages, cudaStream_t st) {
  const size_t entries = num_blocks * num_major_stages;
  jq_plain_stage_count_kernel<<<(unsigned)((entries + 255) / 256), 256, 0, st>>>(
      blocks_start, blocks_data, depth_base, (unsigned)entries);
  if (cudaGetLastError() != cudaSuccess) return JQ_ERR_LAUNCH;
  uint32_t *h = (uint32_t *)malloc(entries * sizeof(uint32_t));
  if (!h) return JQ_ERR_INVALID_ARG;
  int rc = JQ_OK;
  if (cudaMemcpyAsync(h, depth_base, entries * sizeof(uint32_t), cudaMemcpyDeviceToHost, st) !=
          cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess) {
    rc = JQ_ERR_CUDA;
  } else {
    size_t total = 0;
    for (size_t e = 0; e < entries; ++e) {
      const uint32_t c = h[e];
      h[e] = (uint32_t)total;
      total += c;
    }
    if (num_stages) *num_stages = total;
    if (!depth) {
      // counting only
    } else if (total > depth_capacity || total > 0xffffffffu) {
      rc = JQ_ERR_INVALID_ARG;
    } else {
      if (cudaMemcpyAsync(depth_base, h, entries * sizeof(uint32_t), cudaMemcpyHostToDevice, st) !=
          cudaSuccess) {
        rc = JQ_ERR_CUDA;
      } else {
        jq_plain_depth_kernel<<<(unsigned)entries, NT, 0, st>>>(blocks_start, blocks_data,
                                                                depth_base, depth,
                                                                (unsigned)entries);
        if (cudaGetLastError() != cudaSuccess) rc = JQ_ERR_LAUNCH;
        else if (cudaStreamSynchronize(st) != cudaSuccess) rc = JQ_ERR_CUDA;
      }
    }
  }
  free(h);
  return rc;
}

// The legacy wrappers' stage-depth tables for this script (device memory
// of the cache); false when they cannot be made, and then every level runs.
bool legacy_depth(jq_sim_args *a) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return false;
  DepthCache &dc = g_depth_cache[dev];
  const size_t entries = a->num_blocks * a->num_major_stages;
  if (dc.base_cap < entries) {
    if (dc.base) cudaFree(dc.base);
    dc.base = nullptr;
    dc.base_cap = 0;
    if (cudaMalloc(&dc.base, entries * sizeof(uint32_t)) != cudaSuccess) return false;
    dc.base_cap = entries;
  }
  size_t stages = 0;
  if (plain_prepare(a->blocks_start, a->blocks_data, a->num_blocks, a->num_major_stages, dc.base,
                    nullptr, 0, &stages, nullptr) != JQ_OK ||
      stages == 0)
    return false;
  if (dc.depth_cap < stages) {
    if (dc.depth) cudaFree(dc.depth);
    dc.depth = nullptr;
    dc.depth_cap = 0;
    if (cudaMalloc(&dc.depth, stages) != cudaSuccess) return false;
    dc.depth_cap = stages;
  }
  if (plain_prepare(a->blocks_start, a->blocks_data, a->num_blocks, a->num_major_stages, dc.base,
                    dc.depth, dc.depth_cap, nullptr, nullptr) != JQ_OK)
    return false;
  a->stage_depth = dc.depth;
  a->stage_depth_base = dc.base;
  return true;
}

int launch_plain(const jq_sim_args *a, uint32_t event_cap) {
  if (!a || a->num_blocks == 0 || a->num_major_stages == 0 || a->num_major_stages > 32 ||
      !a->blocks_start || !a->blocks_data || !a->states)
    return JQ_ERR_INVALID_ARG;
  if (a->timing_constraints && !a->events) return JQ_ERR_INVALID_ARG;
  cudaStream_t st = (cudaStream_t)a->stream;
  const int slot = launch_slot(a->stream, true);
  if (slot < 0) return JQ_ERR_TOO_MANY_STREAMS;
  const bool track = a->arrival_state_offset != 0 || a->timing_constraints != nullptr;
  int dev = 0;
  cudaGetDevice(&dev);
  size_t maxb = 0;
  if (jq_max_blocks(dev, &maxb) != JQ_OK) return JQ_ERR_LAUNCH;
  if (a->num_blocks > maxb) return JQ_ERR_TOO_MANY_BLOCKS;
  PlainParams P;
  P.num_blocks = (unsigned)a->num_blocks;
  P.num_major_stages = (unsigned)a->num_major_stages;
  P.blocks_start = a->blocks_start;
  P.blocks_data = a->blocks_data;
  P.sram = a->sram_data;
  P.sram_x = a->sram_xmask;
  P.num_cycles = a->num_cycles;
  P.state_size = a->state_size;
  P.states = a->states;
  P.constraints = a->timing_constraints;
  P.events = a->events;
  P.event_cap = event_cap;
  P.arrival_off = a->arrival_state_offset;
  P.first_cycle = a->first_cycle;
  P.timeout = a->barrier_timeout_cycles ? a->barrier_timeout_cycles : DEFAULT_BARRIER_TIMEOUT;
  P.slot = slot;
  P.depth = a->stage_depth;
  P.depth_base = a->stage_depth_base;
  if ((P.depth == nullptr) != (P.depth_base == nullptr)) return JQ_ERR_INVALID_ARG;
  // reset this slot's barrier (ordered before the kernel on the stream)
  jq_plain_reset_kernel<<<1, 1, 0, st>>>(slot);
  if (cudaGetLastError() != cudaSuccess) return JQ_ERR_LAUNCH;
  void *args[] = {&P};
  cudaError_t e = track ? cudaLaunchCooperativeKernel((void *)jq_plain_kernel<true>, P.num_blocks,
                                                      NT, args, 0, st)
                        : cudaLaunchCooperativeKernel((void *)jq_plain_kernel<false>, P.num_blocks,
                                                      NT, args, 0, st);
  return e == cudaSuccess ? JQ_OK : JQ_ERR_LAUNCH;
}

void die_on(int rc, const char *what) {
  if (rc == JQ_OK) return;
  cudaError_t e = cudaGetLastError();
  printf("CUDA error at %s: %s (%s)\n", what, jq_strerror(rc), cudaGetErrorString(e));
  exit(EXIT_FAILURE);
}

// Status of the slot's launches so far: JQ_OK, the kernel's recorded error,
// or JQ_ERR_CUDA.  Synchronizes the stream and clears the recorded error.
int read_status(void *stream) {
  if (cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess) return JQ_ERR_CUDA;
  const int slot = launch_slot(stream, false);
  if (slot < 0) return JQ_OK;  // nothing launched on this stream
  int flag = 0;
  if (cudaMemcpyFromSymbol(&flag, g_status, sizeof(int), slot * sizeof(int)) != cudaSuccess)
    return JQ_ERR_CUDA;
  static const int zero = 0;
  if (cudaMemcpyToSymbol(g_status, &zero, sizeof(int), slot * sizeof(int)) != cudaSuccess)
    return JQ_ERR_CUDA;
  return flag;
}

// The legacy wrappers: launch on the legacy default stream, then wait for
// the launch and exit on any error, as the reference's checkCudaErrors does
// for launch errors (csrc/kernel_v1.cu:6-14).  The reference's grid.sync()
// cannot time out; this interpreter's bounded barrier can, and a launch that
// ended that way has left the snapshots half-written, so it is an error here
// too.  The wait makes these calls synchronous; their caller synchronizes
// right after them anyway (src/bin/jacquard.rs:1131, 1149).
void legacy_launch(const jq_sim_args *a0, uint32_t event_cap, const char *what) {
  jq_sim_args a1 = *a0;
  jq_sim_args *a = &a1;
  legacy_depth(a);
  die_on(launch_plain(a, event_cap), what);
  const int rc = read_status(nullptr);
  if (rc == JQ_OK) return;
  printf("CUDA error at %s: %s (%s)\n", what, jq_strerror(rc),
         cudaGetErrorString(cudaGetLastError()));
  exit(EXIT_FAILURE);
}

}  // namespace

extern "C" {

int jq_max_blocks(int device, size_t *max_blocks) {
  if (device < 0 || device >= 64 || !max_blocks) return JQ_ERR_INVALID_ARG;
  if (!g_max_blocks_cache[device]) {
    int sms = 0, a = 0, b = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
      return JQ_ERR_LAUNCH;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, jq_plain_kernel<true>, NT, 0) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, jq_plain_kernel<false>, NT, 0) != cudaSuccess)
      return JQ_ERR_LAUNCH;
    g_max_blocks_cache[device] = sms * (a < b ? a : b);
  }
  *max_blocks = (size_t)g_max_blocks_cache[device];
  return JQ_OK;
}

int jq_simulate(const jq_sim_args *a) { return launch_plain(a, a ? a->event_capacity : 0); }

int jq_plain_prepare(const size_t *blocks_start, const uint32_t *blocks_data, size_t num_blocks,
                     size_t num_major_stages, uint32_t *stage_depth_base, uint8_t *stage_depth,
                     size_t depth_capacity, size_t *num_stages, void *stream) {
  if (!blocks_start || !blocks_data || !stage_depth_base || num_blocks == 0 ||
      num_major_stages == 0)
    return JQ_ERR_INVALID_ARG;
  return plain_prepare(blocks_start, blocks_data, num_blocks, num_major_stages, stage_depth_base,
                       stage_depth, depth_capacity, num_stages, (cudaStream_t)stream);
}

int jq_sim_status(void *stream) { return read_status(stream); }

const char *jq_strerror(int code) {
  switch (code) {
    case JQ_OK: return "ok";
    case JQ_ERR_INVALID_ARG: return "invalid argument";
    case JQ_ERR_LAUNCH: return "kernel launch failed";
    case JQ_ERR_BARRIER_TIMEOUT: return "grid barrier wait timed out";
    case JQ_ERR_CUDA: return "CUDA error";
    case JQ_ERR_TOO_MANY_BLOCKS: return "more blocks than can be co-resident";
    case JQ_ERR_EVENT_OVERFLOW: return "event buffer overflowed";
    case JQ_ERR_TOO_MANY_STREAMS:
      return "launches on more distinct streams than the interpreter has barrier slots";
    case JQ_ERR_NOALLOC_LIMIT:
      return "request exceeds the built-in no-allocation workspace (JQ_MLP_NOALLOC_MAX_CTAS CTAs)";
    default: return "unknown status";
  }
}

void simulate_v1_noninteractive_simple_scan_cuda(size_t num_blocks, size_t num_major_stages,
                                                 const size_t *blocks_start,
                                                 const uint32_t *blocks_data, uint32_t *sram_data,
                                                 uint32_t *sram_xmask, size_t num_cycles,
                                                 size_t state_size, uint32_t *states_noninteractive,
                                                 int32_t arrival_state_offset) {
  jq_sim_args a = {};
  a.num_blocks = num_blocks;
  a.num_major_stages = num_major_stages;
  a.blocks_start = blocks_start;
  a.blocks_data = blocks_data;
  a.sram_data = sram_data;
  a.sram_xmask = sram_xmask;
  a.num_cycles = num_cycles;
  a.state_size = state_size;
  a.states = states_noninteractive;
  a.arrival_state_offset = arrival_state_offset;
  legacy_launch(&a, 0, "simulate_v1_noninteractive_simple_scan_cuda");
}

void simulate_v1_noninteractive_timed_cuda(size_t num_blocks, size_t num_major_stages,
                                           const size_t *blocks_start, const uint32_t *blocks_data,
                                           uint32_t *sram_data, uint32_t *sram_xmask,
                                           size_t num_cycles, size_t state_size,
                                           uint32_t *states_noninteractive,
                                           const uint32_t *timing_constraints,
                                           uint8_t *event_buffer, int32_t arrival_state_offset) {
  jq_sim_args a = {};
  a.num_blocks = num_blocks;
  a.num_major_stages = num_major_stages;
  a.blocks_start = blocks_start;
  a.blocks_data = blocks_data;
  a.sram_data = sram_data;
  a.sram_xmask = sram_xmask;
  a.num_cycles = num_cycles;
  a.state_size = state_size;
  a.states = states_noninteractive;
  a.timing_constraints = timing_constraints;
  a.events = (jq_event_buffer *)event_buffer;
  a.arrival_state_offset = arrival_state_offset;
  // the reference's EventBuffer holds MAX_EVENTS = 1024 records
  legacy_launch(&a, 1024, "simulate_v1_noninteractive_timed_cuda");
}

}  // extern "C"
