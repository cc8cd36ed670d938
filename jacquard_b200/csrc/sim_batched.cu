// Bit-lane batched interpreter for sm_100a: many independent stimulus streams
// run the same script in one launch.
//
// Layout: a lane word is one u32 holding one signal of 32 streams.  The state
// is lane-major, T[lane * signals + signal] for L lane words (32*L streams),
// where `signal` is the bit position of the plain layout (word*32 + bit); the
// X plane sits at signal offset xoff*32 exactly as in the plain layout.  A
// work item touches one lane, so its commit writes are contiguous and the
// signals one global-read mask selects share a 128-byte line.  In this
// form the boomerang 16-pair bit shuffle becomes a word gather and every tree
// position evaluates one 32-stream word:
//     v[p] = (v[p+L] ^ xa_p) & ((v[p+2L] ^ xb_p) | ob_p),  L = msb(p)
// (the plain kernel's level-0 / shared / warp / bit-level tree steps are all
// this one positional rule).  Semantics per stream are those of the plain
// interpreter (csrc/kernel_v1_impl.cuh:32-563).
//
// Work item = (script block, lane word) for one (cycle, major stage); CTAs
// take items from a ticket counter (block-major, so the L lane items of one
// block run back to back and share its script in L2).  Each 20 KB script
// chunk is staged into shared memory with a TMA bulk copy (cp.async.bulk,
// mbarrier completion, double-buffered one chunk ahead).  Tree levels 1..4 of
// a stage stay in registers: thread t owns positions t + 512k, whose
// children are its own.  Timing arrivals / setup-hold events are handled by
// the plain interpreter (they do not depend on the stimulus stream).
#include "sim_common.cuh"

#include <cstdio>

namespace jqk {

constexpr int BT = 512;  // threads per CTA
constexpr uint32_t CHUNK_BYTES = STAGE_WORDS * 4;

static __device__ unsigned int g_ticket[BAR_SLOTS];

struct BatchParams {
  unsigned num_blocks, num_major_stages, lanes;
  const size_t *blocks_start;
  const uint32_t *blocks_data;
  uint32_t *sram, *sram_x;  // [stream][sram_words]
  size_t sram_words;
  size_t num_cycles;
  size_t sig_per_snap;      // effective words * 32
  uint32_t *state_a, *state_b;  // ping-pong snapshots, lane-major
  const uint32_t *stim;     // [cycle+1][lanes][input_sigs] input values, or null
  size_t input_sigs;        // stimulus signals per lane per cycle
  const uint32_t *input_regions;  // (dst signal, src signal, count) triples or null
  uint32_t n_input_regions;
  const uint32_t *po_sig;   // signals recorded per cycle
  uint32_t n_po;
  uint32_t *wave;           // [cycle][n_po][lanes]
  uint32_t *record;         // optional full snapshots [cycle+1][lanes][sig]
  uint32_t wo_slots;        // max num_ios over the script (wo capacity)
  const uint32_t *block_list;        // non-empty blocks per major stage, or null
  const uint32_t *block_list_start;  // num_major_stages + 1 offsets
  unsigned long long *part_cycles;   // optional per-partition SM-clock totals
  const uint32_t *part_base;         // first partition index of (stage, block)
  uint64_t timeout;
  int slot;
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void tma_load_1d(void *dst, const void *src, uint32_t bytes,
                                            uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
// Bounded wait for the barrier phase with the given parity.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint64_t limit) {
  uint32_t done = 0;
  uint64_t t0 = clock64();
  for (;;) {
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (done) return true;
    if ((uint64_t)(clock64() - t0) > limit) return false;
  }
}

// 16-bit shuffle index q (0..8191) of a 5120-word chunk: the plain layout
// puts bit k of thread T at chunk[(k>>3)*1024 + T*4 + ((k>>1)&3)], low half
// for even k.
__device__ __forceinline__ uint32_t perm_at(const uint32_t *chunk, uint32_t q) {
  const uint32_t T = q >> 5, k = q & 31;
  const uint32_t w = chunk[(k >> 3) * 1024 + T * 4 + ((k >> 1) & 3)];
  return (k & 1) ? (w >> 16) : (w & 0xffffu);
}
// Tree-state address of position p in shared memory: a bijective XOR
// swizzle that gives the 32 lanes of a warp distinct banks under the
// residue ownership map (lane bits sit at position bits 4..8).
__device__ __forceinline__ uint32_t sw(uint32_t p) { return p ^ ((p >> 4) & 31u); }
__device__ __forceinline__ uint32_t bitmask(uint32_t word, uint32_t q) {
  return 0u - ((word >> (q & 31)) & 1u);
}

struct Shared {
  uint32_t meta[256];
  uint64_t bar[2];
  int ok;
  uint32_t ticket;
};

// One (block, lane) work item: the block's partition list for one lane word.
// Tree state S and writeouts WO hold (value, X) pairs so one shared-memory
// access moves both lanes; flags are read as one uint4 (xa, xb, ob, delay).
__device__ void run_item(const BatchParams &P, Shared &sh, uint2 *S, uint2 *WO, uint32_t *chunks,
                         uint32_t &uses0, uint32_t &uses1, const uint32_t *script,
                         const uint32_t *in, uint32_t *out, uint32_t lane, uint32_t pid0,
                         bool &failed) {
  const int t = threadIdx.x;
  const size_t lane_base = (size_t)lane * P.sig_per_snap;
  size_t off = 0;
  uint32_t pid = pid0;
  for (;;) {
    __syncthreads();
    const long long t_start = clock64();
    if (t < 256) sh.meta[t] = __ldg(script + off + t);
    __syncthreads();
    const uint32_t ns = sh.meta[0];
    if (!ns) break;
    const uint32_t is_last = sh.meta[1], num_ios = sh.meta[2], io_off = sh.meta[3];
    const uint32_t num_srams = sh.meta[4], sram_off = sh.meta[5], R = sh.meta[6];
    const uint32_t num_dup = sh.meta[7];
    const bool is_x = sh.meta[8] != 0;
    const uint32_t xsig = sh.meta[9] * 32u;
    const uint32_t *gr = script + off + 256;
    const uint32_t *ch0 = gr + 512 * (size_t)R;
    const uint32_t nchunks = ns + 2;

    // chunk 0 -> buffer 0 (the previous item/partition finished with both)
    if (t == 0) {
      mbar_expect_tx(&sh.bar[0], CHUNK_BYTES);
      tma_load_1d(chunks, ch0, CHUNK_BYTES, &sh.bar[0]);
    }

    // ---- global read, in two phases so that the loads overlap (hooks of the
    // previous partition read S before this point: the loop-top barrier):
    // (a) thread t < 256 enumerates its (idx, mask) bits and stores, at the
    //     destination position, the source signal (bit 31 = current-cycle
    //     staged IO) or NONE for the unfilled tail; positions follow the
    //     kernel's append order (first appended bit ends up most significant);
    // (b) all threads load their 16 positions with independent loads.
    uint32_t *Sv = reinterpret_cast<uint32_t *>(S);  // staging: .x words
    if (t < 256) {
      uint2 pr[16];
#pragma unroll
      for (int r = 0; r < 16; ++r)
        pr[r] = (uint32_t)r < R ? ldg2(gr + 512 * r + 2 * t) : make_uint2(0, 0);
      uint32_t total = 0;
#pragma unroll
      for (int r = 0; r < 16; ++r) total += __popc(pr[r].y);
      for (uint32_t r = 16; r < R; ++r) total += __popc(__ldg(gr + 512 * r + 2 * t + 1));
      uint32_t i = 0;
#pragma unroll
      for (int r = 0; r < 16; ++r) {
        uint32_t m = pr[r].y;
        const uint32_t stg = pr[r].x & 0x80000000u;
        const uint32_t w = pr[r].x & 0x7fffffffu;
        while (m) {
          const uint32_t k = __ffs(m) - 1;
          m &= m - 1;
          Sv[2 * sw(32 * t + (total - 1 - i))] = stg | (w * 32 + k);
          ++i;
        }
      }
      for (uint32_t r = 16; r < R; ++r) {
        const uint2 im = ldg2(gr + 512 * r + 2 * t);
        uint32_t m = im.y;
        const uint32_t stg = im.x & 0x80000000u;
        const uint32_t w = im.x & 0x7fffffffu;
        while (m) {
          const uint32_t k = __ffs(m) - 1;
          m &= m - 1;
          Sv[2 * sw(32 * t + (total - 1 - i))] = stg | (w * 32 + k);
          ++i;
        }
      }
      for (uint32_t k = total; k < 32; ++k) Sv[2 * sw(32 * t + k)] = 0xffffffffu;
    }
    __syncthreads();
    {
      uint32_t e[16], v[16], vx[16];
#pragma unroll
      for (int k = 0; k < 16; ++k) e[k] = Sv[2 * sw(t + BT * k)];
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        v[k] = 0;
        vx[k] = 0;
        if (e[k] != 0xffffffffu) {
          const uint32_t *base = (e[k] >> 31) ? out : in;
          const size_t sg = lane_base + (e[k] & 0x7fffffffu);
          v[k] = ldcg(base + sg);
          if (is_x) vx[k] = ldcg(base + xsig + sg);
        }
      }
#pragma unroll
      for (int k = 0; k < 16; ++k) S[sw(t + BT * k)] = make_uint2(v[k], vx[k]);
    }

    // Thread -> tree residue map: thread (warp w, lane l) owns positions whose
    // value mod 512 is u = w | l << 4.  Levels 1..4 then read only the
    // thread's own registers, levels 5..9 read lanes of the same warp
    // (residue bits 4..8 are lane bits), and only positions 1..15 need one
    // exchange through shared memory.
    const uint32_t lane_i = t & 31, warp_i = t >> 5;
    const uint32_t u = warp_i | (lane_i << 4);
    for (uint32_t ci = 0; ci < nchunks; ++ci) {
      const uint32_t b = ci & 1;
      uint32_t *C = chunks + b * STAGE_WORDS;
      // The other buffer's last reader finished before the final barrier of
      // the previous chunk, so the next chunk can be issued right away.
      if (ci == 0) __syncthreads();
      if (t == 0 && ci + 1 < nchunks) {
        mbar_expect_tx(&sh.bar[b ^ 1], CHUNK_BYTES);
        tma_load_1d(chunks + (b ^ 1) * STAGE_WORDS, ch0 + (size_t)STAGE_WORDS * (ci + 1),
                    CHUNK_BYTES, &sh.bar[b ^ 1]);
      }
      uint32_t &uses = b ? uses1 : uses0;
      if (!mbar_wait(&sh.bar[b], uses & 1u, P.timeout)) {
        failed = true;
        // let any copy still in flight into this CTA land before leaving
        if (t == 0) {
          mbar_wait(&sh.bar[0], uses0 & 1u, P.timeout);
          mbar_wait(&sh.bar[1], uses1 & 1u, P.timeout);
        }
      }
      ++uses;
      if (__syncthreads_or(failed)) {
        failed = true;
        return;
      }
      const uint4 *F4 = reinterpret_cast<const uint4 *>(C + 4096);  // xa, xb, ob, pad
#define JQ_FL(p, XA, XB, OB)                    \
  const uint4 fl_##XA = F4[(p) >> 5];           \
  const uint32_t XA = bitmask(fl_##XA.x, (p));  \
  const uint32_t XB = bitmask(fl_##XA.y, (p));  \
  const uint32_t OB = bitmask(fl_##XA.z, (p));

      if (ci < ns) {
        // ---------------- boomerang stage ci
        // level 1 (positions 4096 + j): gather both inputs into registers
        uint2 ga[8], gb[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const uint32_t j = u + 512 * k;
          ga[k] = S[sw(perm_at(C, j))];
          gb[k] = S[sw(perm_at(C, j + 4096))];
        }
        __syncthreads();  // all gathers done before the in-place overwrite
        uint32_t v1[8], x1[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const uint32_t p = 4096 + u + 512 * k;
          JQ_FL(p, XA, XB, OB)
          xand(ga[k].x, ga[k].y, gb[k].x, gb[k].y, XA, XB, OB, v1[k], x1[k]);
          if (!is_x) x1[k] = 0;
          S[sw(p)] = make_uint2(v1[k], x1[k]);
        }
        uint32_t v2[4], x2[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const uint32_t p = 2048 + u + 512 * k;
          JQ_FL(p, XA, XB, OB)
          xand(v1[k], x1[k], v1[k + 4], x1[k + 4], XA, XB, OB, v2[k], x2[k]);
          if (!is_x) x2[k] = 0;
          S[sw(p)] = make_uint2(v2[k], x2[k]);
        }
        uint32_t v3[2], x3[2];
#pragma unroll
        for (int k = 0; k < 2; ++k) {
          const uint32_t p = 1024 + u + 512 * k;
          JQ_FL(p, XA, XB, OB)
          xand(v2[k], x2[k], v2[k + 2], x2[k + 2], XA, XB, OB, v3[k], x3[k]);
          if (!is_x) x3[k] = 0;
          S[sw(p)] = make_uint2(v3[k], x3[k]);
        }
        uint32_t v4, x4;
        {
          const uint32_t p = 512 + u;
          JQ_FL(p, XA, XB, OB)
          xand(v3[0], x3[0], v3[1], x3[1], XA, XB, OB, v4, x4);
          if (!is_x) x4 = 0;
          S[sw(p)] = make_uint2(v4, x4);
        }
        // level 5: position u (lanes 16..31) from level-4 u-256 (lane ^ 16) and u
        uint32_t cv, cx;
        {
          const uint32_t a = __shfl_xor_sync(0xffffffffu, v4, 16);
          const uint32_t ax = __shfl_xor_sync(0xffffffffu, x4, 16);
          const uint32_t p = u;
          JQ_FL(p & 511, XA, XB, OB)
          xand(a, ax, v4, x4, XA, XB, OB, cv, cx);
          if (!is_x) cx = 0;
          if (lane_i >= 16) S[sw(p)] = make_uint2(cv, cx);
        }
        // levels 6..9: the parent of residue u with lane bit k set (lanes
        // [2^k, 2^(k+1))) reads lanes l + 2^k and l + 2^(k+1)
#pragma unroll
        for (int k = 3; k >= 0; --k) {
          const uint32_t d = 1u << k;
          const uint32_t a = __shfl_sync(0xffffffffu, cv, (lane_i + d) & 31);
          const uint32_t bb = __shfl_sync(0xffffffffu, cv, (lane_i + 2 * d) & 31);
          const uint32_t ax = __shfl_sync(0xffffffffu, cx, (lane_i + d) & 31);
          const uint32_t bx = __shfl_sync(0xffffffffu, cx, (lane_i + 2 * d) & 31);
          if (lane_i >= d && lane_i < 2 * d) {
            const uint32_t p = u;
            JQ_FL(p, XA, XB, OB)
            xand(a, ax, bb, bx, XA, XB, OB, cv, cx);
            if (!is_x) cx = 0;
            S[sw(p)] = make_uint2(cv, cx);
          }
        }
        __syncthreads();
        // levels 10..13 (positions 15..1) in warp 0 from positions 16..31
        if (t < 32) {
          uint2 h = t < 16 ? S[sw(16 + t)] : make_uint2(0, 0);
          uint32_t hv = h.x, hx = h.y;
#pragma unroll
          for (uint32_t len = 8; len >= 1; len >>= 1) {
            const uint32_t bb = __shfl_sync(0xffffffffu, hv, (t + len) & 31);
            const uint32_t bx = __shfl_sync(0xffffffffu, hx, (t + len) & 31);
            if ((uint32_t)t < len) {
              const uint32_t p = len + t;
              JQ_FL(p, XA, XB, OB)
              uint32_t r, rx;
              xand(hv, hx, bb, bx, XA, XB, OB, r, rx);
              if (!is_x) rx = 0;
              S[sw(p)] = make_uint2(r, rx);
              hv = r;
              hx = rx;
            }
          }
          if (t == 0) S[0] = make_uint2(0, 0);
        }
        __syncthreads();
        // writeout hooks of this stage
        for (uint32_t q = t; q < num_ios * 32; q += BT) {
          const uint32_t slot = q >> 5;
          const uint32_t hw = sh.meta[128 + slot / 2];
          const uint32_t hook = (slot & 1) ? (hw >> 16) : (hw & 0xffffu);
          if ((hook >> 8) == ci) WO[q] = S[sw((hook & 255u) * 32 + (q & 31))];
        }
      } else if (ci == ns) {
        // ---------------- SRAM & duplicate permutation + SRAM ports
        const uint32_t nq = (num_srams * 4 + num_dup) * 32;
        // stage the permuted words in S (free now: all hooks are done)
        for (uint32_t q = t; q < nq; q += BT) {
          const uint2 w = WO[perm_at(C, q)];
          const uint4 fl = F4[q >> 5];
          const uint32_t inv = bitmask(fl.x, q), set0 = bitmask(fl.y, q);
          S[q] = make_uint2((w.x & ~set0) ^ inv, is_x ? (w.y & ~set0) : 0u);
        }
        __syncthreads();
        // one warp per SRAM, lane = stream within the lane word
        const int warp = t >> 5, ln = t & 31;
        for (uint32_t i = warp; i < num_srams; i += BT / 32) {
          const uint2 *A = S + (4 * i) * 32;
          uint32_t ra = 0, wa = 0, en = 0, data = 0, datax = 0;
#pragma unroll
          for (int k = 0; k < 16; ++k) {
            ra |= ((A[k].x >> ln) & 1u) << k;
            wa |= ((A[16 + k].x >> ln) & 1u) << k;
          }
#pragma unroll 8
          for (int k = 0; k < 32; ++k) {
            en |= ((A[32 + k].x >> ln) & 1u) << k;
            const uint2 dk = A[64 + k];
            data |= ((dk.x >> ln) & 1u) << k;
            datax |= ((dk.y >> ln) & 1u) << k;
          }
          const size_t stream = (size_t)lane * 32 + ln;
          uint32_t *ram = P.sram + stream * P.sram_words + sram_off + (size_t)i * SRAM_WORDS;
          const uint32_t r = ldcg(ram + ra), w0 = ldcg(ram + wa);
          uint32_t rx = 0;
          const bool hx = is_x && P.sram_x != nullptr;
          uint32_t *ramx = hx ? P.sram_x + stream * P.sram_words + sram_off + (size_t)i * SRAM_WORDS
                              : nullptr;
          uint32_t w0x = 0;
          if (hx) {
            rx = ldcg(ramx + ra);
            w0x = ldcg(ramx + wa);
          }
          ram[wa] = (w0 & ~en) | (data & en);
          if (hx) ramx[wa] = (w0x & ~en) | (datax & en);
          // transpose the 32 streams' read words into 32 signal words
          const uint32_t slotw = (num_ios - num_srams + i) * 32;
#pragma unroll 4
          for (int k = 0; k < 32; ++k) {
            const uint32_t word = __ballot_sync(0xffffffffu, (r >> k) & 1u);
            const uint32_t wordx = __ballot_sync(0xffffffffu, (rx >> k) & 1u);
            if (ln == k) WO[slotw + k] = make_uint2(word, is_x ? wordx : 0u);
          }
        }
        for (uint32_t q = t; q < num_dup * 32; q += BT)
          WO[(num_ios - num_srams - num_dup) * 32 + q] = S[num_srams * 4 * 32 + q];
        __syncthreads();
      } else {
        // ---------------- clock-enable permutation and commit (4 words per
        // thread in flight)
        const uint32_t nq = num_ios * 32;
        for (uint32_t q0 = t; q0 < nq; q0 += 4 * BT) {
          uint32_t cp[4], cpx[4], wv[4], wx[4], old[4], oldx[4];
          size_t sg[4];
#pragma unroll
          for (int uu = 0; uu < 4; ++uu) {
            const uint32_t q = q0 + uu * BT;
            if (q < nq) {
              const uint2 src = WO[perm_at(C, q)];
              const uint4 fl = F4[q >> 5];
              const uint32_t inv = bitmask(fl.x, q), set0 = bitmask(fl.y, q),
                             dinv = bitmask(fl.z, q);
              const uint2 me = WO[q];
              cp[uu] = (src.x & ~set0) ^ inv;
              cpx[uu] = is_x ? (src.y & ~set0) : 0u;
              wv[uu] = me.x ^ dinv;
              wx[uu] = me.y;
              sg[uu] = lane_base + (size_t)io_off * 32 + q;
              old[uu] = ldcg(in + sg[uu]);
              oldx[uu] = is_x ? ldcg(in + xsig + sg[uu]) : 0u;
            }
          }
#pragma unroll
          for (int uu = 0; uu < 4; ++uu) {
            const uint32_t q = q0 + uu * BT;
            if (q < nq) {
              out[sg[uu]] = (old[uu] & ~cp[uu]) | (wv[uu] & cp[uu]);
              if (is_x)
                out[xsig + sg[uu]] =
                    (oldx[uu] & ~cp[uu] & ~cpx[uu]) | (wx[uu] & cp[uu] & ~cpx[uu]) | cpx[uu];
            }
          }
        }
      }
#undef JQ_FL
    }
    off += 256 + 512 * (size_t)R + STAGE_WORDS * ((size_t)ns + 2);
    if (P.part_cycles) {
      // per-partition kernel time, measured by the simulator itself (the
      // training signal of the partition cost model)
      __syncthreads();
      if (t == 0) atomicAdd(&P.part_cycles[pid], (unsigned long long)(clock64() - t_start));
    }
    ++pid;
    if (is_last) break;
  }
}

__global__ void __launch_bounds__(BT, 1) jq_batched_kernel(BatchParams P) {
  extern __shared__ __align__(128) uint8_t dyn[];
  __shared__ Shared sh;
  uint32_t *chunks = reinterpret_cast<uint32_t *>(dyn);               // 2 x 20 KB
  uint2 *S = reinterpret_cast<uint2 *>(chunks + 2 * STAGE_WORDS);      // 8192 (v, x)
  uint2 *WO = S + 8192;                                               // wo_slots*32
  const int t = threadIdx.x;
  if (t == 0) {
    mbar_init(&sh.bar[0], 1);
    mbar_init(&sh.bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (uint32_t q = t; q < P.wo_slots * 32; q += BT) WO[q] = make_uint2(0, 0);
  __syncthreads();
  uint32_t uses0 = 0, uses1 = 0;
  bool failed = false;
  const size_t snap = P.sig_per_snap * P.lanes;

  for (size_t c = 0; c < P.num_cycles; ++c) {
    const uint32_t *in = (c & 1) ? P.state_b : P.state_a;
    uint32_t *out = (c & 1) ? P.state_a : P.state_b;
    // inputs of snapshot c+1 into the output buffer's input region
    if (P.stim) {
      // stimulus row layout [lane][input_sigs]; each input region copies
      // stimulus signals [src, src+count) to state signals [dst, dst+count)
      // (one region at 0 when no list is given)
      const uint32_t *src = P.stim + (c + 1) * P.input_sigs * P.lanes;
      for (size_t q = (size_t)blockIdx.x * BT + t; q < P.input_sigs * P.lanes;
           q += (size_t)gridDim.x * BT) {
        const size_t l = q / P.input_sigs, i = q % P.input_sigs;
        size_t dst = i;
        if (P.input_regions) {
          for (uint32_t r = 0; r < P.n_input_regions; ++r) {
            const uint32_t d0 = P.input_regions[3 * r], s0 = P.input_regions[3 * r + 1],
                           n = P.input_regions[3 * r + 2];
            if (i >= s0 && i < s0 + n) dst = d0 + (i - s0);
          }
        }
        out[l * P.sig_per_snap + dst] = src[q];
      }
    }
    for (unsigned ms = 0; ms < P.num_major_stages; ++ms) {
      const uint32_t nblk = P.block_list ? P.block_list_start[ms + 1] - P.block_list_start[ms]
                                         : P.num_blocks;
      const uint32_t items = nblk * P.lanes;
      for (;;) {
        __syncthreads();
        if (t == 0) sh.ticket = atomicAdd(&g_ticket[P.slot], 1u);
        __syncthreads();
        const uint32_t tk = sh.ticket;
        if (tk >= items) break;
        const uint32_t bi = tk / P.lanes, lane = tk % P.lanes;
        const uint32_t blk = P.block_list ? P.block_list[P.block_list_start[ms] + bi] : bi;
        const uint32_t *script = P.blocks_data + P.blocks_start[(size_t)ms * P.num_blocks + blk];
        const uint32_t pid0 = P.part_base ? P.part_base[(size_t)ms * P.num_blocks + blk] : 0u;
        run_item(P, sh, S, WO, chunks, uses0, uses1, script, in, out, lane, pid0, failed);
        if (failed) {
          if (t == 0) atomicExch(&g_status[P.slot], JQ_ERR_BARRIER_TIMEOUT);
          return;
        }
      }
      // last arriver re-arms the ticket counter inside the barrier
      __syncthreads();
      if (t == 0) {
        unsigned gen = ld_acquire(&g_bar_gen[P.slot]);
        __threadfence();
        unsigned arrived = atomicAdd(&g_bar_count[P.slot], 1u);
        int ok = 1;
        if (arrived == gridDim.x - 1) {
          g_ticket[P.slot] = 0;
          g_bar_count[P.slot] = 0;
          __threadfence();
          atomicAdd(&g_bar_gen[P.slot], 1u);
        } else {
          uint64_t t0 = clock64();
          while (ld_acquire(&g_bar_gen[P.slot]) == gen) {
            __nanosleep(64);
            if ((uint64_t)(clock64() - t0) > P.timeout) {
              ok = 0;
              atomicExch(&g_status[P.slot], JQ_ERR_BARRIER_TIMEOUT);
              break;
            }
          }
        }
        if (ok && *((volatile int *)&g_status[P.slot]) != 0) ok = 0;
        sh.ok = ok;
      }
      __syncthreads();
      if (!sh.ok) return;
    }
    // record outputs of this cycle
    for (size_t q = (size_t)blockIdx.x * BT + t; q < (size_t)P.n_po * P.lanes;
         q += (size_t)gridDim.x * BT) {
      const uint32_t po = (uint32_t)(q / P.lanes), l = (uint32_t)(q % P.lanes);
      P.wave[(c * P.n_po + po) * P.lanes + l] = ldcg(out + (size_t)l * P.sig_per_snap + P.po_sig[po]);
    }
    if (P.record) {
      uint32_t *dst = P.record + (c + 1) * snap;
      for (size_t q = (size_t)blockIdx.x * BT + t; q < snap; q += (size_t)gridDim.x * BT)
        dst[q] = ldcg(out + q);
    }
    // the recording reads `out`; the next cycle writes into `in`: the next
    // major-stage barrier already orders them, no extra barrier needed.
  }
}

}  // namespace jqk

using namespace jqk;

// Re-arms one slot's barrier, ticket and status before a launch.  A kernel
// (not a host copy) so the reset is captured in CUDA graphs with the launch.
__global__ void jq_batched_reset_kernel(int slot) {
  g_bar_count[slot] = 0;
  g_ticket[slot] = 0;
  g_status[slot] = 0;
}

extern "C" {

int jq_batched_smem_bytes(uint32_t wo_slots) {
  return (int)(2 * CHUNK_BYTES + 2 * 8192 * 4 + 2 * wo_slots * 32 * 4);
}

int jq_batched_max_blocks(int device, uint32_t wo_slots, size_t *max_blocks) {
  int smem = jq_batched_smem_bytes(wo_slots);
  if (cudaFuncSetAttribute(jq_batched_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) !=
      cudaSuccess)
    return JQ_ERR_LAUNCH;
  int sms = 0, per = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, jq_batched_kernel, BT, smem) != cudaSuccess)
    return JQ_ERR_LAUNCH;
  *max_blocks = (size_t)sms * per;
  return JQ_OK;
}

int jq_simulate_batched(const jq_batch_args *a) {
  if (!a || a->lanes == 0 || a->num_blocks == 0 || a->num_major_stages == 0 ||
      a->num_major_stages > 32 || !a->state_a || !a->state_b || a->wo_slots > 256 ||
      (a->n_po && (!a->po_signals || !a->wave)))
    return JQ_ERR_INVALID_ARG;
  cudaStream_t st = (cudaStream_t)a->stream;
  int dev = 0;
  cudaGetDevice(&dev);
  size_t maxg = 0;
  if (jq_batched_max_blocks(dev, a->wo_slots, &maxg) != JQ_OK || maxg == 0) return JQ_ERR_LAUNCH;
  size_t grid = a->grid ? a->grid : maxg;
  if (grid > maxg) return JQ_ERR_TOO_MANY_BLOCKS;
  BatchParams P;
  P.num_blocks = (unsigned)a->num_blocks;
  P.num_major_stages = (unsigned)a->num_major_stages;
  P.lanes = a->lanes;
  P.blocks_start = a->blocks_start;
  P.blocks_data = a->blocks_data;
  P.sram = a->sram_data;
  P.sram_x = a->sram_xmask;
  P.sram_words = a->sram_words_per_stream;
  P.num_cycles = a->num_cycles;
  P.sig_per_snap = a->signals_per_snapshot;
  P.state_a = a->state_a;
  P.state_b = a->state_b;
  P.stim = a->stimulus;
  P.input_sigs = a->input_signals;
  P.input_regions = a->input_regions;
  P.n_input_regions = a->n_input_regions;
  P.po_sig = a->po_signals;
  P.n_po = a->n_po;
  P.wave = a->wave;
  P.record = a->record;
  P.wo_slots = a->wo_slots ? a->wo_slots : 256;
  P.block_list = a->block_list;
  P.block_list_start = a->block_list_start;
  P.part_cycles = a->part_cycles;
  P.part_base = a->part_base;
  if (P.part_cycles && !P.part_base) return JQ_ERR_INVALID_ARG;
  P.timeout = a->barrier_timeout_cycles ? a->barrier_timeout_cycles : DEFAULT_BARRIER_TIMEOUT;
  P.slot = 1;
  jq_batched_reset_kernel<<<1, 1, 0, st>>>(P.slot);
  if (cudaGetLastError() != cudaSuccess) return JQ_ERR_LAUNCH;
  int smem = jq_batched_smem_bytes(P.wo_slots);
  void *args[] = {&P};
  cudaError_t e = cudaLaunchCooperativeKernel((void *)jq_batched_kernel, (unsigned)grid, BT, args,
                                              smem, st);
  return e == cudaSuccess ? JQ_OK : JQ_ERR_LAUNCH;
}

int jq_batched_status(void *stream) {
  if (cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess) return JQ_ERR_CUDA;
  int flags[1] = {0};
  if (cudaMemcpyFromSymbol(flags, g_status, sizeof(int), 1 * sizeof(int)) != cudaSuccess)
    return JQ_ERR_CUDA;
  static const int zero_i[1] = {0};
  cudaMemcpyToSymbol(g_status, zero_i, sizeof(int), 1 * sizeof(int));
  return flags[0];
}

}  // extern "C"
