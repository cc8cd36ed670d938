// Bit-lane batched interpreter for sm_100a: many independent stimulus streams
// run the same script in one launch.
//
// Layout: a lane word is one u32 holding one signal of 32 streams.  The state
// is signal-major, T[signal * L + lane] for L lane words (32*L streams), where
// `signal` is the bit position of the plain layout (word*32 + bit); the X
// plane sits at signal offset xoff*32 exactly as in the plain layout.  In this
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
  uint32_t *state_a, *state_b;  // ping-pong snapshots, signal-major
  const uint32_t *stim;     // [cycle+1][input_sigs][lanes] input values, or null
  size_t input_sigs;        // input region signals (states_start * 32)
  const uint32_t *po_sig;   // signals recorded per cycle
  uint32_t n_po;
  uint32_t *wave;           // [cycle][n_po][lanes]
  uint32_t *record;         // optional full snapshots [cycle+1][sig][lanes]
  uint32_t wo_slots;        // max num_ios over the script (wo capacity)
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
__device__ void run_item(const BatchParams &P, Shared &sh, uint32_t *S, uint32_t *SX, uint32_t *WO,
                         uint32_t *WOX, uint32_t *chunks, uint32_t &uses0, uint32_t &uses1,
                         const uint32_t *script, const uint32_t *in, uint32_t *out, uint32_t lane,
                         bool &failed) {
  const int t = threadIdx.x;
  const uint32_t L = P.lanes;
  size_t off = 0;
  for (;;) {
    __syncthreads();
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

    // ---- global read, in two phases so that the loads overlap:
    // (a) thread t < 256 enumerates its (idx, mask) bits and stores, at the
    //     destination position, the source signal (bit 31 = current-cycle
    //     staged IO) or NONE for the unfilled tail; positions follow the
    //     kernel's append order (first appended bit ends up most significant);
    // (b) all threads load their 16 positions with independent loads.
    if (t < 256) {
      // all (idx, mask) pairs of this thread in flight at once (R <= 16 in
      // registers; longer lists are read a second time from global)
      uint2 pr[16];
#pragma unroll
      for (int r = 0; r < 16; ++r) pr[r] = (uint32_t)r < R ? ldg2(gr + 512 * r + 2 * t) : make_uint2(0, 0);
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
          S[32 * t + (total - 1 - i)] = stg | (w * 32 + k);
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
          S[32 * t + (total - 1 - i)] = stg | (w * 32 + k);
          ++i;
        }
      }
      for (uint32_t k = total; k < 32; ++k) S[32 * t + k] = 0xffffffffu;
    }
    __syncthreads();
    {
      uint32_t e[16], v[16], vx[16];
#pragma unroll
      for (int k = 0; k < 16; ++k) e[k] = S[t + BT * k];
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        v[k] = 0;
        vx[k] = 0;
        if (e[k] != 0xffffffffu) {
          const uint32_t *base = (e[k] >> 31) ? out : in;
          const size_t sg = (size_t)(e[k] & 0x7fffffffu) * L + lane;
          v[k] = ldcg(base + sg);
          if (is_x) vx[k] = ldcg(base + (size_t)xsig * L + sg);
        }
      }
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        S[t + BT * k] = v[k];
        SX[t + BT * k] = vx[k];
      }
    }

    for (uint32_t ci = 0; ci < nchunks; ++ci) {
      const uint32_t b = ci & 1;
      uint32_t *C = chunks + b * STAGE_WORDS;
      // prefetch the next chunk into the other buffer (its last reader
      // finished before the __syncthreads that ended chunk ci-1)
      __syncthreads();
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
      const uint32_t *F = C + 4096;  // flags: xa, xb, ob, pad per word

      if (ci < ns) {
        // ---------------- boomerang stage ci
        // level 1 (positions 4096 + j): gather both inputs into registers
        uint32_t va[8], vb[8], xa_[8], xb_[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const uint32_t j = t + 512 * k;
          const uint32_t pa = perm_at(C, j), pb = perm_at(C, j + 4096);
          va[k] = S[pa];
          vb[k] = S[pb];
          xa_[k] = is_x ? SX[pa] : 0u;
          xb_[k] = is_x ? SX[pb] : 0u;
        }
        __syncthreads();  // all gathers done before the in-place overwrite
        uint32_t v1[8], x1[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const uint32_t p = 4096 + t + 512 * k;
          const uint32_t fw = (p >> 5) * 4;
          const uint32_t XA = bitmask(F[fw], p), XB = bitmask(F[fw + 1], p), OB = bitmask(F[fw + 2], p);
          xand(va[k], xa_[k], vb[k], xb_[k], XA, XB, OB, v1[k], x1[k]);
          S[p] = v1[k];
          SX[p] = is_x ? x1[k] : 0u;
        }
        // level 2: positions 2048 + t + 512k from level-1 k and k+4
        uint32_t v2[4], x2[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const uint32_t p = 2048 + t + 512 * k;
          const uint32_t fw = (p >> 5) * 4;
          xand(v1[k], x1[k], v1[k + 4], x1[k + 4], bitmask(F[fw], p), bitmask(F[fw + 1], p),
               bitmask(F[fw + 2], p), v2[k], x2[k]);
          S[p] = v2[k];
          SX[p] = is_x ? x2[k] : 0u;
        }
        uint32_t v3[2], x3[2];
#pragma unroll
        for (int k = 0; k < 2; ++k) {
          const uint32_t p = 1024 + t + 512 * k;
          const uint32_t fw = (p >> 5) * 4;
          xand(v2[k], x2[k], v2[k + 2], x2[k + 2], bitmask(F[fw], p), bitmask(F[fw + 1], p),
               bitmask(F[fw + 2], p), v3[k], x3[k]);
          S[p] = v3[k];
          SX[p] = is_x ? x3[k] : 0u;
        }
        {
          const uint32_t p = 512 + t;
          const uint32_t fw = (p >> 5) * 4;
          uint32_t v4, x4;
          xand(v3[0], x3[0], v3[1], x3[1], bitmask(F[fw], p), bitmask(F[fw + 1], p),
               bitmask(F[fw + 2], p), v4, x4);
          S[p] = v4;
          SX[p] = is_x ? x4 : 0u;
        }
        __syncthreads();
        // levels 5..7 in shared memory (256, 128, 64 positions)
#pragma unroll
        for (uint32_t len = 256; len >= 64; len >>= 1) {
          if ((uint32_t)t < len) {
            const uint32_t p = len + t;
            const uint32_t fw = (p >> 5) * 4;
            uint32_t r, rx;
            xand(S[p + len], SX[p + len], S[p + 2 * len], SX[p + 2 * len], bitmask(F[fw], p),
                 bitmask(F[fw + 1], p), bitmask(F[fw + 2], p), r, rx);
            S[p] = r;
            SX[p] = is_x ? rx : 0u;
          }
          __syncthreads();
        }
        // levels 8..13 (positions 32..63 down to 1) inside warp 0
        if (t < 32) {
          const uint32_t fw0 = 4 * 0, fw1 = 4 * 1;
          uint32_t cur, curx;
          {
            const uint32_t p = 32 + t;
            xand(S[p + 32], SX[p + 32], S[p + 64], SX[p + 64], bitmask(F[fw1], p),
                 bitmask(F[fw1 + 1], p), bitmask(F[fw1 + 2], p), cur, curx);
            if (!is_x) curx = 0;
            S[p] = cur;
            SX[p] = curx;
          }
          // lane i holds position 2*len + i of the previous level; position
          // len + i reads 2*len + i (own) and 3*len + i (lane i + len)
          uint32_t hv = cur, hx = curx;
#pragma unroll
          for (uint32_t len = 16; len >= 1; len >>= 1) {
            const uint32_t bb = __shfl_sync(0xffffffffu, hv, (t + len) & 31);
            const uint32_t bx = __shfl_sync(0xffffffffu, hx, (t + len) & 31);
            if ((uint32_t)t < len) {
              const uint32_t p = len + t;
              uint32_t r, rx;
              xand(hv, hx, bb, bx, bitmask(F[fw0], p), bitmask(F[fw0 + 1], p),
                   bitmask(F[fw0 + 2], p), r, rx);
              if (!is_x) rx = 0;
              S[p] = r;
              SX[p] = rx;
              hv = r;
              hx = rx;
            }
          }
          if (t == 0) {
            S[0] = 0;
            SX[0] = 0;
          }
        }
        __syncthreads();
        // writeout hooks of this stage
        for (uint32_t q = t; q < num_ios * 32; q += BT) {
          const uint32_t slot = q >> 5;
          const uint32_t hw = sh.meta[128 + slot / 2];
          const uint32_t hook = (slot & 1) ? (hw >> 16) : (hw & 0xffffu);
          if ((hook >> 8) == ci) {
            const uint32_t src = (hook & 255u) * 32 + (q & 31);
            WO[q] = S[src];
            WOX[q] = SX[src];
          }
        }
      } else if (ci == ns) {
        // ---------------- SRAM & duplicate permutation + SRAM ports
        const uint32_t nq = (num_srams * 4 + num_dup) * 32;
        // stage the permuted words in S (free now: all hooks are done)
        for (uint32_t q = t; q < nq; q += BT) {
          const uint32_t src = perm_at(C, q);
          const uint32_t inv = bitmask(F[(q >> 5) * 4], q), set0 = bitmask(F[(q >> 5) * 4 + 1], q);
          S[q] = (WO[src] & ~set0) ^ inv;
          SX[q] = is_x ? (WOX[src] & ~set0) : 0u;
        }
        __syncthreads();
        // one warp per SRAM, lane = stream within the lane word
        const int warp = t >> 5, ln = t & 31;
        for (uint32_t i = warp; i < num_srams; i += BT / 32) {
          const uint32_t *A = S + (4 * i) * 32;
          uint32_t ra = 0, wa = 0, en = 0, data = 0, datax = 0;
#pragma unroll
          for (int k = 0; k < 16; ++k) {
            ra |= ((A[k] >> ln) & 1u) << k;
            wa |= ((A[16 + k] >> ln) & 1u) << k;
          }
#pragma unroll 8
          for (int k = 0; k < 32; ++k) {
            en |= ((A[32 + k] >> ln) & 1u) << k;
            data |= ((A[64 + k] >> ln) & 1u) << k;
            datax |= ((SX[(4 * i + 2) * 32 + k] >> ln) & 1u) << k;
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
            if (ln == k) {
              WO[slotw + k] = word;
              WOX[slotw + k] = is_x ? wordx : 0u;
            }
          }
        }
        for (uint32_t q = t; q < num_dup * 32; q += BT) {
          const uint32_t dst = (num_ios - num_srams - num_dup) * 32 + q;
          WO[dst] = S[num_srams * 4 * 32 + q];
          WOX[dst] = SX[num_srams * 4 * 32 + q];
        }
      } else {
        // ---------------- clock-enable permutation and commit (4 words per
        // thread in flight)
        const uint32_t nq = num_ios * 32;
        for (uint32_t q0 = t; q0 < nq; q0 += 4 * BT) {
          uint32_t cp[4], cpx[4], wv[4], wx[4], old[4], oldx[4];
          size_t sg[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const uint32_t q = q0 + u * BT;
            if (q < nq) {
              const uint32_t src = perm_at(C, q);
              const uint32_t fw = (q >> 5) * 4;
              const uint32_t inv = bitmask(F[fw], q), set0 = bitmask(F[fw + 1], q),
                             dinv = bitmask(F[fw + 2], q);
              cp[u] = (WO[src] & ~set0) ^ inv;
              cpx[u] = is_x ? (WOX[src] & ~set0) : 0u;
              wv[u] = WO[q] ^ dinv;
              wx[u] = WOX[q];
              sg[u] = ((size_t)io_off * 32 + q) * L + lane;
              old[u] = ldcg(in + sg[u]);
              oldx[u] = is_x ? ldcg(in + (size_t)xsig * L + sg[u]) : 0u;
            }
          }
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const uint32_t q = q0 + u * BT;
            if (q < nq) {
              out[sg[u]] = (old[u] & ~cp[u]) | (wv[u] & cp[u]);
              if (is_x)
                out[(size_t)xsig * L + sg[u]] =
                    (oldx[u] & ~cp[u] & ~cpx[u]) | (wx[u] & cp[u] & ~cpx[u]) | cpx[u];
            }
          }
        }
      }
    }
    off += 256 + 512 * (size_t)R + STAGE_WORDS * ((size_t)ns + 2);
    if (is_last) break;
  }
}

__global__ void __launch_bounds__(BT, 1) jq_batched_kernel(BatchParams P) {
  extern __shared__ __align__(128) uint8_t dyn[];
  __shared__ Shared sh;
  uint32_t *chunks = reinterpret_cast<uint32_t *>(dyn);        // 2 x 20 KB
  uint32_t *S = chunks + 2 * STAGE_WORDS;                       // 8192
  uint32_t *SX = S + 8192;                                      // 8192
  uint32_t *WO = SX + 8192;                                     // wo_slots*32
  uint32_t *WOX = WO + P.wo_slots * 32;
  const int t = threadIdx.x;
  if (t == 0) {
    mbar_init(&sh.bar[0], 1);
    mbar_init(&sh.bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (uint32_t q = t; q < P.wo_slots * 32; q += BT) {
    WO[q] = 0;
    WOX[q] = 0;
  }
  __syncthreads();
  uint32_t uses0 = 0, uses1 = 0;
  bool failed = false;
  const size_t snap = P.sig_per_snap * P.lanes;
  const uint32_t items = P.num_blocks * P.lanes;
  for (size_t c = 0; c < P.num_cycles; ++c) {
    const uint32_t *in = (c & 1) ? P.state_b : P.state_a;
    uint32_t *out = (c & 1) ? P.state_a : P.state_b;
    // inputs of snapshot c+1 into the output buffer's input region
    if (P.stim) {
      const uint32_t *src = P.stim + (c + 1) * P.input_sigs * P.lanes;
      for (size_t q = (size_t)blockIdx.x * BT + t; q < P.input_sigs * P.lanes;
           q += (size_t)gridDim.x * BT)
        out[q] = src[q];
    }
    for (unsigned ms = 0; ms < P.num_major_stages; ++ms) {
      for (;;) {
        __syncthreads();
        if (t == 0) sh.ticket = atomicAdd(&g_ticket[P.slot], 1u);
        __syncthreads();
        const uint32_t tk = sh.ticket;
        if (tk >= items) break;
        const uint32_t blk = tk / P.lanes, lane = tk % P.lanes;
        const uint32_t *script = P.blocks_data + P.blocks_start[(size_t)ms * P.num_blocks + blk];
        run_item(P, sh, S, SX, WO, WOX, chunks, uses0, uses1, script, in, out, lane, failed);
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
      P.wave[(c * P.n_po + po) * P.lanes + l] = ldcg(out + (size_t)P.po_sig[po] * P.lanes + l);
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
  P.po_sig = a->po_signals;
  P.n_po = a->n_po;
  P.wave = a->wave;
  P.record = a->record;
  P.wo_slots = a->wo_slots ? a->wo_slots : 256;
  P.timeout = a->barrier_timeout_cycles ? a->barrier_timeout_cycles : DEFAULT_BARRIER_TIMEOUT;
  P.slot = 1;
  static const unsigned zero_u[1] = {0};
  static const int zero_i[1] = {0};
  if (cudaMemcpyToSymbolAsync(g_bar_count, zero_u, sizeof(unsigned), P.slot * sizeof(unsigned),
                              cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyToSymbolAsync(g_ticket, zero_u, sizeof(unsigned), P.slot * sizeof(unsigned),
                              cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyToSymbolAsync(g_status, zero_i, sizeof(int), P.slot * sizeof(int),
                              cudaMemcpyHostToDevice, st) != cudaSuccess)
    return JQ_ERR_LAUNCH;
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
