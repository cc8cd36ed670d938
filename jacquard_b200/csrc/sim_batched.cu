// Bit-lane batched interpreter for sm_100a: many independent stimulus streams
// run the same script in one launch.
//
// Layout: a lane word is one u32 holding one signal of 32 streams, where
// `signal` is the bit position of the plain layout (word*32 + bit) and the X
// plane of signal s is signal V + s.  The state interleaves lane groups: the
// (value, X) words of a lane pair for one signal are one 16-byte quad, or
// those of 8 lane words one 64-byte run (phys() below), so a work item reads
// or commits a signal of its lane group with one access per 16 bytes of
// adjacent threads.  In this form the boomerang 16-pair bit shuffle
// becomes a word gather and every tree position evaluates one 32-stream word:
//     v[p] = (v[p+L] ^ xa_p) & ((v[p+2L] ^ xb_p) | ob_p),  L = msb(p)
// (the plain kernel's level-0 / shared / warp / bit-level tree steps are all
// this one positional rule).  Semantics per stream are those of the plain
// interpreter (csrc/kernel_v1_impl.cuh:32-563).
//
// Work item = (script block, lane word, lane pair or lane octet) for one
// (cycle, major stage); octet items (run_item8) run compact partitions only,
// with 64-byte tree slots and writeouts named in place.  When a major stage
// has no more items than CTAs, CTA i runs item i
// (a per-launch table in shared memory holds its script offset and first
// partition); otherwise CTAs take items from a ticket counter.  Major stages
// are separated by a split grid barrier: arrive after the last commit, wait
// inside the next item once its script data is requested.  The script is
// first rewritten by jq_batched_prepare (liveness of tree positions, a
// thread-major tree form or a compact one-word-per-live-position form,
// compacted global-read slots).  Each script chunk is staged into shared
// memory with a TMA bulk copy (cp.async.bulk, mbarrier completion):
// double-buffered one chunk ahead, or for octet items all of a partition's
// chunks at once; the global read copies its slots with cp.async.  Setup/hold checks run per stream in the commit: a word's arrival
// does not depend on the stream (it follows from the script's delays and
// each script block's execution order), so the caller computes the arrival
// tables once with the plain interpreter, and only the clock-enable gate of
// the check differs between streams.
#include "sim_common.cuh"

#include <cstdio>
#include <cstdlib>

namespace jqk {

constexpr int BT = 512;  // threads per CTA
constexpr uint32_t CHUNK_BYTES = STAGE_WORDS * 4;

// Grid-barrier arrivals and work tickets of the batched kernel: 64-bit and
// monotonic within a launch (never reset between major stages).
static __device__ unsigned long long g_bcount[BAR_SLOTS];
static __device__ unsigned long long g_bticket[BAR_SLOTS];
// Arrival counts of lane-pair groups (see jq_batched_kernel): lane pairs
// never read each other's words, so when every CTA runs one item of a fixed
// lane pair, the CTAs of a lane pair synchronize only among themselves.
constexpr uint32_t MAX_GROUPS = 16;
static __device__ unsigned long long g_bgroup[BAR_SLOTS * MAX_GROUPS];

__device__ __forceinline__ unsigned long long ld_acquire64(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
// Global-read source table sentinels (jq_batched_prepare).
constexpr uint32_t GR_EMPTY = 0xffffffffu;  // needed, no source: stored as 0
constexpr uint32_t GR_SKIP = 0xfffffffeu;   // not needed by any gather

struct BatchParams {
  unsigned num_blocks, num_major_stages, lanes;
  const size_t *blocks_start;
  const uint32_t *blocks_data;
  uint32_t *sram, *sram_x;  // [stream][sram_words]
  size_t sram_words;
  size_t num_cycles;
  size_t sig_per_snap;      // effective words * 32
  int xhalf;                // X interleaved (layout 1 or 2): signals [V, 2V)
                            // are the X of [0, V)
  int layout;               // state layout (phys()): 0 pairs, 1 quads, 2 octets
  uint32_t slot_cap;        // octet items: tree slots of 64 bytes in shared memory
  size_t vsig;              // V: value signals (sig_per_snap / 2 with xhalf)
  uint32_t *state_a, *state_b;  // ping-pong snapshots, interleaved lane pairs (phys())
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
  const uint32_t *gr_sources;        // per partition: source signal of each of
                                     // the 8192 global-read positions
  // setup/hold checks (null constraints: none): [clock_ps, one u32 per state
  // word], the u16 arrival of each state word in a launch's first cycle and
  // in later cycles, the event sink
  const uint32_t *constraints;
  const uint32_t *arr_first, *arr_steady;
  jq_event_buffer *events;
  uint32_t event_cap, first_cycle;
  uint64_t timeout;        // grid-barrier wait limit (SM clocks)
  uint64_t chunk_timeout;  // script-chunk copy wait limit: fixed, so a short
                           // barrier limit never leaves a copy in flight
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

// 16-bit shuffle index q (0..8191) of a chunk in the script's own layout:
// bit k of thread T at chunk[(k>>3)*1024 + T*4 + ((k>>1)&3)], low half for
// even k (src/flatten.rs:984-1076).
__device__ __forceinline__ uint32_t perm_src(const uint32_t *chunk, uint32_t q) {
  const uint32_t T = q >> 5, k = q & 31;
  const uint32_t w = chunk[(k >> 3) * 1024 + T * 4 + ((k >> 1) & 3)];
  return (k & 1) ? (w >> 16) : (w & 0xffffu);
}
// Shuffle index q of a prepared SRAM/duplicate or clock-enable chunk:
// entries in q order, two per word.
__device__ __forceinline__ uint32_t perm_lin(const uint32_t *chunk, uint32_t q) {
  const uint32_t w = chunk[q >> 1];
  return (q & 1) ? (w >> 16) : (w & 0xffffu);
}
// Tree-state address of position p in shared memory: a bijective XOR
// swizzle that gives the 32 lanes of a warp distinct banks under the
// residue ownership map (lane bits sit at position bits 4..8).
__host__ __device__ __forceinline__ uint32_t sw(uint32_t p) { return p ^ ((p >> 4) & 31u); }
__device__ __forceinline__ uint32_t bitmask(uint32_t word, uint32_t q) {
  return 0u - ((word >> (q & 31)) & 1u);
}
// All-ones when bit `i` (a compile-time constant) of w is set.
template <int i>
__device__ __forceinline__ uint32_t mk(uint32_t w) {
  return (uint32_t)((int32_t)(w << (31 - i)) >> 31);
}
// Residue of thread t under the tree ownership map: warp w, lane l -> w | l<<4.
__host__ __device__ __forceinline__ uint32_t residue(uint32_t t) { return (t >> 5) | ((t & 31u) << 4); }
// Tree position i (0..15) of the thread with residue u: level-1..4 positions
// u + 512k, then u itself (levels 5..9, when u >= 16).
__host__ __device__ __forceinline__ uint32_t owned_pos(uint32_t u, int i) {
  return i < 8 ? 4096 + u + 512 * i
               : i < 12 ? 2048 + u + 512 * (i - 8)
                        : i < 14 ? 1024 + u + 512 * (i - 12) : i == 14 ? 512 + u : u;
}

// Word of (lane l, signal s) in the batched state, by state layout:
//   layout 1, lane-pair quads (X interleaved, signals [V, 2V) the X of
//     [0, V)): ((l >> 1) * V + s mod V) * 4 + 2 * (l & 1) + (s >= V),
//     i.e. (v_even, x_even, v_odd, x_odd) per lane pair and value signal;
//   layout 2, lane octets (X interleaved): ((l >> 3) * V + s mod V) * 16 +
//     2 * (l & 7) + (s >= V), i.e. the 64 bytes (v0, x0, ..., v7, x7) of a
//     signal for 8 lane words (256 streams) are adjacent;
//   layout 0, lane pairs without X: ((l >> 1) * sig + s) * 2 + (l & 1).
__host__ __device__ __forceinline__ size_t phys(int layout, size_t vsig, size_t sig, uint32_t l,
                                                size_t s) {
  if (layout) {
    const bool x = s >= vsig;
    const size_t sv = x ? s - vsig : s;
    if (layout == 2) return ((((size_t)(l >> 3)) * vsig + sv) << 4) + 2 * (l & 7) + (x ? 1 : 0);
    return ((((size_t)(l >> 1)) * vsig + sv) << 2) + 2 * (l & 1) + (x ? 1 : 0);
  }
  return ((((size_t)(l >> 1)) * sig + s) << 1) + (l & 1);
}
__device__ __forceinline__ size_t phys(const BatchParams &P, uint32_t l, size_t s) {
  return phys(P.layout, P.vsig, P.sig_per_snap, l, s);
}
// log2 of the words one signal of a lane group spans: 1 (pair), 2 (quad),
// 4 (octet)
__device__ __forceinline__ uint32_t sig_shift_of(const BatchParams &P) {
  return P.layout == 2 ? 4u : P.layout == 1 ? 2u : 1u;
}

constexpr uint32_t MAX_MAJOR_STAGES = 32;  // jq_simulate_batched's limit

// 32x32 bit transpose across a warp: lane l holds row l on entry and
// column l on return (bit r of the result = bit l of lane r's input), by
// swapping off-diagonal blocks of 16, 8, 4, 2 and 1 bits.
__device__ __forceinline__ uint32_t warp_transpose32(uint32_t x) {
  const uint32_t lane = threadIdx.x & 31;
  uint32_t m = 0x0000ffffu;
#pragma unroll
  for (int j = 16; j; j >>= 1, m ^= m << j) {
    const uint32_t y = __shfl_xor_sync(0xffffffffu, x, j);
    x = (lane & j) ? (x & ~m) | ((y & ~m) >> j) : (x & m) | ((y & m) << j);
  }
  return x;
}

struct Shared {
  uint32_t meta[256];
  uint64_t bar[2];
  int ok;
  uint32_t ticket;
  int dyn;  // items of this major stage come from the ticket counter
  // per major stage, resolved once per launch: its item count and, when it
  // assigns items statically (at most one per CTA), this CTA's item: script
  // offset (~0 when it has none), first partition, first partition's
  // writeout count and IO offset
  uint32_t st_items[MAX_MAJOR_STAGES];
  size_t st_off[MAX_MAJOR_STAGES];
  uint32_t st_pid[MAX_MAJOR_STAGES];
  uint32_t st_nio[MAX_MAJOR_STAGES];
  uint32_t st_io[MAX_MAJOR_STAGES];
  size_t script_words;  // blocks_start[num_major_stages * num_blocks]
  unsigned long long *bar_count;  // this CTA's grid-barrier arrival count
  uint32_t bar_size;              // CTAs that arrive on it per barrier
};

// Bytes to copy of chunk k of a partition: compact partitions list the
// used prefix of each chunk in metadata words 11 + k (0: the whole chunk).
__device__ __forceinline__ uint32_t chunk_bytes(const Shared &sh, uint32_t k) {
  const uint32_t b = (sh.meta[10] & 1u) && k < 116 ? sh.meta[11 + k] : 0u;
  return b ? b : CHUNK_BYTES;
}

// Word offset of the flag words (a uint4 per 32 entries) in a prepared
// SRAM/duplicate or clock-enable chunk of nq entries: right after the entries
// in the compact form (metadata word 10 bit 0; the chunk is copied only that
// far), at word 4096 otherwise.
__host__ __device__ __forceinline__ uint32_t perm_flag_off(uint32_t nq) {
  return ((nq >> 1) + 3) & ~3u;
}
__device__ __forceinline__ const uint4 *perm_flags(const Shared &sh, const uint32_t *C,
                                                   uint32_t nq) {
  return reinterpret_cast<const uint4 *>(C + ((sh.meta[10] & 1u) ? perm_flag_off(nq) : 4096u));
}

// Grid barrier between major stages, split in two so a CTA can load its
// next item's script data between arriving and waiting.  The arrival count
// is 64-bit and monotonic within a launch (the target grows by the grid each
// barrier).  Arrive: a release reduction (this CTA's writes, ordered by the
// CTA barrier, become visible before the count moves), which thread 0 does
// not wait for.  Wait: thread 0 polls the count with acquire loads until it
// reaches the target, and the error status; the other warps run
// `others(i, n)` (i = 0..n-1) meanwhile.  The CTA learns the outcome; false
// when the barrier failed.
__device__ __forceinline__ void prefetch_l2(const void *p) {
  asm volatile("prefetch.L2 [%0];" ::"l"(p));
}

__device__ __forceinline__ void grid_arrive(const Shared &sh, unsigned long long &bar_target) {
  __syncthreads();
  if (threadIdx.x == 0) {
    bar_target += sh.bar_size;
    asm volatile("red.release.gpu.global.add.u64 [%0], 1;" ::"l"(sh.bar_count) : "memory");
  }
}

template <class F>
__device__ bool grid_wait(const BatchParams &P, Shared &sh, unsigned long long bar_target,
                          F &&others) {
  const int t = threadIdx.x;
  if (t >= 32) others((uint32_t)t - 32, (uint32_t)BT - 32);
  if (t == 0) {
    int ok = 1;
    uint64_t t0 = clock64();
    while (ld_acquire64(sh.bar_count) < bar_target) {
      if (*((volatile int *)&g_status[P.slot]) != 0) {
        ok = 0;
        break;
      }
      __nanosleep(64);
      if ((uint64_t)(clock64() - t0) > P.timeout) {
        ok = 0;
        atomicExch(&g_status[P.slot], JQ_ERR_BARRIER_TIMEOUT);
        break;
      }
    }
    sh.ok = ok;
  }
  __syncthreads();
  return sh.ok != 0;
}

// One event record (csrc/event_buffer.h Event) at index idx of the sink;
// `reserved` carries the stream.  Past the capacity only the overflow flag.
__device__ __forceinline__ void put_event(const BatchParams &P, uint32_t idx, uint32_t type,
                                          uint32_t word, uint32_t cycle, uint32_t slack,
                                          uint32_t arr, uint32_t cv, uint32_t stream) {
  if (idx < P.event_cap) {
    jq_event *e = &P.events->events[idx];
    e->event_type = type;
    e->message_id = word;
    e->cycle = cycle;
    e->reserved = stream;
    e->data[0] = word;
    e->data[1] = slack;
    e->data[2] = arr;
    e->data[3] = cv;
  } else {
    atomicExch(&P.events->overflow, 1u);
  }
}

// Setup/hold check of state word `word` for the streams of lane words l0 and
// l1 (bit masks m0, m1: the streams whose clock enable is set on any signal
// of the word), with the same predicate as the plain interpreter
// (csrc/kernel_v1_impl.cuh:536-558) applied per stream: the word's arrival
// does not depend on the stream, its clock enable does.  Called by a whole
// warp with the same arguments; lane j writes the records of stream bit j.
__device__ void check_word(const BatchParams &P, uint32_t word, uint32_t m0, uint32_t l0,
                           uint32_t m1, uint32_t l1, uint32_t cycle, bool first) {
  if (!(m0 | m1)) return;
  const uint32_t cv = __ldg(P.constraints + 1 + word);
  if (!cv) return;
  const uint32_t a = __ldg((first ? P.arr_first : P.arr_steady) + word) & 0xffffu;
  const uint32_t clock_ps = __ldg(P.constraints);
  const uint32_t su = cv >> 16, ho = cv & 0xffffu;
  const uint32_t lane = threadIdx.x & 31, below = (1u << lane) - 1u;
  const uint32_t n0 = __popc(m0), n = n0 + __popc(m1);
#pragma unroll
  for (int kind = 0; kind < 2; ++kind) {
    const bool v = kind == 0 ? (a > 0 && a + su > clock_ps) : (a < ho);
    if (!v) continue;
    const uint32_t type = kind == 0 ? 4u : 5u;
    const uint32_t slack = kind == 0 ? (uint32_t)((int32_t)clock_ps - (int32_t)a - (int32_t)su)
                                     : (uint32_t)((int32_t)a - (int32_t)ho);
    const uint32_t c = kind == 0 ? su : ho;
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(&P.events->count, n);
    base = __shfl_sync(0xffffffffu, base, 0);
    if ((m0 >> lane) & 1u)
      put_event(P, base + __popc(m0 & below), type, word, cycle, slack, a, c, 32 * l0 + lane);
    if ((m1 >> lane) & 1u)
      put_event(P, base + n0 + __popc(m1 & below), type, word, cycle, slack, a, c, 32 * l1 + lane);
  }
}

// One (block, lane) work item: the block's partition list for one lane word.
// Tree state and writeouts hold (value, X) pairs so one shared-memory access
// moves both.  The script is in the prepared layout (jq_batched_prepare):
//   boomerang chunk: words [0, 4096) two uint4 planes [2][512 threads], the
//     thread's 16 gather sources (level-1 inputs a then b, already swizzled,
//     with the liveness bits of the prepare step);
//     words [4096, 5120) one uint2 per thread: xa bits 0..15 | xb bits 16..31,
//     ob bits 0..15 of its 16 owned positions, then bits 16..31 the store
//     mask of those positions, except that in deep stages warp-0 threads
//     t < 8 hold there the flags of tree positions 8+t, 4+t, 2+t, 1+t
//     (levels 10..13) at bits 16+m (xa), 20+m (xb), 24+m (ob);
//   SRAM/duplicate and clock-enable chunks: shuffle entries in q order,
//     flags unchanged.
// With `ds` the tree state is double-buffered (stage ci reads buffer ci&1 and
// writes the other), which removes the barrier between gather and overwrite.
template <bool DS>
__device__ void run_item(const BatchParams &P, Shared &sh, uint2 *S, uint2 *WO, uint32_t *chunks,
                         uint32_t &uses0, uint32_t &uses1, const uint32_t *script,
                         const uint32_t *in, uint32_t *out, uint32_t lane, uint32_t pid0,
                         bool &failed, unsigned long long &next_ticket, bool &have_next,
                         uint32_t cyc) {
  const int t = threadIdx.x;
  // the lane's words: with xhalf (v, x) pairs at 4 * (pair * V + s) + 2 * odd
  // (X-capable partitions always run in the quad layout), else values at
  // 2 * (pair * sig + s) + odd
  const size_t lane_base = P.xhalf ? (((size_t)(lane >> 1) * P.vsig) << 2) + 2 * (lane & 1)
                                   : (((size_t)(lane >> 1) * P.sig_per_snap) << 1) + (lane & 1);
  const uint32_t sig_shift = P.xhalf ? 2 : 1;
  constexpr bool ds = DS;
  uint2 *const Sb0 = S;
  uint2 *const Sb1 = ds ? S + 8192 : S;
  size_t off = 0;
  uint32_t pid = pid0;
  for (;;) {
    __syncthreads();
    const long long t_start = clock64();
    if (t < 256) sh.meta[t] = __ldg(script + off + t);
    // global-read sources of this partition (only used when it exists)
    uint32_t e[16];
    {
      const uint32_t *src = P.gr_sources + (size_t)pid * 8192;
#pragma unroll
      for (int k = 0; k < 16; ++k) e[k] = __ldg(src + t + BT * k);
    }
    __syncthreads();
    const uint32_t ns = sh.meta[0];
    if (!ns) break;
    const uint32_t is_last = sh.meta[1], num_ios = sh.meta[2], io_off = sh.meta[3];
    const uint32_t num_srams = sh.meta[4], sram_off = sh.meta[5], R = sh.meta[6];
    const uint32_t num_dup = sh.meta[7];
    const bool is_x = sh.meta[8] != 0;
    const uint32_t *gr = script + off + 256;
    const uint32_t *ch0 = gr + 512 * (size_t)R;
    // chunk sequence: the ns boomerang stages, the SRAM/duplicate chunk
    // (only when the partition has SRAMs or duplicates), the clock-enable chunk
    const bool has_sram = (num_srams | num_dup) != 0;
    const uint32_t nchunks = ns + (has_sram ? 2 : 1);

    // chunk 0 -> buffer 0 (the previous item/partition finished with both)
    if (t == 0) {
      const uint32_t nb = chunk_bytes(sh, 0);
      mbar_expect_tx(&sh.bar[0], nb);
      tma_load_1d(chunks, ch0, nb, &sh.bar[0]);
    }

    // ---- global read into tree buffer 0.  The source signal of every
    // position (the kernel's bit-append order, resolved once per script by
    // jq_batched_prepare; bit 31 = current-cycle staged IO, GR_EMPTY = none,
    // GR_SKIP = read by no needed gather) was loaded at the top of the
    // partition; up to 32 independent state loads per thread follow.
    {
      uint32_t v[16], vx[16];
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        v[k] = 0;
        vx[k] = 0;
        if (e[k] < GR_SKIP) {
          const uint32_t *base = (e[k] >> 31) ? out : in;
          const size_t w = lane_base + ((size_t)(e[k] & 0x7fffffffu) << sig_shift);
          if (P.xhalf) {
            const uint2 q = __ldcg(reinterpret_cast<const uint2 *>(base + w));
            v[k] = q.x;
            vx[k] = is_x ? q.y : 0u;
          } else {
            v[k] = ldcg(base + w);
          }
        }
      }
#pragma unroll
      for (int k = 0; k < 16; ++k)
        if (e[k] != GR_SKIP) Sb0[sw(t + BT * k)] = make_uint2(v[k], vx[k]);
    }

    // Thread -> tree residue map: thread (warp w, lane l) owns positions whose
    // value mod 512 is u = w | l << 4.  Levels 1..4 then read only the
    // thread's own registers, levels 5..9 read lanes of the same warp
    // (residue bits 4..8 are lane bits), and only positions 1..15 need one
    // exchange through shared memory.  Under the swizzle every owned
    // position p = base + u has address base + us.
    const uint32_t lane_i = t & 31, warp_i = t >> 5;
    const uint32_t u = residue(t);
    const uint32_t us = sw(u);
    // writeout hook (stage << 8 | 32-position group) of slot warp_i + 16 *
    // lane_i (lanes 0..15; num_ios <= 256), all ones when there is none
    uint32_t my_hook = 0xffffffffu;
    if (lane_i < 16 && warp_i + 16 * lane_i < num_ios) {
      const uint32_t slot = warp_i + 16 * lane_i;
      const uint32_t hw = sh.meta[128 + slot / 2];
      my_hook = (slot & 1) ? (hw >> 16) : (hw & 0xffffu);
    }
    // compact form (jq_batched_prepare): stages as dense slot lists, hooks
    // naming 32-slot blocks of the stage's region
    const bool compact = sh.meta[10] & 1u;
    uint32_t prev_base = 0;
    for (uint32_t ci = 0; ci < nchunks; ++ci) {
      const uint32_t b = ci & 1;
      uint32_t *C = chunks + b * STAGE_WORDS;
      if (ci == 0) __syncthreads();  // global read complete
      // The other buffer's last reader finished before the final barrier of
      // the previous chunk, so the next chunk can be issued right away.
      if (t == 0 && ci + 1 < nchunks) {
        const uint32_t nxt = (!has_sram && ci + 1 == ns) ? ns + 1 : ci + 1;  // script chunk
        const uint32_t nb = chunk_bytes(sh, nxt);
        mbar_expect_tx(&sh.bar[b ^ 1], nb);
        tma_load_1d(chunks + (b ^ 1) * STAGE_WORDS, ch0 + (size_t)STAGE_WORDS * nxt, nb,
                    &sh.bar[b ^ 1]);
      }
      uint32_t &uses = b ? uses1 : uses0;
      // warp-uniform, so the shuffles below run with full warps
      const bool ok = __all_sync(0xffffffffu, mbar_wait(&sh.bar[b], uses & 1u, P.chunk_timeout));
      ++uses;
      // a chunk never arrived: every thread leaves together, after letting
      // the copy still in flight into the other buffer land
#define JQ_FAIL_IF(cond)                                               \
  if (__syncthreads_or(cond)) {                                        \
    failed = true;                                                     \
    if (t == 0 && ci + 1 < nchunks)                                    \
      mbar_wait(&sh.bar[b ^ 1], (b ? uses0 : uses1) & 1u, P.chunk_timeout);  \
    return;                                                            \
  }
      // hooks of a compact stage: 32-slot blocks of its region
#define JQ_HOOKS_COMPACT(stage, pbase)                                                        \
  for (uint32_t hm = __ballot_sync(0xffffffffu, (my_hook >> 8) == (stage)); hm; hm &= hm - 1) { \
    const uint32_t j = __ffs(hm) - 1;                                                         \
    const uint32_t blk = __shfl_sync(0xffffffffu, my_hook, j) & 255u;                         \
    WO[(warp_i + 16 * j) * 32 + lane_i] = Sb0[(pbase) + 32 * blk + lane_i];                   \
  }
      if (compact && ci == ns && ok) JQ_HOOKS_COMPACT(ns - 1, prev_base)
      if (ci < ns && compact) {
        // ---------------- compact stage ci: one word per live position; it
        // reads the previous region and writes its own, disjoint one, so one
        // barrier per stage (a stage-0 region that overlaps the global read
        // is computed in full before it is stored)
        const uint32_t n = ok ? C[0] : 0u, base = ok ? C[1] : 0u;
#define JQ_COMPACT_EVAL(i, r)                                                              \
  {                                                                                        \
    const uint32_t en = C[4 + (i)];                                                              \
    const uint2 ga = ((en >> 29) & 1u) ? make_uint2(0, 0) : Sb0[en & 8191u];               \
    const uint2 gb = ((en >> 30) & 1u) ? make_uint2(0, 0) : Sb0[(en >> 13) & 8191u];       \
    xand(ga.x, ga.y, gb.x, gb.y, 0u - ((en >> 26) & 1u), 0u - ((en >> 27) & 1u),           \
         0u - ((en >> 28) & 1u), r.x, r.y);                                                \
  }
        // slots below ov (stage 0 only, at most 4 * BT) lie over the global
        // read: held in registers until every thread has gathered
        const uint32_t ov = ok ? C[2] : 0u;
        uint2 h[4] = {make_uint2(0, 0), make_uint2(0, 0), make_uint2(0, 0), make_uint2(0, 0)};
        if (ok) {
          if (ci > 0) JQ_HOOKS_COMPACT(ci - 1, prev_base)
          // n <= 4096 slots: at most 8 per thread
#pragma unroll
          for (int k = 0; k < 8; ++k) {
            const uint32_t i = t + BT * k;
            if (i >= n) break;
            uint2 r;
            JQ_COMPACT_EVAL(i, r)
            if (k < 4 && i < ov)
              h[k < 4 ? k : 0] = r;
            else
              Sb0[base + i] = r;
          }
        }
        JQ_FAIL_IF(!ok)
        if (ov) {
#pragma unroll
          for (int k = 0; k < 4; ++k)
            if (t + BT * k < ov) Sb0[base + t + BT * k] = h[k];
          __syncthreads();
        }
#undef JQ_COMPACT_EVAL
        prev_base = base;
      } else if (ci < ns) {
        // ---------------- boomerang stage ci
        const uint2 *Sp = (ci & 1) ? Sb1 : Sb0;
        uint2 *Sn = (ci & 1) ? Sb0 : Sb1;
        uint2 ga[8], gb[8];
        uint32_t A = 0, B = 0, sm = 0;
        // no position below 512 live: levels 5..13 are skipped (uniform:
        // every thread's entry 0 carries it)
        bool shallow = false, flat = false;
        if (ok) {
          const uint4 *P4 = reinterpret_cast<const uint4 *>(C);
          const uint4 pa = P4[t], pb = P4[BT + t];
          const uint2 fl = reinterpret_cast<const uint2 *>(C + 4096)[t];
          A = fl.x;
          B = fl.y;
          shallow = (pa.x >> 13) & 1u;
          flat = (pa.x >> 29) & 1u;  // only level 1, only positions read from outside
          sm = t < 8 && !shallow ? 0xffffu : (B >> 16);  // owned positions to store
          // gathers the prepared liveness marks as not needed read nothing
#define JQ_G(dst, w, h) \
  dst = (((w) >> (16 * (h) + 15)) & 1u) ? Sp[((w) >> (16 * (h))) & 0x1fffu] : make_uint2(0, 0);
          JQ_G(ga[0], pa.x, 0) JQ_G(ga[1], pa.x, 1) JQ_G(ga[2], pa.y, 0) JQ_G(ga[3], pa.y, 1)
          JQ_G(ga[4], pa.z, 0) JQ_G(ga[5], pa.z, 1) JQ_G(ga[6], pa.w, 0) JQ_G(ga[7], pa.w, 1)
          JQ_G(gb[0], pb.x, 0) JQ_G(gb[1], pb.x, 1) JQ_G(gb[2], pb.y, 0) JQ_G(gb[3], pb.y, 1)
          JQ_G(gb[4], pb.z, 0) JQ_G(gb[5], pb.z, 1) JQ_G(gb[6], pb.w, 0) JQ_G(gb[7], pb.w, 1)
#undef JQ_G
        }
        if (!ds) {
          // single buffer: all gathers done before the in-place overwrite
          JQ_FAIL_IF(!ok)
        }
        if (ok && flat) {
#define JQ_F1(k)                                                                     \
  if ((sm >> (k)) & 1u) {                                                            \
    uint32_t v, x;                                                                   \
    xand(ga[k].x, ga[k].y, gb[k].x, gb[k].y, mk<k>(A), mk<16 + k>(A), mk<k>(B), v, x); \
    Sn[4096 + 512 * k + us] = make_uint2(v, x);                                      \
  }
          JQ_F1(0) JQ_F1(1) JQ_F1(2) JQ_F1(3) JQ_F1(4) JQ_F1(5) JQ_F1(6) JQ_F1(7)
#undef JQ_F1
          if (t == 0) Sn[0] = make_uint2(0, 0);
        } else if (ok) {
          // level 1 (positions 4096 + u + 512k); owned position i is stored
          // only when read from outside its stage (bit i of sm)
          uint32_t v1[8], x1[8];
#define JQ_L1(k)                                                                         \
  xand(ga[k].x, ga[k].y, gb[k].x, gb[k].y, mk<k>(A), mk<16 + k>(A), mk<k>(B), v1[k], x1[k]); \
  if (((sm >> (k)) & 1u)) Sn[4096 + 512 * k + us] = make_uint2(v1[k], x1[k]);
          JQ_L1(0) JQ_L1(1) JQ_L1(2) JQ_L1(3) JQ_L1(4) JQ_L1(5) JQ_L1(6) JQ_L1(7)
#undef JQ_L1
          uint32_t v2[4], x2[4];
#define JQ_L2(k)                                                                           \
  xand(v1[k], x1[k], v1[k + 4], x1[k + 4], mk<8 + k>(A), mk<24 + k>(A), mk<8 + k>(B), v2[k], \
       x2[k]);                                                                             \
  if (((sm >> (8 + k)) & 1u)) Sn[2048 + 512 * k + us] = make_uint2(v2[k], x2[k]);
          JQ_L2(0) JQ_L2(1) JQ_L2(2) JQ_L2(3)
#undef JQ_L2
          uint32_t v3[2], x3[2];
          xand(v2[0], x2[0], v2[2], x2[2], mk<12>(A), mk<28>(A), mk<12>(B), v3[0], x3[0]);
          if (((sm >> 12) & 1u)) Sn[1024 + us] = make_uint2(v3[0], x3[0]);
          xand(v2[1], x2[1], v2[3], x2[3], mk<13>(A), mk<29>(A), mk<13>(B), v3[1], x3[1]);
          if (((sm >> 13) & 1u)) Sn[1536 + us] = make_uint2(v3[1], x3[1]);
          uint32_t v4, x4;
          xand(v3[0], x3[0], v3[1], x3[1], mk<14>(A), mk<30>(A), mk<14>(B), v4, x4);
          if (((sm >> 14) & 1u)) Sn[512 + us] = make_uint2(v4, x4);
          if (shallow) {
            if (t == 0) Sn[0] = make_uint2(0, 0);
          } else {
            // levels 5..9: the thread's position u (u >= 16) at the level of
            // its lane: level 5 (lanes 16..31) from level-4 residues u-256
            // (lane ^ 16) and u; level 6+k' (lanes [2^k, 2^(k+1))) from lanes
            // l + 2^k and l + 2^(k+1)
            const uint32_t XA = mk<15>(A), XB = mk<31>(A), OB = mk<15>(B);
            uint32_t cv, cx;
            {
              const uint32_t a = __shfl_xor_sync(0xffffffffu, v4, 16);
              const uint32_t ax = __shfl_xor_sync(0xffffffffu, x4, 16);
              xand(a, ax, v4, x4, XA, XB, OB, cv, cx);
              if (lane_i >= 16) Sn[us] = make_uint2(cv, cx);
            }
#pragma unroll
            for (int k = 3; k >= 0; --k) {
              const uint32_t d = 1u << k;
              const uint32_t a = __shfl_sync(0xffffffffu, cv, (lane_i + d) & 31);
              const uint32_t bb = __shfl_sync(0xffffffffu, cv, (lane_i + 2 * d) & 31);
              const uint32_t ax = __shfl_sync(0xffffffffu, cx, (lane_i + d) & 31);
              const uint32_t bx = __shfl_sync(0xffffffffu, cx, (lane_i + 2 * d) & 31);
              if (lane_i >= d && lane_i < 2 * d) {
                xand(a, ax, bb, bx, XA, XB, OB, cv, cx);
                Sn[us] = make_uint2(cv, cx);
              }
            }
          }
        }
        JQ_FAIL_IF(!ok)
        if (!shallow) {
          // levels 10..13 (positions 15..1) in warp 0 from positions 16..31
          if (t < 32) {
            uint2 h = t < 16 ? Sn[sw(16 + t)] : make_uint2(0, 0);
            uint32_t hv = h.x, hx = h.y;
            // rolled: this serial section runs in one warp, keep its code short
#pragma unroll 1
            for (int m = 0; m < 4; ++m) {
              const uint32_t len = 8u >> m;
              const uint32_t bb = __shfl_sync(0xffffffffu, hv, (t + len) & 31);
              const uint32_t bx = __shfl_sync(0xffffffffu, hx, (t + len) & 31);
              if ((uint32_t)t < len) {
                uint32_t r, rx;
                xand(hv, hx, bb, bx, 0u - ((B >> (16 + m)) & 1u), 0u - ((B >> (20 + m)) & 1u),
                     0u - ((B >> (24 + m)) & 1u), r, rx);
                Sn[len + t] = make_uint2(r, rx);
                hv = r;
                hx = rx;
              }
            }
            if (t == 0) Sn[0] = make_uint2(0, 0);
          }
          __syncthreads();
        }
        // writeout hooks of this stage: warp w copies those of slots w,
        // w+16, ... (lane j holds slot w+16j's hook)
        for (uint32_t hm = __ballot_sync(0xffffffffu, (my_hook >> 8) == ci); hm; hm &= hm - 1) {
          const uint32_t j = __ffs(hm) - 1;
          const uint32_t g = __shfl_sync(0xffffffffu, my_hook, j) & 255u;
          WO[(warp_i + 16 * j) * 32 + lane_i] = Sn[sw(g * 32 + lane_i)];
        }
      } else if (has_sram && ci == ns) {
        // ---------------- SRAM & duplicate permutation + SRAM ports
        JQ_FAIL_IF(!ok)  // hooks done, chunk landed
        uint2 *St = Sb0;  // staging (the last stage's hooks are done)
        const uint32_t nq = (num_srams * 4 + num_dup) * 32;
        const uint4 *F4 = perm_flags(sh, C, nq);
        for (uint32_t q = t; q < nq; q += BT) {
          const uint2 w = WO[perm_lin(C, q)];
          const uint4 fl = F4[q >> 5];
          const uint32_t inv = bitmask(fl.x, q), set0 = bitmask(fl.y, q);
          St[q] = make_uint2((w.x & ~set0) ^ inv, is_x ? (w.y & ~set0) : 0u);
        }
        __syncthreads();
        // one warp per SRAM, lane = stream within the lane word
        const int warp = t >> 5, ln = t & 31;
        for (uint32_t i = warp; i < num_srams; i += BT / 32) {
          const uint2 *Aw = St + (4 * i) * 32;
          // staged rows (read address 0..15, write address 16..31, write
          // enable 32..63, data 64..95) to per-stream bits by warp transposes
          const uint32_t addr = warp_transpose32(Aw[ln].x);
          const uint32_t ra = addr & 0xffffu, wa = addr >> 16;
          const uint32_t en = warp_transpose32(Aw[32 + ln].x);
          const uint2 dk = Aw[64 + ln];
          const uint32_t data = warp_transpose32(dk.x), datax = warp_transpose32(dk.y);
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
          WO[slotw + ln] = make_uint2(warp_transpose32(r), is_x ? warp_transpose32(rx) : 0u);
        }
        for (uint32_t q = t; q < num_dup * 32; q += BT)
          WO[(num_ios - num_srams - num_dup) * 32 + q] = St[num_srams * 4 * 32 + q];
        __syncthreads();
      } else {
        // ---------------- clock-enable permutation and commit
        JQ_FAIL_IF(!ok)
        // the item's last commit: take the next work ticket now, so its
        // latency overlaps the commit
        if (t == 0 && is_last && sh.dyn) {
          next_ticket = atomicAdd(&g_bticket[P.slot], 1ull);
          have_next = true;
        }
        const uint32_t nq = num_ios * 32;
        const uint4 *F4 = perm_flags(sh, C, nq);
        // the old word is loaded only by warps where some stream of their
        // state word keeps its value (clock enable clear): none, when every
        // enable is set
        for (uint32_t q = t; q < nq; q += BT) {  // warp-uniform bound
          const uint2 src = WO[perm_lin(C, q)];
          const uint4 fl = F4[q >> 5];
          const uint32_t inv = bitmask(fl.x, q), set0 = bitmask(fl.y, q), dinv = bitmask(fl.z, q);
          const uint2 me = WO[q];
          const uint32_t cp = (src.x & ~set0) ^ inv, cpx = is_x ? (src.y & ~set0) : 0u;
          if (P.constraints)  // a warp holds the 32 signals of one word
            check_word(P, io_off + (q >> 5), __reduce_or_sync(0xffffffffu, cp), lane, 0u, 0u,
                       P.first_cycle + cyc, cyc == 0);
          const size_t sg = lane_base + (((size_t)io_off * 32 + q) << sig_shift);
          uint32_t old = 0, oldx = 0;
          if (__any_sync(0xffffffffu, cp != 0xffffffffu)) {
            if (is_x) {  // quad layout: (v, x) adjacent
              const uint2 o = __ldcg(reinterpret_cast<const uint2 *>(in + sg));
              old = o.x;
              oldx = o.y;
            } else {
              old = ldcg(in + sg);
            }
          }
          const uint32_t nv = (old & ~cp) | ((me.x ^ dinv) & cp);
          if (is_x)
            *reinterpret_cast<uint2 *>(out + sg) =
                make_uint2(nv, (oldx & ~cp & ~cpx) | (me.y & cp & ~cpx) | cpx);
          else
            out[sg] = nv;
        }
      }
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
#undef JQ_FAIL_IF
#undef JQ_HOOKS_COMPACT

// X-propagating AND of two lane words at once: (v0, x0, v1, x1) operands.
__device__ __forceinline__ uint4 xand2(uint4 a, uint4 b, uint32_t xa, uint32_t xb, uint32_t ob) {
  uint4 r;
  xand(a.x, a.y, b.x, b.y, xa, xb, ob, r.x, r.y);
  xand(a.z, a.w, b.z, b.w, xa, xb, ob, r.z, r.w);
  return r;
}
__device__ __forceinline__ uint4 shfl4(uint4 v, uint32_t src) {
  return make_uint4(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src),
                    __shfl_sync(0xffffffffu, v.z, src), __shfl_sync(0xffffffffu, v.w, src));
}
__device__ __forceinline__ uint4 shfl4_xor(uint4 v, uint32_t m) {
  return make_uint4(__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m),
                    __shfl_xor_sync(0xffffffffu, v.z, m), __shfl_xor_sync(0xffffffffu, v.w, m));
}

// A lane-pair work item: the block's partition list for lane words 2lp and
// 2lp+1 together.  Same steps as run_item; every tree position, writeout and
// staged word holds (v0, x0, v1, x1), so the script chunks, the flag masks,
// the barriers and the load latencies of a stage are shared by both lane
// words.  The tree state is single-buffered (128 KB), so a barrier separates
// the gathers of a stage from its first writes.
__device__ void run_item2(const BatchParams &P, Shared &sh, uint4 *S, uint4 *WO, uint32_t *chunks,
                          uint32_t &uses0, uint32_t &uses1, const uint32_t *script,
                          const uint32_t *in, uint32_t *out, uint32_t lp, uint32_t pid0,
                          bool &failed, unsigned long long &next_ticket, bool &have_next,
                          bool &pending, unsigned long long &bar_target, uint32_t cyc) {
  const int t = threadIdx.x;
  // the pair's words: quads (v0, x0, v1, x1) at 4 * (lp * V + s) with
  // xhalf, else (v0, v1) at 2 * (lp * sig + s)
  const size_t pair_base = P.xhalf ? ((size_t)lp * P.vsig) << 2 : ((size_t)lp * P.sig_per_snap) << 1;
  size_t off = 0;
  uint32_t pid = pid0;
  for (;;) {
    __syncthreads();
    // per-partition timing (part_cycles) counts the item's own work: from
    // its start, or from the end of the barrier wait it took over
    long long t_start = clock64();
    if (t < 256) sh.meta[t] = __ldg(script + off + t);
    uint32_t e[16];
    {
      const uint32_t *src = P.gr_sources + (size_t)pid * 8192;
#pragma unroll
      for (int k = 0; k < 16; ++k) e[k] = __ldg(src + t + BT * k);
    }
    __syncthreads();
    const uint32_t ns = sh.meta[0];
    if (!ns) break;
    const uint32_t is_last = sh.meta[1], num_ios = sh.meta[2], io_off = sh.meta[3];
    const uint32_t num_srams = sh.meta[4], sram_off = sh.meta[5], R = sh.meta[6];
    const uint32_t num_dup = sh.meta[7];
    const bool is_x = sh.meta[8] != 0;
    const uint32_t *ch0 = script + off + 256 + 512 * (size_t)R;
    const bool has_sram = (num_srams | num_dup) != 0;
    const uint32_t nchunks = ns + (has_sram ? 2 : 1);
    if (t == 0) {
      const uint32_t nb = chunk_bytes(sh, 0);
      mbar_expect_tx(&sh.bar[0], nb);
      tma_load_1d(chunks, ch0, nb, &sh.bar[0]);
    }
    // the wait of the grid barrier that ends the previous major stage (the
    // CTA arrived before this item), deferred to here so the metadata,
    // global-read sources and chunk 0 (script data, never written) are on
    // their way meanwhile; the waiting warps prefetch the commit rows
    if (pending) {
      pending = false;
      const uint32_t *rows = in + pair_base + (((size_t)io_off * 32) << (P.xhalf ? 2 : 1));
      const uint32_t nl = num_ios * (P.xhalf ? 4 : 2);  // 128-byte lines
      if (!grid_wait(P, sh, bar_target, [&](uint32_t i0, uint32_t n) {
            for (uint32_t l = i0; l < nl; l += n) prefetch_l2(rows + 32 * (size_t)l);
          })) {
        failed = true;
        if (t == 0) mbar_wait(&sh.bar[0], uses0 & 1u, P.chunk_timeout);
        return;
      }
      t_start = clock64();
    }
    // ---- global read, both lane words.  X-capable partitions of the quad
    // layout copy each slot's 16 bytes straight into shared memory with
    // cp.async (L2 only, so words other SMs wrote before the barrier are
    // seen), all 16 slots in flight at once; the others load through
    // registers in two halves of 8 positions.
    if (P.xhalf && is_x) {
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        const uint32_t ek = e[k];
        uint4 *dst = &S[sw(t + BT * k)];
        if (ek < GR_SKIP) {
          const uint32_t *bp = (ek >> 31) ? out : in;
          const uint32_t *src = bp + pair_base + ((size_t)(ek & 0x7fffffffu) << 2);
          asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src)
                       : "memory");
        } else if (ek == GR_EMPTY) {
          *dst = make_uint4(0, 0, 0, 0);
        }
      }
      asm volatile("cp.async.wait_all;" ::: "memory");
    } else {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      uint4 v[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const uint32_t ek = e[8 * h + k];
        v[k] = make_uint4(0, 0, 0, 0);
        if (ek < GR_SKIP) {
          const uint32_t *bp = (ek >> 31) ? out : in;
          const size_t sg = ek & 0x7fffffffu;
          if (P.xhalf) {
            v[k] = __ldcg(reinterpret_cast<const uint4 *>(bp + pair_base + (sg << 2)));
            if (!is_x) v[k].y = v[k].w = 0u;
          } else {
            const uint2 q = __ldcg(reinterpret_cast<const uint2 *>(bp + pair_base + (sg << 1)));
            v[k].x = q.x;
            v[k].z = q.y;
          }
        }
      }
#pragma unroll
      for (int k = 0; k < 8; ++k)
        if (e[8 * h + k] != GR_SKIP) S[sw(t + BT * (8 * h + k))] = v[k];
    }
    }
    const uint32_t lane_i = t & 31, warp_i = t >> 5;
    const uint32_t u = residue(t);
    const uint32_t us = sw(u);
    // writeout hook (stage << 8 | 32-position group) of slot warp_i + 16 *
    // lane_i (lanes 0..15; num_ios <= 256), all ones when there is none
    uint32_t my_hook = 0xffffffffu;
    if (lane_i < 16 && warp_i + 16 * lane_i < num_ios) {
      const uint32_t slot = warp_i + 16 * lane_i;
      const uint32_t hw = sh.meta[128 + slot / 2];
      my_hook = (slot & 1) ? (hw >> 16) : (hw & 0xffffu);
    }
    // compact form (jq_batched_prepare): stages as dense slot lists, hooks
    // naming 32-slot blocks of the stage's region
    const bool compact = sh.meta[10] & 1u;
    uint32_t prev_base = 0;
    for (uint32_t ci = 0; ci < nchunks; ++ci) {
      const uint32_t b = ci & 1;
      uint32_t *C = chunks + b * STAGE_WORDS;
      if (ci == 0) __syncthreads();  // global read complete
      if (t == 0 && ci + 1 < nchunks) {
        const uint32_t nxt = (!has_sram && ci + 1 == ns) ? ns + 1 : ci + 1;
        const uint32_t nb = chunk_bytes(sh, nxt);
        mbar_expect_tx(&sh.bar[b ^ 1], nb);
        tma_load_1d(chunks + (b ^ 1) * STAGE_WORDS, ch0 + (size_t)STAGE_WORDS * nxt, nb,
                    &sh.bar[b ^ 1]);
      }
      uint32_t &uses = b ? uses1 : uses0;
      const bool ok = __all_sync(0xffffffffu, mbar_wait(&sh.bar[b], uses & 1u, P.chunk_timeout));
      ++uses;
#define JQ_FAIL_IF(cond)                                               \
  if (__syncthreads_or(cond)) {                                        \
    failed = true;                                                     \
    if (t == 0 && ci + 1 < nchunks)                                    \
      mbar_wait(&sh.bar[b ^ 1], (b ? uses0 : uses1) & 1u, P.chunk_timeout);  \
    return;                                                            \
  }
#define JQ_HOOKS_COMPACT(stage, pbase)                                                        \
  for (uint32_t hm = __ballot_sync(0xffffffffu, (my_hook >> 8) == (stage)); hm; hm &= hm - 1) { \
    const uint32_t j = __ffs(hm) - 1;                                                         \
    const uint32_t blk = __shfl_sync(0xffffffffu, my_hook, j) & 255u;                         \
    WO[(warp_i + 16 * j) * 32 + lane_i] = S[(pbase) + 32 * blk + lane_i];                     \
  }
      if (compact && ci == ns && ok) JQ_HOOKS_COMPACT(ns - 1, prev_base)
      if (ci < ns && compact) {
        // ---------------- compact stage ci (see run_item)
        const uint32_t n = ok ? C[0] : 0u, base = ok ? C[1] : 0u;
#define JQ_COMPACT_EVAL(i, r)                                                                \
  {                                                                                          \
    const uint32_t en = C[4 + (i)];                                                                \
    const uint4 ga = ((en >> 29) & 1u) ? make_uint4(0, 0, 0, 0) : S[en & 8191u];             \
    const uint4 gb = ((en >> 30) & 1u) ? make_uint4(0, 0, 0, 0) : S[(en >> 13) & 8191u];     \
    r = xand2(ga, gb, 0u - ((en >> 26) & 1u), 0u - ((en >> 27) & 1u), 0u - ((en >> 28) & 1u)); \
  }
        const uint32_t ov = ok ? C[2] : 0u;  // held slots (stage 0)
        uint4 h[4] = {make_uint4(0, 0, 0, 0), make_uint4(0, 0, 0, 0), make_uint4(0, 0, 0, 0), make_uint4(0, 0, 0, 0)};
        if (ok) {
          if (ci > 0) JQ_HOOKS_COMPACT(ci - 1, prev_base)
          // n <= 4096 slots: at most 8 per thread
#pragma unroll
          for (int k = 0; k < 8; ++k) {
            const uint32_t i = t + BT * k;
            if (i >= n) break;
            uint4 r;
            JQ_COMPACT_EVAL(i, r)
            if (k < 4 && i < ov)
              h[k < 4 ? k : 0] = r;
            else
              S[base + i] = r;
          }
        }
        JQ_FAIL_IF(!ok)
        if (ov) {
#pragma unroll
          for (int k = 0; k < 4; ++k)
            if (t + BT * k < ov) S[base + t + BT * k] = h[k];
          __syncthreads();
        }
#undef JQ_COMPACT_EVAL
        prev_base = base;
      } else if (ci < ns) {
        // ---------------- boomerang stage ci
        uint4 v1[8];
        uint32_t A = 0, B = 0, sm = 0;
        bool shallow = false, flat = false;  // no position below 512 / 4096 live
        if (ok) {
          const uint4 *P4 = reinterpret_cast<const uint4 *>(C);
          const uint4 pa = P4[t], pb = P4[BT + t];
          const uint2 fl = reinterpret_cast<const uint2 *>(C + 4096)[t];
          A = fl.x;
          B = fl.y;
          shallow = (pa.x >> 13) & 1u;
          flat = (pa.x >> 29) & 1u;
          sm = t < 8 && !shallow ? 0xffffu : (B >> 16);
#define JQ_G(w, h) \
  ((((w) >> (16 * (h) + 15)) & 1u) ? S[((w) >> (16 * (h))) & 0x1fffu] : make_uint4(0, 0, 0, 0))
#define JQ_L1(k, wa, wb, h) v1[k] = xand2(JQ_G(wa, h), JQ_G(wb, h), mk<k>(A), mk<16 + k>(A), mk<k>(B));
          if (flat) {
            // only the positions read from outside (warp-uniform skips where
            // no lane has one)
#define JQ_F1(k, wa, wb, h) \
  if ((sm >> (k)) & 1u) JQ_L1(k, wa, wb, h)
            JQ_F1(0, pa.x, pb.x, 0) JQ_F1(1, pa.x, pb.x, 1) JQ_F1(2, pa.y, pb.y, 0)
            JQ_F1(3, pa.y, pb.y, 1) JQ_F1(4, pa.z, pb.z, 0) JQ_F1(5, pa.z, pb.z, 1)
            JQ_F1(6, pa.w, pb.w, 0) JQ_F1(7, pa.w, pb.w, 1)
#undef JQ_F1
          } else {
            JQ_L1(0, pa.x, pb.x, 0) JQ_L1(1, pa.x, pb.x, 1) JQ_L1(2, pa.y, pb.y, 0)
            JQ_L1(3, pa.y, pb.y, 1) JQ_L1(4, pa.z, pb.z, 0) JQ_L1(5, pa.z, pb.z, 1)
            JQ_L1(6, pa.w, pb.w, 0) JQ_L1(7, pa.w, pb.w, 1)
          }
#undef JQ_L1
#undef JQ_G
        }
        // single buffer: every gather done before the first overwrite
        JQ_FAIL_IF(!ok)
        if (flat) {
#define JQ_ST1(k) \
  if ((sm >> (k)) & 1u) S[4096 + 512 * k + us] = v1[k];
          JQ_ST1(0) JQ_ST1(1) JQ_ST1(2) JQ_ST1(3) JQ_ST1(4) JQ_ST1(5) JQ_ST1(6) JQ_ST1(7)
#undef JQ_ST1
          if (t == 0) S[0] = make_uint4(0, 0, 0, 0);
        } else {
#define JQ_ST1(k) \
  if (((sm >> (k)) & 1u)) S[4096 + 512 * k + us] = v1[k];
          JQ_ST1(0) JQ_ST1(1) JQ_ST1(2) JQ_ST1(3) JQ_ST1(4) JQ_ST1(5) JQ_ST1(6) JQ_ST1(7)
#undef JQ_ST1
          uint4 v2[4];
#define JQ_L2(k)                                                                   \
  v2[k] = xand2(v1[k], v1[k + 4], mk<8 + k>(A), mk<24 + k>(A), mk<8 + k>(B));      \
  if (((sm >> (8 + k)) & 1u)) S[2048 + 512 * k + us] = v2[k];
          JQ_L2(0) JQ_L2(1) JQ_L2(2) JQ_L2(3)
#undef JQ_L2
          const uint4 v30 = xand2(v2[0], v2[2], mk<12>(A), mk<28>(A), mk<12>(B));
          if (((sm >> 12) & 1u)) S[1024 + us] = v30;
          const uint4 v31 = xand2(v2[1], v2[3], mk<13>(A), mk<29>(A), mk<13>(B));
          if (((sm >> 13) & 1u)) S[1536 + us] = v31;
          const uint4 v4 = xand2(v30, v31, mk<14>(A), mk<30>(A), mk<14>(B));
          if (((sm >> 14) & 1u)) S[512 + us] = v4;
          if (shallow) {
            if (t == 0) S[0] = make_uint4(0, 0, 0, 0);
          } else {
            const uint32_t XA = mk<15>(A), XB = mk<31>(A), OB = mk<15>(B);
            uint4 c = xand2(shfl4_xor(v4, 16), v4, XA, XB, OB);
            if (lane_i >= 16) S[us] = c;
#pragma unroll
            for (int k = 3; k >= 0; --k) {
              const uint32_t d = 1u << k;
              const uint4 a = shfl4(c, (lane_i + d) & 31);
              const uint4 bb = shfl4(c, (lane_i + 2 * d) & 31);
              if (lane_i >= d && lane_i < 2 * d) {
                c = xand2(a, bb, XA, XB, OB);
                S[us] = c;
              }
            }
          }
        }
        __syncthreads();
        if (!shallow) {
          // levels 10..13 (positions 15..1) in warp 0 from positions 16..31
          if (t < 32) {
            uint4 h = t < 16 ? S[sw(16 + t)] : make_uint4(0, 0, 0, 0);
#pragma unroll 1
            for (int m = 0; m < 4; ++m) {
              const uint32_t len = 8u >> m;
              const uint4 bb = shfl4(h, (t + len) & 31);
              if ((uint32_t)t < len) {
                h = xand2(h, bb, 0u - ((B >> (16 + m)) & 1u), 0u - ((B >> (20 + m)) & 1u),
                          0u - ((B >> (24 + m)) & 1u));
                S[len + t] = h;
              }
            }
            if (t == 0) S[0] = make_uint4(0, 0, 0, 0);
          }
          __syncthreads();
        }
        for (uint32_t hm = __ballot_sync(0xffffffffu, (my_hook >> 8) == ci); hm; hm &= hm - 1) {
          const uint32_t j = __ffs(hm) - 1;
          const uint32_t g = __shfl_sync(0xffffffffu, my_hook, j) & 255u;
          WO[(warp_i + 16 * j) * 32 + lane_i] = S[sw(g * 32 + lane_i)];
        }
      } else if (has_sram && ci == ns) {
        // ---------------- SRAM & duplicate permutation + SRAM ports
        JQ_FAIL_IF(!ok)
        uint4 *St = S;
        const uint32_t nq = (num_srams * 4 + num_dup) * 32;
        const uint4 *F4 = perm_flags(sh, C, nq);
        for (uint32_t q = t; q < nq; q += BT) {
          const uint4 w = WO[perm_lin(C, q)];
          const uint4 fl = F4[q >> 5];
          const uint32_t inv = bitmask(fl.x, q), set0 = bitmask(fl.y, q);
          St[q] = make_uint4((w.x & ~set0) ^ inv, is_x ? (w.y & ~set0) : 0u, (w.z & ~set0) ^ inv,
                             is_x ? (w.w & ~set0) : 0u);
        }
        __syncthreads();
        // one warp per (SRAM, lane word of the pair), lane = stream
        const int warp = t >> 5, ln = t & 31;
        for (uint32_t ih = warp; ih < num_srams * 2; ih += BT / 32) {
          const uint32_t i = ih >> 1, hsel = ih & 1;
          const uint32_t *Aw = reinterpret_cast<const uint32_t *>(St + (4 * i) * 32) + 2 * hsel;
          // signal words k of the SRAM's staged rows (read address 0..15,
          // write address 16..31, write enable 32..63, data 64..95) to the
          // stream's bits: lane = stream after a warp transpose
          const uint32_t addr = warp_transpose32(Aw[4 * ln]);
          const uint32_t ra = addr & 0xffffu, wa = addr >> 16;
          const uint32_t en = warp_transpose32(Aw[4 * (32 + ln)]);
          const uint2 dk = *reinterpret_cast<const uint2 *>(Aw + 4 * (64 + ln));
          const uint32_t data = warp_transpose32(dk.x), datax = warp_transpose32(dk.y);
          const size_t stream = (size_t)(2 * lp + hsel) * 32 + ln;
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
          // the streams' read words back to 32 signal words (lane = bit)
          const uint32_t slotw = (num_ios - num_srams + i) * 32;
          uint32_t *WOw = reinterpret_cast<uint32_t *>(WO);
          const uint32_t word = warp_transpose32(r), wordx = warp_transpose32(rx);
          *reinterpret_cast<uint2 *>(WOw + 4 * (slotw + ln) + 2 * hsel) =
              make_uint2(word, is_x ? wordx : 0u);
        }
        for (uint32_t q = t; q < num_dup * 32; q += BT)
          WO[(num_ios - num_srams - num_dup) * 32 + q] = St[num_srams * 4 * 32 + q];
        __syncthreads();
      } else {
        // ---------------- clock-enable permutation and commit, both lane words
        JQ_FAIL_IF(!ok)
        if (t == 0 && is_last && sh.dyn) {
          next_ticket = atomicAdd(&g_bticket[P.slot], 1ull);
          have_next = true;
        }
        const uint32_t nq = num_ios * 32;
        const uint4 *F4 = perm_flags(sh, C, nq);
        // The new words come from shared memory; the old words (kept by
        // streams whose clock enable is clear) are loaded only by warps where
        // some stream of their state word keeps its value -- none, when
        // every enable is set.
        for (uint32_t q = t; q < nq; q += BT) {  // warp-uniform bound
          const uint4 src = WO[perm_lin(C, q)];
          const uint4 fl = F4[q >> 5];
          const uint32_t inv = bitmask(fl.x, q), set0 = bitmask(fl.y, q), dinv = bitmask(fl.z, q);
          const uint4 me = WO[q];
          const uint32_t cp0 = (src.x & ~set0) ^ inv, cp1 = (src.z & ~set0) ^ inv;
          if (P.constraints)  // a warp holds the 32 signals of one word
            check_word(P, io_off + (q >> 5), __reduce_or_sync(0xffffffffu, cp0), 2 * lp,
                       __reduce_or_sync(0xffffffffu, cp1), 2 * lp + 1, P.first_cycle + cyc,
                       cyc == 0);
          const size_t sg = (size_t)io_off * 32 + q;
          uint32_t o0 = 0, o1 = 0, ox0 = 0, ox1 = 0;  // old v0, v1, x0, x1
          if (__any_sync(0xffffffffu, (cp0 & cp1) != 0xffffffffu)) {
            if (is_x) {  // quad layout
              const uint4 w = __ldcg(reinterpret_cast<const uint4 *>(in + pair_base + (sg << 2)));
              o0 = w.x;
              ox0 = w.y;
              o1 = w.z;
              ox1 = w.w;
            } else {
              const size_t w = pair_base + (sg << (P.xhalf ? 2 : 1));
              o0 = ldcg(in + w);
              o1 = ldcg(in + w + (P.xhalf ? 2 : 1));
            }
          }
          const uint32_t n0 = (o0 & ~cp0) | ((me.x ^ dinv) & cp0);
          const uint32_t n1 = (o1 & ~cp1) | ((me.z ^ dinv) & cp1);
          if (is_x) {
            const uint32_t cx0 = src.y & ~set0, cx1 = src.w & ~set0;
            *reinterpret_cast<uint4 *>(out + pair_base + (sg << 2)) =
                make_uint4(n0, (ox0 & ~cp0 & ~cx0) | (me.y & cp0 & ~cx0) | cx0, n1,
                           (ox1 & ~cp1 & ~cx1) | (me.w & cp1 & ~cx1) | cx1);
          } else if (P.xhalf) {  // values only; the X words keep theirs
            out[pair_base + (sg << 2)] = n0;
            out[pair_base + (sg << 2) + 2] = n1;
          } else {
            *reinterpret_cast<uint2 *>(out + pair_base + (sg << 1)) = make_uint2(n0, n1);
          }
        }
      }
    }
    off += 256 + 512 * (size_t)R + STAGE_WORDS * ((size_t)ns + 2);
    if (P.part_cycles) {
      __syncthreads();
      if (t == 0) atomicAdd(&P.part_cycles[pid], (unsigned long long)(clock64() - t_start));
    }
    ++pid;
    if (is_last) break;
  }
}
#undef JQ_FAIL_IF
#undef JQ_HOOKS_COMPACT

// Script chunk of an octet item's ci-th copy: the boomerang stages, the
// SRAM/duplicate chunk when the partition has one, the clock-enable chunk.
__device__ __forceinline__ uint32_t oct_chunk(uint32_t ci, uint32_t ns, bool has_sram) {
  return (!has_sram && ci == ns) ? ns + 1 : ci;
}

// Global-read slots an octet item loads (16 rounds of 128 slots).
constexpr uint32_t OCT_MAX_GR = 2048;
// Shared memory of an octet item besides the chunks and tree slots: the
// writeout map (writeout slot -> its first tree slot), for setup/hold checks
// the OR of each writeout word's clock enables per lane word, and the
// partition's global-read source row.
constexpr uint32_t OCT_AUX_WORDS = 256 + 256 * 8 + OCT_MAX_GR;

// An octet work item: the block's partition list for 8 lane words (256
// streams) at once, in the octet state layout, so every state access moves a
// signal's 64 bytes (the 16-byte parts of its four lane pairs) with adjacent
// threads: thread t handles lane pair k = t & 3 of slot / entry / signal
// t >> 2 (+ 128 per round).  Every partition must be in the compact form
// without carries and fit the tree slots (metadata word 127, written by
// jq_batched_prepare: the slots it needs, or ~0).  A tree slot is 64 bytes:
// S[4 * slot + k] holds (v, x) of lane words 2k and 2k+1.  Stage regions are
// never overwritten within a partition, so writeouts are not copied: the
// writeout map names the tree slots a writeout slot's 32 signals occupy (a
// hooked 32-slot block of a stage region, or the SRAM stage's staging and
// read-out slots).
__device__ void run_item8(const BatchParams &P, Shared &sh, uint4 *S, uint32_t *aux,
                          uint32_t *chunks, uint32_t &uses0, uint32_t &uses1,
                          const uint32_t *script, const uint32_t *in, uint32_t *out, uint32_t og,
                          uint32_t pid0, bool &failed, unsigned long long &next_ticket,
                          bool &have_next, bool &pending, unsigned long long &bar_target,
                          uint32_t cyc) {
  const int t = threadIdx.x;
  const uint32_t k = t & 3u, el = (uint32_t)t >> 2;
  uint32_t *const wo_map = aux;
  uint32_t *const clk_or = aux + 256;
  uint32_t *const gr_src = aux + 256 + 256 * 8;
  // the octet's words: signal s (value plane) at 16 * (og * V + s)
  const size_t grp_base = ((size_t)og * P.vsig) << 4;
  size_t off = 0;
  uint32_t pid = pid0;
  for (;;) {
    __syncthreads();
    long long t_start = clock64();
    if (t < 256) sh.meta[t] = __ldg(script + off + t);
    // the global-read sources of slots 0..OCT_MAX_GR-1 into shared memory
    // (16 bytes per thread; the previous item's readers are done)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(gr_src + 4 * t)),
                 "l"(P.gr_sources + (size_t)pid * 8192 + 4 * t)
                 : "memory");
    asm volatile("cp.async.commit_group;" ::: "memory");
    __syncthreads();
    const uint32_t ns = sh.meta[0];
    if (!ns) {  // the list ended: nothing is left in flight
      asm volatile("cp.async.wait_all;" ::: "memory");
      break;
    }
    const uint32_t is_last = sh.meta[1], num_ios = sh.meta[2], io_off = sh.meta[3];
    const uint32_t num_srams = sh.meta[4], sram_off = sh.meta[5], R = sh.meta[6];
    const uint32_t num_dup = sh.meta[7];
    const bool is_x = sh.meta[8] != 0;
    const uint32_t need = sh.meta[127];
    const uint32_t *ch0 = script + off + 256 + 512 * (size_t)R;
    const bool has_sram = (num_srams | num_dup) != 0;
    const uint32_t nchunks = ns + (has_sram ? 2 : 1);
    // a partition the octet form cannot run (the host checks the whole
    // script before choosing this form, so only a malformed launch has one)
    const bool runnable = need <= P.slot_cap && (sh.meta[10] & 1u);
    // Every chunk of the partition at once, packed in order into the chunk
    // buffers (the prepare step admits a partition to the octet form only
    // when they fit): script data, never written, so the copies run during
    // the grid-barrier wait below.
    if (t == 0 && runnable) {
      uint32_t total = 0;
      for (uint32_t ci = 0; ci < nchunks; ++ci) total += chunk_bytes(sh, oct_chunk(ci, ns, has_sram));
      mbar_expect_tx(&sh.bar[0], total);
      uint32_t o = 0;
      for (uint32_t ci = 0; ci < nchunks; ++ci) {
        const uint32_t kc = oct_chunk(ci, ns, has_sram), nb = chunk_bytes(sh, kc);
        tma_load_1d(reinterpret_cast<uint8_t *>(chunks) + o, ch0 + (size_t)STAGE_WORDS * kc, nb,
                    &sh.bar[0]);
        o += nb;
      }
    }
    // the deferred wait of the grid barrier ending the previous major stage
    // (see run_item2); the waiting warps prefetch the commit rows
    if (pending) {
      pending = false;
      const uint32_t *rows = in + grp_base + (((size_t)io_off * 32) << 4);
      const uint32_t nl = num_ios * 16;  // 128-byte lines
      if (!grid_wait(P, sh, bar_target, [&](uint32_t i0, uint32_t n) {
            for (uint32_t l = i0; l < nl; l += n) prefetch_l2(rows + 32 * (size_t)l);
          })) {
        failed = true;
        asm volatile("cp.async.wait_all;" ::: "memory");
        if (t == 0 && runnable) mbar_wait(&sh.bar[0], uses0 & 1u, P.chunk_timeout);
        return;
      }
      t_start = clock64();
    }
    if (!runnable) {
      asm volatile("cp.async.wait_all;" ::: "memory");
      if (t == 0) atomicCAS(&g_status[P.slot], 0, JQ_ERR_INVALID_ARG);
      failed = true;
      return;
    }
    if (P.constraints)
      for (uint32_t i = t; i < num_ios * 8; i += BT) clk_or[i] = 0;
    asm volatile("cp.async.wait_all;" ::: "memory");
    __syncthreads();  // the source row landed
    // ---- global read: slot el + 128 m, its 16-byte part k, into tree slot
    // sw(slot) (the prepared stage-0 entries name the swizzled slot, which
    // stays within the slot's 32-aligned block)
    if (is_x) {
#pragma unroll
      for (int m = 0; m < 16; ++m) {
        const uint32_t ek = gr_src[el + 128 * m];
        uint4 *dst = &S[4 * sw(el + 128 * m) + k];
        if (ek < GR_SKIP) {
          const uint32_t *bp = (ek >> 31) ? out : in;
          const uint32_t *src = bp + grp_base + ((size_t)(ek & 0x7fffffffu) << 4) + 4 * k;
          asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src)
                       : "memory");
        } else if (ek == GR_EMPTY) {
          *dst = make_uint4(0, 0, 0, 0);
        }
      }
      asm volatile("cp.async.wait_all;" ::: "memory");
    } else {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        uint4 v[8];
#pragma unroll
        for (int m = 0; m < 8; ++m) {
          const uint32_t ek = gr_src[el + 128 * (8 * h + m)];
          v[m] = make_uint4(0, 0, 0, 0);
          if (ek < GR_SKIP) {
            const uint32_t *bp = (ek >> 31) ? out : in;
            v[m] = __ldcg(reinterpret_cast<const uint4 *>(
                bp + grp_base + ((size_t)(ek & 0x7fffffffu) << 4) + 4 * k));
            v[m].y = v[m].w = 0u;  // the X planes of a partition without X
          }
        }
#pragma unroll
        for (int m = 0; m < 8; ++m)
          if (gr_src[el + 128 * (8 * h + m)] != GR_SKIP) S[4 * sw(el + 128 * (8 * h + m)) + k] = v[m];
      }
    }
    // writeout slot t's hook (stage << 8 | 32-slot block of the stage's
    // region); the map entry is set when that stage runs
    uint32_t my_hook = 0xffffffffu;
    if ((uint32_t)t < num_ios) {
      const uint32_t hw = sh.meta[128 + t / 2];
      my_hook = (t & 1) ? (hw >> 16) : (hw & 0xffffu);
    }
    // the chunks landed (copies that do not complete within the bounded
    // wait fail the item and the launch) and the global read is complete
    {
      const bool ok = __all_sync(0xffffffffu, mbar_wait(&sh.bar[0], uses0 & 1u, P.chunk_timeout));
      ++uses0;
      if (__syncthreads_or(!ok)) {
        failed = true;
        return;
      }
    }
    uint32_t reg_end = 0;  // end of the last stage region
    const uint32_t *C = chunks;
    for (uint32_t ci = 0; ci < nchunks; ++ci) {
      if (ci) C += chunk_bytes(sh, oct_chunk(ci - 1, ns, has_sram)) / 4;
      if (ci < ns) {
        // ---------------- compact stage ci: entries el + 128 m; its region
        // follows the previous one, so nothing it reads is overwritten
        const uint32_t n = C[0], base = C[1];
        if ((my_hook >> 8) == ci) wo_map[t] = base + 32 * (my_hook & 255u);
        for (uint32_t i = el; i < n; i += 128) {
          const uint32_t en = C[4 + i];
          const uint4 ga = ((en >> 29) & 1u) ? make_uint4(0, 0, 0, 0) : S[4 * (en & 8191u) + k];
          const uint4 gb =
              ((en >> 30) & 1u) ? make_uint4(0, 0, 0, 0) : S[4 * ((en >> 13) & 8191u) + k];
          S[4 * (base + i) + k] = xand2(ga, gb, 0u - ((en >> 26) & 1u), 0u - ((en >> 27) & 1u),
                                        0u - ((en >> 28) & 1u));
        }
        reg_end = base + n;
        __syncthreads();
      } else if (has_sram && ci == ns) {
        // ---------------- SRAM & duplicate permutation + SRAM ports: staged
        // words past the last region, then 32 read-out slots per SRAM
        const uint32_t st0 = (reg_end + 31) & ~31u;
        const uint32_t nq = (num_srams * 4 + num_dup) * 32;
        const uint32_t ro = st0 + nq;
        const uint4 *F4 = perm_flags(sh, C, nq);
        for (uint32_t q = el; q < nq; q += 128) {
          const uint32_t p = perm_lin(C, q);
          const uint4 w = S[4 * (wo_map[p >> 5] + (p & 31u)) + k];
          const uint4 fl = F4[q >> 5];
          const uint32_t inv = bitmask(fl.x, q), set0 = bitmask(fl.y, q);
          S[4 * (st0 + q) + k] = make_uint4((w.x & ~set0) ^ inv, is_x ? (w.y & ~set0) : 0u,
                                            (w.z & ~set0) ^ inv, is_x ? (w.w & ~set0) : 0u);
        }
        __syncthreads();
        // one warp per (SRAM, lane word), lane = stream; a slot's word of
        // lane word lw (value, X) is word 2 lw (+1) of its 16
        uint32_t *Sw = reinterpret_cast<uint32_t *>(S);
        const int warp = t >> 5, ln = t & 31;
        for (uint32_t ih = warp; ih < num_srams * 8; ih += BT / 32) {
          const uint32_t i = ih >> 3, lw = ih & 7u;
          const uint32_t *Aw = Sw + 16 * (size_t)(st0 + 128 * i) + 2 * lw;
          const uint32_t addr = warp_transpose32(Aw[16 * ln]);
          const uint32_t ra = addr & 0xffffu, wa = addr >> 16;
          const uint32_t en = warp_transpose32(Aw[16 * (32 + ln)]);
          const uint32_t data = warp_transpose32(Aw[16 * (64 + ln)]);
          const uint32_t datax = warp_transpose32(Aw[16 * (64 + ln) + 1]);
          const size_t stream = (size_t)(8 * og + lw) * 32 + ln;
          uint32_t *ram = P.sram + stream * P.sram_words + sram_off + (size_t)i * SRAM_WORDS;
          const uint32_t r = ldcg(ram + ra), w0 = ldcg(ram + wa);
          uint32_t rx = 0, w0x = 0;
          const bool hx = is_x && P.sram_x != nullptr;
          uint32_t *ramx = hx ? P.sram_x + stream * P.sram_words + sram_off + (size_t)i * SRAM_WORDS
                              : nullptr;
          if (hx) {
            rx = ldcg(ramx + ra);
            w0x = ldcg(ramx + wa);
          }
          ram[wa] = (w0 & ~en) | (data & en);
          if (hx) ramx[wa] = (w0x & ~en) | (datax & en);
          const uint32_t word = warp_transpose32(r), wordx = warp_transpose32(rx);
          *reinterpret_cast<uint2 *>(Sw + 16 * (size_t)(ro + 32 * i + ln) + 2 * lw) =
              make_uint2(word, is_x ? wordx : 0u);
        }
        // duplicates are the staged words themselves; SRAM read-outs follow
        if ((uint32_t)t < num_dup) wo_map[num_ios - num_srams - num_dup + t] = st0 + 32 * (num_srams * 4 + t);
        if ((uint32_t)t < num_srams) wo_map[num_ios - num_srams + t] = ro + 32 * t;
        __syncthreads();
      } else {
        // ---------------- clock-enable permutation and commit: signal el +
        // 128 m, lane pair k; a warp's 8 signals lie in one state word (two
        // signals per thread per round measured 1% slower)
        if (t == 0 && is_last && sh.dyn) {
          next_ticket = atomicAdd(&g_bticket[P.slot], 1ull);
          have_next = true;
        }
        const uint32_t nq = num_ios * 32;
        const uint4 *F4 = perm_flags(sh, C, nq);
        for (uint32_t q = el; q < nq; q += 128) {  // warp-uniform bound
          const uint32_t p = perm_lin(C, q);
          const uint4 src = S[4 * (wo_map[p >> 5] + (p & 31u)) + k];
          const uint4 me = S[4 * (wo_map[q >> 5] + (q & 31u)) + k];
          const uint4 fl = F4[q >> 5];
          const uint32_t inv = bitmask(fl.x, q), set0 = bitmask(fl.y, q), dinv = bitmask(fl.z, q);
          const uint32_t cp0 = (src.x & ~set0) ^ inv, cp1 = (src.z & ~set0) ^ inv;
          if (P.constraints) {
            atomicOr(&clk_or[(q >> 5) * 8 + 2 * k], cp0);
            atomicOr(&clk_or[(q >> 5) * 8 + 2 * k + 1], cp1);
          }
          const size_t w = grp_base + ((((size_t)io_off * 32 + q)) << 4) + 4 * k;
          uint32_t o0 = 0, o1 = 0, ox0 = 0, ox1 = 0;  // old v0, v1, x0, x1
          if (__any_sync(0xffffffffu, (cp0 & cp1) != 0xffffffffu)) {
            const uint4 o = __ldcg(reinterpret_cast<const uint4 *>(in + w));
            o0 = o.x;
            ox0 = o.y;
            o1 = o.z;
            ox1 = o.w;
          }
          const uint32_t n0 = (o0 & ~cp0) | ((me.x ^ dinv) & cp0);
          const uint32_t n1 = (o1 & ~cp1) | ((me.z ^ dinv) & cp1);
          if (is_x) {
            const uint32_t cx0 = src.y & ~set0, cx1 = src.w & ~set0;
            *reinterpret_cast<uint4 *>(out + w) =
                make_uint4(n0, (ox0 & ~cp0 & ~cx0) | (me.y & cp0 & ~cx0) | cx0, n1,
                           (ox1 & ~cp1 & ~cx1) | (me.w & cp1 & ~cx1) | cx1);
          } else {  // values only; the X words keep theirs
            out[w] = n0;
            out[w + 2] = n1;
          }
        }
        if (P.constraints) {
          // setup/hold checks per state word, a warp per word (check_word
          // per two lane words)
          __syncthreads();
          for (uint32_t j = (uint32_t)t >> 5; j < num_ios; j += BT / 32) {
#pragma unroll 1
            for (uint32_t kk = 0; kk < 4; ++kk)
              check_word(P, io_off + j, clk_or[8 * j + 2 * kk], 8 * og + 2 * kk,
                         clk_or[8 * j + 2 * kk + 1], 8 * og + 2 * kk + 1, P.first_cycle + cyc,
                         cyc == 0);
          }
        }
      }
    }
    off += 256 + 512 * (size_t)R + STAGE_WORDS * ((size_t)ns + 2);
    if (P.part_cycles) {
      __syncthreads();
      if (t == 0) atomicAdd(&P.part_cycles[pid], (unsigned long long)(clock64() - t_start));
    }
    ++pid;
    if (is_last) break;
  }
}


// L2 prefetch of what the CTA's item of major stage ms reads first, when
// that stage assigns items statically (at most one per CTA): the global-read
// source table of its first partition, the head of its script (metadata,
// global-read section, the first two chunks) and the previous-cycle state
// rows `prev` its commit reads (a partition commits to the words it wrote a
// cycle earlier, long evicted by then).  Threads i0 = 0..n-1 share it;
// prefetches are hints and change no data.
// L2 prefetch of what the CTA's item of major stage ms reads first, when
// that stage assigns items statically: the global-read source table of its
// first partition, the head of its script (metadata, global-read section,
// the first two chunks) and the previous-cycle state rows `prev` its commit
// reads (a partition commits to the words it wrote a cycle earlier, long
// evicted by then).  Addresses come from the per-launch item table, so no
// load waits.  Threads i0 = 0..n-1 share it; prefetches are hints and change
// no data.
template <int NL>
__device__ void prefetch_item_l2(const BatchParams &P, const Shared &sh, unsigned ms,
                                 const uint32_t *prev, uint32_t i0, uint32_t n) {
  const size_t so = sh.st_off[ms];
  if (so == ~(size_t)0) return;
  const uint32_t *script = P.blocks_data + so;
  const uint32_t *gr = P.gr_sources + (size_t)sh.st_pid[ms] * 8192;
  const size_t left = sh.script_words - so;  // the window ends with the script data
  constexpr uint32_t GR_LINES = 8192 / 32;                  // 128-byte lines
  constexpr size_t WINDOW = 256 + 512 * 8 + 2 * STAGE_WORDS;
  const uint32_t script_lines = (uint32_t)((left < WINDOW ? left : WINDOW) / 32);
  // commit rows of the first partition: signals [io_off*32, +num_ios*32)
  // of the item's lane pair, contiguous in the interleaved layout
  const uint32_t per = P.lanes / NL;
  const uint32_t lane0 = NL * (blockIdx.x % per);
  const size_t w0 = phys(P, lane0 & ~1u, (size_t)sh.st_io[ms] * 32);
  // 128-byte lines: 32 signals of 2^shift words each per writeout slot
  const uint32_t rows = sh.st_nio[ms] << sig_shift_of(P);
  for (uint32_t l = i0; l < GR_LINES + script_lines + rows; l += n) {
    if (l < GR_LINES)
      prefetch_l2(gr + 32 * l);
    else if (l < GR_LINES + script_lines)
      prefetch_l2(script + 32 * (l - GR_LINES));
    else
      prefetch_l2(prev + w0 + 32 * (size_t)(l - GR_LINES - script_lines));
  }
}

// L2 prefetch of the state words the global read of the CTA's item of major
// stage ms takes from the previous-cycle snapshot `prev` (sources without the
// staged bit), from its first partition's compacted source row.  The loads
// of the row wait, so only CTAs with time to spare call it.
template <int NL>
__device__ void prefetch_global_read_l2(const BatchParams &P, const Shared &sh, unsigned ms,
                                        const uint32_t *prev, uint32_t i0, uint32_t n) {
  if (sh.st_off[ms] == ~(size_t)0) return;
  const uint32_t *row = P.gr_sources + (size_t)sh.st_pid[ms] * 8192;
  const uint32_t per = P.lanes / NL;
  const uint32_t lane0 = NL * (blockIdx.x % per);
  const size_t pb = phys(P, lane0 & ~1u, 0);  // the lane group's word of signal 0
  const uint32_t sh2 = sig_shift_of(P);
  constexpr int K = 18;  // 18 * 480 >= 8192 slots: one round of row loads
  for (uint32_t q0 = i0; q0 < 8192; q0 += K * n) {
    uint32_t ev[K];
#pragma unroll
    for (int k = 0; k < K; ++k) ev[k] = q0 + k * n < 8192 ? __ldg(row + q0 + k * n) : GR_SKIP;
#pragma unroll
    for (int k = 0; k < K; ++k)
      if (ev[k] < 0x80000000u) prefetch_l2(prev + pb + ((size_t)ev[k] << sh2));
  }
}

// NL lane words per work item (1, 2 for run_item2, 8 for run_item8); DS
// only with NL = 1.
template <bool DS, int NL>
__global__ void __launch_bounds__(BT, 1) jq_batched_kernel(BatchParams P) {
  static_assert(NL == 1 || ((NL == 2 || NL == 8) && !DS), "only single lanes double-buffer");
  extern __shared__ __align__(128) uint8_t dyn[];
  __shared__ Shared sh;
  constexpr size_t WB = NL == 2 ? 16 : 8;  // bytes per tree / writeout word (NL 1, 2)
  uint32_t *chunks = reinterpret_cast<uint32_t *>(dyn);               // 2 x 20 KB
  // NL 1, 2: tree state ((1 or 2) x 8192 words), then the writeouts
  // (wo_slots * 32 words); NL 8: the writeout map and clock-enable ORs, then
  // slot_cap tree slots of 64 bytes
  uint8_t *S = dyn + 2 * CHUNK_BYTES + (NL == 8 ? OCT_AUX_WORDS * 4 : 0);
  uint8_t *WO = NL == 8 ? dyn + 2 * CHUNK_BYTES : S + (DS ? 2 : 1) * 8192 * WB;
  const int t = threadIdx.x;
  if (t == 0) {
    mbar_init(&sh.bar[0], 1);
    mbar_init(&sh.bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  const uint32_t wo_words = NL == 8 ? OCT_AUX_WORDS : P.wo_slots * 32 * (uint32_t)(WB / 4);
  for (uint32_t q = t; q < wo_words; q += BT) reinterpret_cast<uint32_t *>(WO)[q] = 0;
  // item table: thread ms resolves major stage ms
  if (t == 0) sh.script_words = P.blocks_start[(size_t)P.num_major_stages * P.num_blocks];
  if ((unsigned)t < P.num_major_stages) {
    const uint32_t nblk = P.block_list ? P.block_list_start[t + 1] - P.block_list_start[t]
                                       : P.num_blocks;
    const uint32_t per = P.lanes / NL;
    const uint32_t items = nblk * per;
    size_t so = ~(size_t)0;
    uint32_t pid = 0, nio = 0, io = 0;
    if (items <= gridDim.x && blockIdx.x < items) {
      const uint32_t bi = blockIdx.x / per;
      const uint32_t blk = P.block_list ? P.block_list[P.block_list_start[t] + bi] : bi;
      const size_t e = (size_t)t * P.num_blocks + blk;
      so = P.blocks_start[e];
      pid = P.part_base[e];
      const uint32_t *sc = P.blocks_data + so;
      if (sc[0]) {
        nio = sc[2];
        io = sc[3];
      }
    }
    sh.st_items[t] = items;
    sh.st_off[t] = so;
    sh.st_pid[t] = pid;
    sh.st_nio[t] = nio;
    sh.st_io[t] = io;
  }
  __syncthreads();
  // Lane groups: with lane pairs or octets and one item per CTA in every
  // major stage, CTA i always runs lane group i % per, and the CTAs of one
  // group (which alone read and write that group's state words, SRAM rows,
  // stimulus and outputs) form their own barrier group.
  const uint32_t per_lp = P.lanes / NL;
  bool grouped = NL >= 2 && per_lp > 1 && per_lp <= MAX_GROUPS && gridDim.x >= per_lp;
  for (unsigned ms = 0; ms < P.num_major_stages; ++ms) grouped &= sh.st_items[ms] <= gridDim.x;
  const uint32_t grp = grouped ? blockIdx.x % per_lp : 0;         // lane pair of this CTA
  const uint32_t grp_rank = grouped ? blockIdx.x / per_lp : blockIdx.x;
  const uint32_t grp_ctas = grouped ? (gridDim.x - grp + per_lp - 1) / per_lp : gridDim.x;
  if (t == 0) {
    sh.bar_count = grouped ? &g_bgroup[(size_t)P.slot * MAX_GROUPS + grp] : &g_bcount[P.slot];
    sh.bar_size = grp_ctas;
  }
  // lanes this CTA copies stimulus for and records: its lane group, or all
  const uint32_t lane_lo = grouped ? NL * grp : 0, lane_n = grouped ? NL : P.lanes;
  __syncthreads();
  uint32_t uses0 = 0, uses1 = 0;
  bool failed = false;
  // thread 0: arrival count that completes the next grid barrier, and the
  // first ticket of the current major stage
  unsigned long long bar_target = 0, ticket_base = 0;
  const size_t snap = P.sig_per_snap * P.lanes;  // lane-major record snapshot
  // Lane-pair items take over the barrier that ends the previous major
  // stage (see run_item2); `pending` marks one owed.
  constexpr bool DEFER = NL >= 2;
  bool pending = false;
  auto no_prefetch = [](uint32_t, uint32_t) {};

  for (size_t c = 0; c < P.num_cycles; ++c) {
    const uint32_t *in = (c & 1) ? P.state_b : P.state_a;
    uint32_t *out = (c & 1) ? P.state_a : P.state_b;
    // inputs of snapshot c+1 into the output buffer's input region
    if (P.stim) {
      // stimulus row layout [lane][input_sigs]; each input region copies
      // stimulus signals [src, src+count) to state signals [dst, dst+count)
      // (one region at 0 when no list is given)
      const uint32_t *src = P.stim + (c + 1) * P.input_sigs * P.lanes;
      for (size_t q = (size_t)grp_rank * BT + t; q < P.input_sigs * lane_n;
           q += (size_t)grp_ctas * BT) {
        const size_t l = lane_lo + q / P.input_sigs, i = q % P.input_sigs;
        size_t dst = i;
        if (P.input_regions) {
          for (uint32_t r = 0; r < P.n_input_regions; ++r) {
            const uint32_t d0 = P.input_regions[3 * r], s0 = P.input_regions[3 * r + 1],
                           n = P.input_regions[3 * r + 2];
            if (i >= s0 && i < s0 + n) dst = d0 + (i - s0);
          }
        }
        out[phys(P, (uint32_t)l, dst)] = src[l * P.input_sigs + i];
      }
    }
    for (unsigned ms = 0; ms < P.num_major_stages; ++ms) {
      const uint32_t per = P.lanes / NL;  // items per block
      const uint32_t items = sh.st_items[ms];
      // at most one item per CTA: item = CTA index (so the CTA knows its
      // next item early and can prefetch it); otherwise tickets
      const bool dyn = items > gridDim.x;
      if (pending && !(DEFER && !dyn && blockIdx.x < items)) {  // no item here to take it
        pending = false;
        if (!grid_wait(P, sh, bar_target, no_prefetch)) return;
      }
      unsigned long long next_ticket = 0;
      bool have_next = false;
      bool done_static = false;
      for (;;) {
        __syncthreads();
        if (t == 0) {
          sh.dyn = dyn;
          // tickets of a dynamic stage are ticket_base + item
          const unsigned long long tk =
              !dyn ? (done_static ? items : blockIdx.x)
                   : (have_next ? next_ticket : atomicAdd(&g_bticket[P.slot], 1ull)) - ticket_base;
          sh.ticket = tk < items ? (uint32_t)tk : items;
        }
        __syncthreads();
        have_next = false;
        done_static = true;
        const uint32_t tk = sh.ticket;
        if (tk >= items) break;
        const uint32_t bi = tk / per, lane = tk % per;
        const uint32_t *script;
        uint32_t pid0;
        if (!dyn) {  // the item table holds this CTA's item
          script = P.blocks_data + sh.st_off[ms];
          pid0 = sh.st_pid[ms];
        } else {
          const uint32_t blk = P.block_list ? P.block_list[P.block_list_start[ms] + bi] : bi;
          script = P.blocks_data + P.blocks_start[(size_t)ms * P.num_blocks + blk];
          pid0 = P.part_base[(size_t)ms * P.num_blocks + blk];
        }
        // the next stage's item: its source row and script head into L2 a
        // whole stage ahead (hints; the row and script are never written)
        if (!dyn && ms + 1 < P.num_major_stages && sh.st_off[ms + 1] != ~(size_t)0) {
          const uint32_t *nrow = P.gr_sources + (size_t)sh.st_pid[ms + 1] * 8192;
          const uint32_t *nscr = P.blocks_data + sh.st_off[ms + 1];
          if (t < 256) prefetch_l2(nrow + 32 * t);
          else if (t < 256 + 48) prefetch_l2(nscr + 32 * (t - 256));  // metadata, chunk 0 head
        }
        if constexpr (NL == 8)
          run_item8(P, sh, reinterpret_cast<uint4 *>(S), reinterpret_cast<uint32_t *>(WO), chunks,
                    uses0, uses1, script, in, out, lane, pid0, failed, next_ticket, have_next,
                    pending, bar_target, (uint32_t)c);
        else if constexpr (NL == 2)
          run_item2(P, sh, reinterpret_cast<uint4 *>(S), reinterpret_cast<uint4 *>(WO), chunks,
                    uses0, uses1, script, in, out, lane, pid0, failed, next_ticket, have_next,
                    pending, bar_target, (uint32_t)c);
        else
          run_item<DS>(P, sh, reinterpret_cast<uint2 *>(S), reinterpret_cast<uint2 *>(WO), chunks,
                       uses0, uses1, script, in, out, lane, pid0, failed, next_ticket, have_next,
                       (uint32_t)c);
        if (failed) {  // the first error recorded stays
          if (t == 0) atomicCAS(&g_status[P.slot], 0, JQ_ERR_BARRIER_TIMEOUT);
          return;
        }
      }
      if (pending) {  // the item had no partition to take it
        pending = false;
        if (!grid_wait(P, sh, bar_target, no_prefetch)) return;
      }
      // every CTA takes exactly one ticket past the last item of a dynamic
      // stage, so the next stage's tickets start items + grid on
      if (t == 0 && dyn) ticket_base += items + gridDim.x;
      grid_arrive(sh, bar_target);
      if (DEFER && ms + 1 < P.num_major_stages) {
        pending = true;  // the wait comes with the next item
      } else {
        // grid barrier; while thread 0 waits, warps 1.. prefetch this CTA's
        // next item into L2 (the next stage's previous-cycle snapshot: `in`,
        // or at the end of the cycle this cycle's `out`)
        const unsigned ms2 = ms + 1 < P.num_major_stages ? ms + 1 : 0;
        const bool more = ms + 1 < P.num_major_stages || c + 1 < P.num_cycles;
        const uint32_t *prev = ms + 1 < P.num_major_stages ? in : out;
        // a CTA that had no item in this stage waits long (the stage's items
        // run meanwhile): it also prefetches the state words its next item's
        // global read takes from `prev`
        const bool idle = blockIdx.x >= items;
        if (!grid_wait(P, sh, bar_target, [&](uint32_t i0, uint32_t n) {
              if (more) prefetch_item_l2<NL>(P, sh, ms2, prev, i0, n);
              if (more && idle) prefetch_global_read_l2<NL>(P, sh, ms2, prev, i0, n);
            }))
          return;
      }
    }
    // record outputs of this cycle
    for (size_t q = (size_t)grp_rank * BT + t; q < (size_t)P.n_po * lane_n;
         q += (size_t)grp_ctas * BT) {
      const uint32_t po = (uint32_t)(q / lane_n), l = lane_lo + (uint32_t)(q % lane_n);
      P.wave[(c * P.n_po + po) * P.lanes + l] = ldcg(out + phys(P, l, P.po_sig[po]));
    }
    if (P.record) {  // lane-major [lane][signal]
      uint32_t *dst = P.record + (c + 1) * snap + (size_t)lane_lo * P.sig_per_snap;
      for (size_t q = (size_t)grp_rank * BT + t; q < P.sig_per_snap * lane_n;
           q += (size_t)grp_ctas * BT)
        dst[q] = ldcg(out + phys(P, lane_lo + (uint32_t)(q / P.sig_per_snap), q % P.sig_per_snap));
    }
    // the recording reads `out`; the next cycle writes into `in`: the next
    // major-stage barrier already orders them, no extra barrier needed.
  }
}

// Script preparation for this kernel (run once per script, on the device):
// every boomerang chunk is rewritten thread-major -- the 16 gather sources of
// each thread (swizzled tree addresses) as two uint4 planes and its owned
// positions' flag bits as one uint2 -- and the SRAM/duplicate and
// clock-enable chunks get their shuffle entries in q order.  Metadata, global
// read sections and sizes are unchanged, so blocks_start stays valid.  One
// CTA per (major stage, block) entry walks its partition list.
//
// Liveness.  A tree position is read from outside its stage when a writeout
// hook of the stage covers it or a needed gather of the next stage names it;
// it is live when it is read from outside or its parent is live (each
// position has one parent: children [2L, 3L) are the a inputs and [3L, 4L)
// the b inputs of [L, 2L)).  A level-1 input is needed when its position is
// live, except a b input whose ob flag forces it to one.  Stages are walked
// last to first, so each stage's needed gathers give the previous stage's
// externally read positions (for stage 0: the global-read positions).  The
// source entries are 13-bit tree addresses; their top bits carry
//   bit 15  the gather is needed (otherwise the kernel reads nothing and
//           uses 0, which only feeds dead positions or an ob-forced input);
//   bit 13  of entry 0: no position below 512 is live (levels 5..13 skipped);
//           of entry 1: no position below 4096 is live (only level 1 runs,
//           and only for positions read from outside).
// Bits 16+i of the second flag word mark owned position i as read from
// outside its stage; only those are stored.  In deep stages threads t < 8
// hold the warp-0 flags there instead and store all their positions.
// The global-read positions stage 0 needs are compacted into slots 0, 1, ...
// of the partition's source row (the rest GR_SKIP: neither loaded nor
// stored), and stage 0's sources name slots.  Dead positions are neither
// stored nor read, so the state they leave in shared memory is never
// observed.

constexpr uint32_t COMPACT_MAX_STAGES = 32;

// Shared memory of the prepare kernel (dynamic).
struct PrepShared {
  uint32_t need_bits[256];  // previous tree's positions read by needed gathers
  uint32_t ext_bits[256];   // this stage's positions read from outside
  uint32_t ext_all[COMPACT_MAX_STAGES][256];  // ext_bits of every stage
  uint32_t warp_sum[BT / 32];
  uint32_t hmask[8];        // hooked 32-position groups of a stage
  uint16_t blk_of[256];     // hooked group -> 32-slot block of its region
  uint16_t slot_prev[8192];  // previous stage's position -> shared-memory word
  uint16_t slot_cur[8192];
  uint16_t pos_of[4096];    // region slot -> position
  uint8_t live[8192];
  // bank-aware slot order of a compact stage (see below)
  uint8_t bucket_of[4096];  // entry -> 9 * (a bank group) + (b bank group), 8 = no load
  uint16_t sorted[4096];    // entries by bucket
  uint16_t order[4096];     // new slot -> entry
  uint16_t bcnt[81], bptr[81];
};

// Exclusive prefix sum of v over the CTA; *total receives the sum.  Every
// thread calls it.
__device__ uint32_t block_excl_scan(uint32_t v, uint32_t *warp_sum, uint32_t *total) {
  const uint32_t t = threadIdx.x;
  uint32_t incl = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t o = __shfl_up_sync(0xffffffffu, incl, d);
    if ((t & 31) >= (uint32_t)d) incl += o;
  }
  __syncthreads();  // earlier readers of warp_sum are done
  if ((t & 31) == 31) warp_sum[t >> 5] = incl;
  __syncthreads();
  uint32_t base = incl - v, n = 0;
  for (uint32_t w = 0; w < BT / 32; ++w) {
    if (w < (t >> 5)) base += warp_sum[w];
    n += warp_sum[w];
  }
  *total = n;
  return base;
}

__global__ void __launch_bounds__(BT) jq_batched_prepare_kernel(
    const size_t *blocks_start, const uint32_t *src, uint32_t *dst, unsigned entries,
    const uint32_t *part_base, uint32_t *gr_sources, size_t num_partitions) {
  extern __shared__ __align__(16) uint8_t prep_dyn[];
  PrepShared &ps = *reinterpret_cast<PrepShared *>(prep_dyn);
  uint32_t *const need_bits = ps.need_bits;
  uint32_t *const ext_bits = ps.ext_bits;
  uint8_t *const live = ps.live;
  const unsigned e = blockIdx.x;
  if (e >= entries) return;
  const uint32_t t = threadIdx.x;
  const uint32_t u = residue(t);
  size_t off = blocks_start[e];
  size_t pid = part_base[e];
  for (;;) {
    const uint32_t ns = src[off];
    if (!ns || pid >= num_partitions) break;
    const uint32_t is_last = src[off + 1], nio = src[off + 2], R = src[off + 6];
    const uint32_t *ch = src + off + 256 + 512 * (size_t)R;
    uint32_t *dch = dst + off + 256 + 512 * (size_t)R;
    int deep0 = 0, flat0 = 0, all_flat = 1;
    // Source entries of one boomerang chunk C -> D: plane m>>2, word m&3
    // holds entries 8*(m>>2) + 2*(m&3) + {0, 1}; entry k < 8 is input a of
    // position 4096+u+512k (source q = u+512k), entry 8+k its input b
    // (q + 4096).  Marks the needed sources in need_bits; with `write` the
    // words are stored, with `slots` a source names the shared-memory word
    // of its compacted global-read slot instead of its position.
    auto write_entries = [&](const uint32_t *C, uint32_t *D, int deep, int flat, bool write,
                             bool slots) {
#pragma unroll
      for (int m = 0; m < 8; ++m) {
        uint32_t w = 0;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const uint32_t en = 8 * (m >> 2) + 2 * (m & 3) + h;
          const uint32_t q = (en < 8) ? u + 512 * en : u + 512 * (en - 8) + 4096;
          const uint32_t P = 4096 + (q & 4095u);
          const bool ob = (C[4096 + 4 * (P >> 5) + 2] >> (P & 31)) & 1u;
          const uint32_t sp = perm_src(C, q) & 8191u;
          const bool need = live[P] && !(en >= 8 && ob);
          if (need && !slots) atomicOr(&need_bits[sp >> 5], 1u << (sp & 31));
          const uint32_t a = slots ? (need ? ps.slot_prev[sp] : 0u) : sw(sp);
          const uint32_t entry = a | ((uint32_t)need << 15) |
                                 ((en == 0 && !deep) ? (1u << 13) : 0u) |
                                 ((en == 1 && flat) ? (1u << 13) : 0u);
          w |= entry << (16 * h);
        }
        if (write) D[4 * ((m >> 2) * BT + t) + (m & 3)] = w;
      }
    };
    for (uint32_t w = t; w < 256; w += BT) need_bits[w] = 0;  // nothing reads the last stage
    __syncthreads();
    // ---- pass 1, last stage to first: liveness and the tree-form chunks
    for (int ci = (int)ns - 1; ci >= 0; --ci) {
      const uint32_t *C = ch + (size_t)ci * STAGE_WORDS;
      uint32_t *D = dch + (size_t)ci * STAGE_WORDS;
      for (uint32_t w = t; w < 256; w += BT) ext_bits[w] = need_bits[w];
      __syncthreads();
      for (uint32_t slot = t; slot < nio; slot += BT) {
        const uint32_t hw = src[off + 128 + slot / 2];
        const uint32_t hook = (slot & 1) ? (hw >> 16) : (hw & 0xffffu);
        if ((hook >> 8) == (uint32_t)ci) ext_bits[hook & 255u] = 0xffffffffu;
      }
      __syncthreads();
      // top-down, one level per pass: position 1, then [2, 4), ..., [4096, 8192)
      if (t == 0) live[0] = 0;
      for (uint32_t M = 1; M <= 4096; M <<= 1) {
        for (uint32_t c = M + t; c < 2 * M; c += BT) {
          uint8_t l = (uint8_t)((ext_bits[c >> 5] >> (c & 31)) & 1u);
          if (M > 1) {
            const uint32_t h = M >> 1;
            l |= live[c < M + h ? c - h : c - M];
          }
          live[c] = l;
        }
        __syncthreads();
      }
      const int deep = __syncthreads_or(t > 0 && live[t]);  // BT = 512
      int upper = 0;  // any live position in [512, 4096) (levels 2..4)
      for (uint32_t c = 512 + t; c < 4096; c += BT) upper |= live[c];
      const int flat = !deep && !__syncthreads_or(upper);  // level 1 only
      deep0 = deep;
      flat0 = flat;
      all_flat &= flat;
      if (ci < (int)COMPACT_MAX_STAGES)
        for (uint32_t w = t; w < 256; w += BT) ps.ext_all[ci][w] = ext_bits[w];
      for (uint32_t w = t; w < 256; w += BT) need_bits[w] = 0;
      __syncthreads();
      // stage 0's entries name global-read slots, known once the needed
      // global-read positions are compacted (below)
      write_entries(C, D, deep, flat, ci > 0, false);
      uint32_t A = 0, B = 0;
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const uint32_t p = owned_pos(u, i);
        if (i == 15 && u < 16) continue;
        const uint32_t *F = C + 4096 + 4 * (p >> 5);
        A |= ((F[0] >> (p & 31)) & 1u) << i;
        A |= ((F[1] >> (p & 31)) & 1u) << (16 + i);
        B |= ((F[2] >> (p & 31)) & 1u) << i;
        // owned position i read from outside its stage (threads t < 8 of
        // deep stages hold the warp-0 flags there instead)
        if (t >= 8 || !deep) B |= ((ext_bits[p >> 5] >> (p & 31)) & 1u) << (16 + i);
      }
      if (t < 8 && deep) {
#pragma unroll
        for (int m = 0; m < 4; ++m) {
          const uint32_t len = 8u >> m;
          if (t >= len) continue;
          const uint32_t p = len + t;
          const uint32_t *F = C + 4096 + 4 * (p >> 5);
          B |= ((F[0] >> (p & 31)) & 1u) << (16 + m);
          B |= ((F[1] >> (p & 31)) & 1u) << (20 + m);
          B |= ((F[2] >> (p & 31)) & 1u) << (24 + m);
        }
      }
      D[4096 + 2 * t] = A;
      D[4096 + 2 * t + 1] = B;
      __syncthreads();  // need_bits complete; ext_bits and live free
    }
    // global-read sources: thread t < 256 appends its masked bits round by
    // round, walking each mask from the lowest set bit; the first appended
    // bit ends up most significant, i.e. at position 32t + total - 1
    // (csrc/kernel_v1_impl.cuh:87-154); unfilled positions are GR_EMPTY.
    uint32_t *row = gr_sources + pid * 8192;
    if (t < 256) {
      const uint32_t *gr = src + off + 256;
      uint32_t *G = row + 32 * t;
      uint32_t total = 0;
      for (uint32_t r = 0; r < R; ++r) total += __popc(gr[512 * r + 2 * t + 1]);
      if (total > 32) total = 32;  // at most 32 bits per thread (script validator)
      uint32_t i = 0;
      for (uint32_t r = 0; r < R; ++r) {
        uint32_t m = gr[512 * r + 2 * t + 1];
        const uint32_t idx = gr[512 * r + 2 * t];
        const uint32_t stg = idx & 0x80000000u, w = idx & 0x7fffffffu;
        while (m && i < 32) {
          const uint32_t k = __ffs(m) - 1;
          m &= m - 1;
          G[total - 1 - i] = stg | (w * 32 + k);
          ++i;
        }
      }
      for (uint32_t k = total; k < 32; ++k) G[k] = GR_EMPTY;
    }
    __syncthreads();
    // Compaction: the global-read positions stage 0 needs, in position
    // order, take slots 0, 1, ... of the row (the rest GR_SKIP), so the
    // kernel's global read has no idle lanes; slot s lands in shared-memory
    // word sw(s).  Thread t owns positions 16t .. 16t+15.
    uint32_t n_gr = 0;
    {
      const uint32_t keep = (need_bits[t >> 1] >> (16 * (t & 1))) & 0xffffu;
      uint32_t vals[16];
#pragma unroll
      for (int j = 0; j < 16; ++j) vals[j] = (keep >> j) & 1u ? row[16 * t + j] : 0u;
      uint32_t base = block_excl_scan(__popc(keep), ps.warp_sum, &n_gr);  // row reads done
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        ps.slot_prev[16 * t + j] = (keep >> j) & 1u ? (uint16_t)sw(base) : (uint16_t)0xffffu;
        if ((keep >> j) & 1u) row[base++] = vals[j];
      }
      for (uint32_t i = n_gr + t; i < 8192; i += BT) row[i] = GR_SKIP;
    }
    __syncthreads();
    write_entries(ch, dch, deep0, flat0, true, true);
    // ---- compact form, when every stage evaluates only level 1 and only
    // positions read from outside.  Stage ci's live positions get the slots
    // of a region of shared memory (its hooked 32-position groups as 32-slot
    // blocks, then the other positions), at the top of the tree buffer for
    // even ci and at the bottom for odd ci, so a stage never writes what it
    // reads and needs one barrier; the global read (slot s at word sw(s),
    // below 32 * ceil(n_gr / 32)) sits at the bottom.  Where stage 0's region
    // reaches into it, the first `ov` slots of stage 0 (at most 4 per
    // thread) are held until every thread has read the global read.  The
    // chunk becomes one word per slot: source words a | b << 13, flags xa <<
    // 26, xb << 27, ob << 28, zero-source flags << 29 (a) and << 30 (b),
    // after a header of four words: the slot count, the region's first word,
    // ov and 0.  Hooks are rewritten to (stage << 8) | block.  Metadata word
    // 10 bit 0 marks the form, words 11 + k the bytes of chunk k to copy
    // (header and slot words; 0 = the whole chunk).
    bool compact = all_flat && ns <= COMPACT_MAX_STAGES;
    const uint32_t gr_top = (n_gr + 31) & ~31u;
    // Direct variant of the compact form: a level-1 position whose b input
    // is forced (ob) only passes its a input on, value a ^ xa and X plane
    // a_x, so unless a hook reads it, it is not stored: its readers take its
    // source instead, with xa folded into their own xa / xb (a ^ xa ^ xa_r
    // and the X plane are unchanged).  Stage regions then follow the global
    // read one after another (nothing is overwritten, so a value lives until
    // the partition ends), which needs the global read plus every stage's
    // stored slots to fit 8192 positions; otherwise the carries stay and the
    // regions alternate ends of the buffer.
    bool direct = false;
    if (compact) {
      uint32_t total = gr_top;
      for (uint32_t ci = 0; ci < ns; ++ci) {
        const uint32_t *C = ch + (size_t)ci * STAGE_WORDS;
        const uint32_t *ex = ps.ext_all[ci];
        if (t < 8) ps.hmask[t] = 0;
        __syncthreads();
        for (uint32_t slot = t; slot < nio; slot += BT) {
          const uint32_t hw = src[off + 128 + slot / 2];
          const uint32_t hook = (slot & 1) ? (hw >> 16) : (hw & 0xffffu);
          if ((hook >> 8) == ci) atomicOr(&ps.hmask[(hook & 255u) >> 5], 1u << (hook & 31u));
        }
        __syncthreads();
        uint32_t nh = 0;
        for (int w = 0; w < 8; ++w) nh += __popc(ps.hmask[w]);
        uint32_t cnt = 0;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const uint32_t pp = 4096 + 8 * t + j;
          const bool hk = (ps.hmask[pp >> 10] >> ((pp >> 5) & 31)) & 1u;
          const bool ob = (C[4096 + 4 * (pp >> 5) + 2] >> (pp & 31)) & 1u;
          if (((ex[pp >> 5] >> (pp & 31)) & 1u) && !hk && !ob) ++cnt;
        }
        uint32_t no = 0;
        block_excl_scan(cnt, ps.warp_sum, &no);  // ends with a barrier-free read
        total += 32 * nh + no;
        __syncthreads();  // hmask read by every thread before the next reset
      }
      direct = total <= 8192;
    }
    // Source references of the previous stage's positions (slot_prev) and of
    // this stage's (slot_cur): a shared-memory word below 8192, bit 13 set
    // when the value is to be inverted (direct variant), REF_ZERO for the
    // constant 0 (and for positions nothing reads), REF_ONE for constant 1.
    constexpr uint32_t REF_ZERO = 0xffffu, REF_ONE = 0xfffeu;
    uint32_t next_base = gr_top;  // end of the stage regions (direct variant)
    if (compact) {
      for (uint32_t ci = 0; ci < ns; ++ci) {
        const uint32_t *C = ch + (size_t)ci * STAGE_WORDS;
        uint32_t *D = dch + (size_t)ci * STAGE_WORDS;
        const uint32_t *ex = ps.ext_all[ci];
        if (t < 8) ps.hmask[t] = 0;
        __syncthreads();
        for (uint32_t slot = t; slot < nio; slot += BT) {
          const uint32_t hw = src[off + 128 + slot / 2];
          const uint32_t hook = (slot & 1) ? (hw >> 16) : (hw & 0xffffu);
          if ((hook >> 8) == ci) atomicOr(&ps.hmask[(hook & 255u) >> 5], 1u << (hook & 31u));
        }
        __syncthreads();
        const bool hooked_t = t < 256 && ((ps.hmask[t >> 5] >> (t & 31)) & 1u);
        uint32_t nh = 0;
        const uint32_t bg = block_excl_scan(hooked_t ? 1u : 0u, ps.warp_sum, &nh);
        if (hooked_t) ps.blk_of[t] = (uint16_t)bg;
        // other level-1 positions read from outside: thread t owns
        // 4096+8t..+7; in the direct variant the pass-throughs among them are
        // aliases (`alias`), not slots
        uint32_t mine = 0, alias = 0;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const uint32_t pp = 4096 + 8 * t + j;
          const bool hk = (ps.hmask[pp >> 10] >> ((pp >> 5) & 31)) & 1u;
          const bool ob = (C[4096 + 4 * (pp >> 5) + 2] >> (pp & 31)) & 1u;
          if (((ex[pp >> 5] >> (pp & 31)) & 1u) && !hk) {
            if (direct && ob)
              alias |= 1u << j;
            else
              mine |= 1u << j;
          }
        }
        uint32_t no = 0;
        uint32_t rk = block_excl_scan(__popc(mine), ps.warp_sum, &no);
        const uint32_t n = 32 * nh + no;
        const uint32_t base = direct ? next_base : (ci & 1) ? 0u : 8192u - n;
        next_base += n;
        const uint32_t ov = (!direct && ci == 0 && gr_top > base) ? gr_top - base : 0u;
        if (ov > 4 * BT) {  // stage 0 only (uniform): keep the tree form
          compact = false;
          break;
        }
        for (uint32_t pp = t; pp < 8192; pp += BT) ps.slot_cur[pp] = (uint16_t)REF_ZERO;
        __syncthreads();
        for (uint32_t pp = t; pp < 8192; pp += BT) {
          const uint32_t g = pp >> 5;
          if ((ps.hmask[g >> 5] >> (g & 31)) & 1u) {
            const uint32_t sl = 32 * ps.blk_of[g] + (pp & 31);
            ps.slot_cur[pp] = (uint16_t)(base + sl);
            ps.pos_of[sl] = (uint16_t)pp;
          }
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const uint32_t pp = 4096 + 8 * t + j;
          if ((mine >> j) & 1u) {
            const uint32_t sl = 32 * nh + rk++;
            ps.slot_cur[pp] = (uint16_t)(base + sl);
            ps.pos_of[sl] = (uint16_t)pp;
          } else if ((alias >> j) & 1u) {
            // the a input's reference, inverted once more when xa is set
            const uint32_t xa = (C[4096 + 4 * (pp >> 5)] >> (pp & 31)) & 1u;
            const uint32_t sa = perm_src(C, pp - 4096) & 8191u;
            uint32_t r = (ci > 0 && sa == 0) ? REF_ZERO : ps.slot_prev[sa];
            if (xa) r = r == REF_ZERO ? REF_ONE : r == REF_ONE ? REF_ZERO : r ^ (1u << 13);
            ps.slot_cur[pp] = (uint16_t)r;
          }
        }
        __syncthreads();
        // Bank-aware order of the slots no hook reads ([32 nh, n)).  A gather
        // of the kernel's compact stage reads 16 bytes per lane, and the 8
        // lanes of a quarter warp are served in one wavefront when their
        // addresses fall in distinct 16-byte bank groups (word mod 8).  Each
        // group of 8 slots (a quarter warp: the region starts 32-aligned
        // after the hooked blocks) takes entries whose a sources, and whose b
        // sources, lie in distinct bank groups where the remaining entries
        // allow it (greedy, fullest bucket first).
        {
          const uint32_t h0 = 32 * nh, m = n - h0;
          for (uint32_t i = t; i < m; i += BT) {
            const uint32_t P = ps.pos_of[h0 + i];
            const uint32_t ob = (C[4096 + 4 * (P >> 5) + 2] >> (P & 31)) & 1u;
            const uint32_t sa = perm_src(C, P - 4096) & 8191u, sb = perm_src(C, P) & 8191u;
            const uint32_t ra = (ci > 0 && sa == 0) ? REF_ZERO : ps.slot_prev[sa];
            const uint32_t rb = (ob || (ci > 0 && sb == 0)) ? REF_ZERO : ps.slot_prev[sb];
            const uint32_t ba = ra >= REF_ONE ? 8u : (ra & 7u), bb = rb >= REF_ONE ? 8u : (rb & 7u);
            ps.bucket_of[i] = (uint8_t)(9 * ba + bb);
          }
          if (t < 81) ps.bcnt[t] = 0;
          __syncthreads();
          if (t == 0 && m > 8) {
            for (uint32_t i = 0; i < m; ++i) ++ps.bcnt[ps.bucket_of[i]];
            uint32_t acc = 0;
            for (int b = 0; b < 81; ++b) {
              ps.bptr[b] = (uint16_t)acc;
              acc += ps.bcnt[b];
            }
            for (uint32_t i = 0; i < m; ++i) ps.sorted[ps.bptr[ps.bucket_of[i]]++] = (uint16_t)i;
            for (int b = 0; b < 81; ++b) ps.bptr[b] = (uint16_t)(ps.bptr[b] - ps.bcnt[b]);
            for (uint32_t g = 0; g < m; g += 8) {
              uint32_t used_a = 0, used_b = 0;
              for (uint32_t k = 0; k < 8 && g + k < m; ++k) {
                int best = -1, any = -1;
                uint32_t best_c = 0, any_c = 0;
                for (int b = 0; b < 81; ++b) {
                  const uint32_t c = ps.bcnt[b];
                  if (!c) continue;
                  if (c > any_c) { any = b; any_c = c; }
                  const uint32_t ba = (uint32_t)b / 9, bb = (uint32_t)b % 9;
                  const bool free_a = ba == 8 || !((used_a >> ba) & 1u);
                  const bool free_b = bb == 8 || !((used_b >> bb) & 1u);
                  if (free_a && free_b && c > best_c) { best = b; best_c = c; }
                }
                if (best < 0) best = any;
                ps.order[g + k] = ps.sorted[ps.bptr[best] + --ps.bcnt[best]];
                const uint32_t ba = (uint32_t)best / 9, bb = (uint32_t)best % 9;
                if (ba < 8) used_a |= 1u << ba;
                if (bb < 8) used_b |= 1u << bb;
              }
            }
          } else if (t == 0) {
            for (uint32_t i = 0; i < m; ++i) ps.order[i] = (uint16_t)i;
          }
          __syncthreads();
          for (uint32_t i = t; i < m; i += BT) ps.sorted[i] = ps.pos_of[h0 + ps.order[i]];
          __syncthreads();
          for (uint32_t i = t; i < m; i += BT) {
            const uint32_t P = ps.sorted[i];
            ps.pos_of[h0 + i] = (uint16_t)P;
            ps.slot_cur[P] = (uint16_t)(base + h0 + i);
          }
          __syncthreads();
        }
        for (uint32_t i = t; i < n; i += BT) {
          const uint32_t P = ps.pos_of[i];
          const uint32_t *F = C + 4096 + 4 * (P >> 5);
          uint32_t xa = (F[0] >> (P & 31)) & 1u, xb = (F[1] >> (P & 31)) & 1u;
          const uint32_t ob = (F[2] >> (P & 31)) & 1u;
          const uint32_t sa = perm_src(C, P - 4096) & 8191u, sb = perm_src(C, P) & 8191u;
          // a source of stage >= 1 at position 0 is the constant 0
          const uint32_t ra = (ci > 0 && sa == 0) ? REF_ZERO : ps.slot_prev[sa];
          const uint32_t rb = (ob || (ci > 0 && sb == 0)) ? REF_ZERO : ps.slot_prev[sb];
          const uint32_t za = ra >= REF_ONE, zb = rb >= REF_ONE;
          // an inverted source (or the constant 1) flips the input's own flag
          xa ^= za ? (ra == REF_ONE) : (ra >> 13) & 1u;
          xb ^= zb ? (rb == REF_ONE) : (rb >> 13) & 1u;
          const uint32_t wa = za ? 0u : ra & 8191u, wb = zb ? 0u : rb & 8191u;
          D[4 + i] = wa | (wb << 13) | (xa << 26) | (xb << 27) | (ob << 28) | (za << 29) | (zb << 30);
        }
        if (t == 0) {
          D[0] = n;
          D[1] = base;
          D[2] = ov;
          D[3] = 0;
          // copy size of this chunk: the header and the slot words
          dst[off + 11 + ci] = ((4 + n) * 4 + 15) & ~15u;
        }
        if (t < 128 && 2 * t < nio) {  // meta word 128 + t: hooks of slots 2t, 2t+1
          uint32_t w = dst[off + 128 + t];
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const uint32_t hk = (w >> (16 * h)) & 0xffffu;
            if (2 * t + h < nio && (hk >> 8) == ci) {
              const uint32_t nw = (ci << 8) | ps.blk_of[hk & 255u];
              w = (w & ~(0xffffu << (16 * h))) | (nw << (16 * h));
            }
          }
          dst[off + 128 + t] = w;
        }
        __syncthreads();
        for (uint32_t pp = t; pp < 8192; pp += BT) ps.slot_prev[pp] = ps.slot_cur[pp];
        __syncthreads();
      }
    }
    // Metadata word 127: the 64-byte tree slots an octet item needs for this
    // partition (run_item8: global-read slots, stage regions, then the SRAM
    // stage's staged words and read-outs), or ~0 when the octet form cannot
    // run it: it needs the compact form without carries (regions never
    // overwritten, so writeouts name tree slots), at most OCT_MAX_GR
    // global-read slots, and a hook for every writeout slot but the SRAM and
    // duplicate ones.
    {
      const uint32_t nsr = src[off + 4], ndup = src[off + 7];
      bool hooked = true;
      for (uint32_t j = t; j < nio; j += BT) {
        const uint32_t hw = src[off + 128 + j / 2];
        const uint32_t hook = (j & 1) ? (hw >> 16) : (hw & 0xffffu);
        if (j + nsr + ndup < nio && (hook >> 8) >= ns) hooked = false;
      }
      hooked = !__syncthreads_or(!hooked);
      if (t == 0) {
        const bool oct = compact && direct && hooked && n_gr <= OCT_MAX_GR;
        dst[off + 127] = oct ? ((next_base + 31) & ~31u) + (nsr * 4 + ndup) * 32 + nsr * 32
                             : 0xffffffffu;
      }
    }
    if (t == 0) dst[off + 10] = compact ? 1u : 0u;
    // SRAM/duplicate and clock-enable chunks: shuffle entries in q order, two
    // per word.  In the compact form only the nq entries the kernel reads are
    // kept, followed by their flag words (perm_flag_off), and the chunk's copy
    // size (metadata word 11 + ci) ends there; otherwise all 8192 entries,
    // flags at word 4096 as in the script.
    for (uint32_t ci = ns; ci < ns + 2; ++ci) {
      const uint32_t *C = ch + (size_t)ci * STAGE_WORDS;
      uint32_t *D = dch + (size_t)ci * STAGE_WORDS;
      const uint32_t nq = ci == ns ? (src[off + 4] * 4 + src[off + 7]) * 32 : nio * 32;
      const uint32_t n2 = compact ? nq / 2 : 4096;
      for (uint32_t q2 = t; q2 < n2; q2 += BT)
        D[q2] = perm_src(C, 2 * q2) | (perm_src(C, 2 * q2 + 1) << 16);
      if (compact) {
        const uint32_t fo = perm_flag_off(nq), nf = 4 * (nq / 32);
        for (uint32_t i = t; i < nf; i += BT) D[fo + i] = C[4096 + i];
        if (t == 0) {
          const uint32_t bytes = (fo + nf) * 4;
          dst[off + 11 + ci] = bytes < 16 ? 16u : bytes;
        }
      }
    }
    // an octet item copies all of a partition's chunks into its two chunk
    // buffers at once: a partition whose copies do not fit is not admitted
    if (t == 0 && compact && dst[off + 127] != 0xffffffffu) {
      const bool sr = (src[off + 4] | src[off + 7]) != 0;
      uint32_t total = dst[off + 12 + ns];  // clock-enable chunk
      if (sr) total += dst[off + 11 + ns];
      for (uint32_t ci = 0; ci < ns; ++ci) total += dst[off + 11 + ci];
      if (total > 2 * CHUNK_BYTES) dst[off + 127] = 0xffffffffu;
    }
    __syncthreads();  // shared state read before the next partition reuses it
    off += 256 + 512 * (size_t)R + STAGE_WORDS * ((size_t)ns + 2);
    ++pid;
    if (is_last) break;
  }
}

// Largest octet slot need (metadata word 127 of the prepared script) over
// each entry's partition list, into *need by atomic maximum.
__global__ void jq_batched_need_kernel(const size_t *blocks_start, const uint32_t *prep,
                                       uint32_t *need, unsigned entries) {
  const unsigned e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= entries) return;
  size_t off = blocks_start[e];
  uint32_t m = 0;
  for (;;) {
    const uint32_t ns = prep[off];
    if (!ns) break;
    const uint32_t w = prep[off + 127];
    m = w > m ? w : m;
    if (prep[off + 1]) break;
    off += 256 + 512 * (size_t)prep[off + 6] + STAGE_WORDS * ((size_t)ns + 2);
  }
  if (m) atomicMax(need, m);
}

// Number of partitions in each (major stage, block) entry's list.
__global__ void jq_batched_count_kernel(const size_t *blocks_start, const uint32_t *src,
                                        uint32_t *counts, unsigned entries) {
  const unsigned e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= entries) return;
  size_t off = blocks_start[e];
  uint32_t n = 0;
  for (;;) {
    const uint32_t ns = src[off];
    if (!ns) break;
    ++n;
    if (src[off + 1]) break;
    off += 256 + 512 * (size_t)src[off + 6] + STAGE_WORDS * ((size_t)ns + 2);
  }
  counts[e] = n;
}

}  // namespace jqk

using namespace jqk;

// Lane-major [lane][signal] snapshot <-> the interleaved batched state.
__global__ void jq_batched_pack_kernel(const uint32_t *lm, uint32_t *st, uint32_t lanes,
                                       size_t sig, int layout, int unpack) {
  const size_t n = (size_t)lanes * sig;
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
       q += (size_t)gridDim.x * blockDim.x) {
    const size_t w = phys(layout, sig / 2, sig, (uint32_t)(q / sig), q % sig);
    if (unpack)
      st[q] = lm[w];  // st: lane-major output, lm: batched input
    else
      st[w] = lm[q];
  }
}

// Re-arms one slot's barrier, ticket and status before a launch.  A kernel
// (not a host copy) so the reset is captured in CUDA graphs with the launch.
__global__ void jq_batched_reset_kernel(int slot) {
  g_bcount[slot] = 0;
  g_bticket[slot] = 0;
  g_status[slot] = 0;
  for (uint32_t g = 0; g < MAX_GROUPS; ++g) g_bgroup[(size_t)slot * MAX_GROUPS + g] = 0;
}

extern "C" {

// Kernel variant: lane words per work item and tree-state buffering.
struct Variant {
  int nl;   // 1, 2 or 8 lane words per item
  bool ds;  // double-buffered tree state (nl == 1 only)
};

static const void *variant_fn(Variant v) {
  if (v.nl == 8) return (const void *)jq_batched_kernel<false, 8>;
  if (v.nl == 2) return (const void *)jq_batched_kernel<false, 2>;
  return v.ds ? (const void *)jq_batched_kernel<true, 1> : (const void *)jq_batched_kernel<false, 1>;
}

// Opt-in shared memory per CTA left for the dynamic part of variant v.
static size_t dyn_smem_limit(Variant v) {
  int dev = 0, optin = 0;
  cudaFuncAttributes fa;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess ||
      cudaFuncGetAttributes(&fa, variant_fn(v)) != cudaSuccess || (size_t)optin < fa.sharedSizeBytes)
    return 0;
  return (size_t)optin - fa.sharedSizeBytes;
}

// 64-byte tree slots of an octet item: what the opt-in shared memory leaves
// after the chunk buffers and the writeout map.
static uint32_t oct_slot_capacity() {
  const size_t lim = dyn_smem_limit(Variant{8, false});
  const size_t fixed = 2 * (size_t)CHUNK_BYTES + OCT_AUX_WORDS * 4;
  if (lim <= fixed) return 0;
  const size_t n = (lim - fixed) / 64;
  return (uint32_t)(n < 8192 ? n : 8192);
}

static size_t smem_layout_bytes(uint32_t wo_slots, Variant v) {
  if (v.nl == 8) return 2 * (size_t)CHUNK_BYTES + OCT_AUX_WORDS * 4 + (size_t)oct_slot_capacity() * 64;
  const size_t wb = v.nl == 2 ? 16 : 8;
  return 2 * (size_t)CHUNK_BYTES + (v.ds ? 2 : 1) * 8192 * wb + (size_t)wo_slots * 32 * wb;
}

static bool variant_fits(uint32_t wo_slots, Variant v) {
  return smem_layout_bytes(wo_slots, v) <= dyn_smem_limit(v);
}

// want_nl 0 = automatic: lane pairs when the lane count is even and their
// shared memory fits, else single lanes, double-buffered when that fits.
// The octet layout (2) runs octet items only.  nl = 0 in the result: the
// requested variant is not possible.
static Variant pick_variant(uint32_t wo_slots, uint32_t lanes, uint32_t want_nl, int layout) {
  if (layout == 2)
    return (want_nl == 0 || want_nl == 8) && lanes % 8 == 0 && oct_slot_capacity() > 0
               ? Variant{8, false}
               : Variant{0, false};
  if (want_nl == 8) return Variant{0, false};
  if (want_nl != 1 && lanes % 2 == 0 && variant_fits(wo_slots, Variant{2, false}))
    return Variant{2, false};
  if (want_nl == 2) return Variant{0, false};
  return Variant{1, variant_fits(wo_slots, Variant{1, true})};
}

int jq_batched_smem_bytes(uint32_t wo_slots) {
  return (int)smem_layout_bytes(wo_slots, pick_variant(wo_slots, 1, 1, 0));
}

static int variant_max_blocks(int device, uint32_t wo_slots, Variant v, size_t *max_blocks) {
  const void *fn = variant_fn(v);
  const int smem = (int)smem_layout_bytes(wo_slots, v);
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)
    return JQ_ERR_LAUNCH;
  int sms = 0, per = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, BT, smem) != cudaSuccess)
    return JQ_ERR_LAUNCH;
  *max_blocks = (size_t)sms * per;
  return JQ_OK;
}

int jq_batched_max_blocks(int device, uint32_t wo_slots, size_t *max_blocks) {
  // every variant runs one CTA per SM
  return variant_max_blocks(device, wo_slots, pick_variant(wo_slots, 1, 1, 0), max_blocks);
}

int jq_batched_oct_capacity(uint32_t *slots) {
  if (!slots) return JQ_ERR_INVALID_ARG;
  *slots = oct_slot_capacity();
  return JQ_OK;
}

size_t jq_batched_gr_words(size_t num_partitions) { return (num_partitions + 1) * 8192; }

size_t jq_batched_state_words(uint32_t lanes, size_t signals) {
  return (size_t)((lanes + 1) & ~1u) * signals;
}

static int pack_launch(const uint32_t *src, uint32_t *dst, uint32_t lanes, size_t signals,
                       int32_t x_interleaved, int unpack, void *stream) {
  if (!src || !dst || lanes == 0 || signals == 0 || x_interleaved < 0 || x_interleaved > 2 ||
      (x_interleaved && (signals & 1)) || (x_interleaved == 2 && lanes % 8))
    return JQ_ERR_INVALID_ARG;
  const size_t n = (size_t)lanes * signals;
  const unsigned grid = (unsigned)((n + 255) / 256 < 148 * 16 ? (n + 255) / 256 : 148 * 16);
  jq_batched_pack_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(src, dst, lanes, signals,
                                                                   x_interleaved, unpack);
  return cudaGetLastError() == cudaSuccess ? JQ_OK : JQ_ERR_LAUNCH;
}

int jq_batched_pack_state(const uint32_t *lane_major, uint32_t lanes, size_t signals,
                          int32_t x_interleaved, uint32_t *state, void *stream) {
  return pack_launch(lane_major, state, lanes, signals, x_interleaved, 0, stream);
}

int jq_batched_unpack_state(const uint32_t *state, uint32_t lanes, size_t signals,
                            int32_t x_interleaved, uint32_t *lane_major, void *stream) {
  return pack_launch(state, lane_major, lanes, signals, x_interleaved, 1, stream);
}

int jq_batched_prepare(const size_t *blocks_start, const uint32_t *blocks_data,
                       size_t blocks_data_len, size_t num_blocks, size_t num_major_stages,
                       size_t num_partitions, uint32_t *out, uint32_t *part_base,
                       uint32_t *gr_sources, void *stream) {
  if (!blocks_start || !blocks_data || !out || !part_base || !gr_sources || num_blocks == 0 ||
      num_major_stages == 0 || out == blocks_data)
    return JQ_ERR_INVALID_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  const size_t entries = num_blocks * num_major_stages;
  jq_batched_count_kernel<<<(unsigned)((entries + 255) / 256), 256, 0, st>>>(
      blocks_start, blocks_data, part_base, (unsigned)entries);
  if (cudaGetLastError() != cudaSuccess) return JQ_ERR_LAUNCH;
  uint32_t *h = (uint32_t *)malloc(entries * sizeof(uint32_t));
  if (!h) return JQ_ERR_INVALID_ARG;
  if (cudaMemcpyAsync(h, part_base, entries * sizeof(uint32_t), cudaMemcpyDeviceToHost, st) !=
          cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess) {
    free(h);
    return JQ_ERR_CUDA;
  }
  // counts -> first partition index of each entry (script order)
  size_t total = 0;
  for (size_t e = 0; e < entries; ++e) {
    const uint32_t c = h[e];
    h[e] = (uint32_t)total;
    total += c;
  }
  int rc = JQ_OK;
  if (total != num_partitions) {
    rc = JQ_ERR_INVALID_ARG;
  } else if (cudaMemcpyAsync(part_base, h, entries * sizeof(uint32_t), cudaMemcpyHostToDevice,
                             st) != cudaSuccess ||
             cudaMemcpyAsync(out, blocks_data, blocks_data_len * sizeof(uint32_t),
                             cudaMemcpyDeviceToDevice, st) != cudaSuccess) {
    rc = JQ_ERR_CUDA;
  } else {
    const int psmem = (int)sizeof(PrepShared);
    if (cudaFuncSetAttribute(jq_batched_prepare_kernel,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, psmem) != cudaSuccess) {
      rc = JQ_ERR_LAUNCH;
    } else {
      jq_batched_prepare_kernel<<<(unsigned)entries, BT, psmem, st>>>(
          blocks_start, blocks_data, out, (unsigned)entries, part_base, gr_sources,
          num_partitions);
      if (cudaGetLastError() != cudaSuccess) rc = JQ_ERR_LAUNCH;
      else if (cudaStreamSynchronize(st) != cudaSuccess) rc = JQ_ERR_CUDA;
    }
  }
  free(h);
  return rc;
}

int jq_batched_slot_need(const size_t *blocks_start, const uint32_t *prepared, size_t num_blocks,
                         size_t num_major_stages, uint32_t *need, void *stream) {
  if (!blocks_start || !prepared || !need || num_blocks == 0 || num_major_stages == 0)
    return JQ_ERR_INVALID_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  const size_t entries = num_blocks * num_major_stages;
  if (cudaMemsetAsync(need, 0, sizeof(uint32_t), st) != cudaSuccess) return JQ_ERR_CUDA;
  jq_batched_need_kernel<<<(unsigned)((entries + 255) / 256), 256, 0, st>>>(
      blocks_start, prepared, need, (unsigned)entries);
  return cudaGetLastError() == cudaSuccess ? JQ_OK : JQ_ERR_LAUNCH;
}

int jq_simulate_batched(const jq_batch_args *a) {
  if (!a || a->lanes == 0 || a->num_blocks == 0 || a->num_major_stages == 0 ||
      a->num_major_stages > 32 || !a->state_a || !a->state_b || a->wo_slots > 256 ||
      (a->n_po && (!a->po_signals || !a->wave)))
    return JQ_ERR_INVALID_ARG;
  cudaStream_t st = (cudaStream_t)a->stream;
  int dev = 0;
  cudaGetDevice(&dev);
  const uint32_t wo_slots = a->wo_slots ? a->wo_slots : 256;
  if ((a->lanes_per_item > 2 && a->lanes_per_item != 8) || a->x_interleaved < 0 ||
      a->x_interleaved > 2)
    return JQ_ERR_INVALID_ARG;
  const Variant v = pick_variant(wo_slots, a->lanes, a->lanes_per_item, a->x_interleaved);
  if (v.nl == 0) return JQ_ERR_INVALID_ARG;
  size_t maxg = 0;
  if (variant_max_blocks(dev, wo_slots, v, &maxg) != JQ_OK || maxg == 0) return JQ_ERR_LAUNCH;
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
  if (a->x_interleaved && (P.sig_per_snap & 1)) return JQ_ERR_INVALID_ARG;
  P.xhalf = a->x_interleaved != 0;
  P.layout = a->x_interleaved;
  P.slot_cap = v.nl == 8 ? oct_slot_capacity() : 0;
  P.vsig = P.xhalf ? P.sig_per_snap / 2 : P.sig_per_snap;
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
  P.wo_slots = wo_slots;
  P.block_list = a->block_list;
  P.block_list_start = a->block_list_start;
  P.part_cycles = a->part_cycles;
  P.part_base = a->part_base;
  P.gr_sources = a->gr_sources;
  if (!P.part_base || !P.gr_sources) return JQ_ERR_INVALID_ARG;
  P.constraints = a->timing_constraints;
  P.arr_first = a->arrival_first;
  P.arr_steady = a->arrival_steady;
  P.events = a->events;
  P.event_cap = a->event_capacity;
  P.first_cycle = a->first_cycle;
  if (P.constraints && (!P.arr_first || !P.arr_steady || !P.events)) return JQ_ERR_INVALID_ARG;
  P.timeout = a->barrier_timeout_cycles ? a->barrier_timeout_cycles : DEFAULT_BARRIER_TIMEOUT;
  P.chunk_timeout = DEFAULT_BARRIER_TIMEOUT;
  P.slot = launch_slot(a->stream, true);
  if (P.slot < 0) return JQ_ERR_TOO_MANY_STREAMS;
  jq_batched_reset_kernel<<<1, 1, 0, st>>>(P.slot);
  if (cudaGetLastError() != cudaSuccess) return JQ_ERR_LAUNCH;
  const int smem = (int)smem_layout_bytes(P.wo_slots, v);
  void *args[] = {&P};
  cudaError_t e = cudaLaunchCooperativeKernel(variant_fn(v), (unsigned)grid, BT, args, smem, st);
  return e == cudaSuccess ? JQ_OK : JQ_ERR_LAUNCH;
}

int jq_batched_status(void *stream) {
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

}  // extern "C"
