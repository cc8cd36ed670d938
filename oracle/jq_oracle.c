/*
 * jq_oracle.c -- CPU oracle for the Boolean-processor interpreter.
 *
 * TEST INFRASTRUCTURE ONLY (see jq_oracle.h).  A plain-C restatement of the
 * reference's CPU executor and of the CUDA kernel's observable semantics, used
 * to check the product kernels bit for bit.  Function-level citations below
 * point at the reference file:line each block follows.
 */
#define _GNU_SOURCE
#include "jq_oracle.h"

#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#define NT 256                 /* threads per block: src/flatten.rs:24 */
#define SRAM_WORDS 8192u       /* AIGPDK_SRAM_SIZE: src/aigpdk.rs:20-22 */
#define STAGE_WORDS 5120u      /* 4 shuffle chunks + 1 flag chunk of 256x4 */

#define E_SCRIPT_OVERRUN -1
#define E_STATE_OOB -2
#define E_SRAM_OOB -3
#define E_TOO_MANY_STAGES -4
#define E_SIZE_MISMATCH -5

/* Per-block state the kernel keeps in shared memory for the whole launch
 * (kernel_v1_impl.cuh:583-591): zeroed once, then only overwritten by writeout
 * hooks, SRAM reads and duplicates.  Slots that no hook writes keep older
 * values -- the oracle must carry them exactly like the CTA does. */
typedef struct {
  uint32_t wo[NT];
  uint32_t wo_x[NT];
  uint16_t wo_arr[NT];
} blk_persist;

typedef struct {
  jqo_event *events;
  size_t cap;
  uint64_t *count;
} event_sink;

void jqo_xprop_and(uint32_t a_v, uint32_t a_x, uint32_t b_v, uint32_t b_x,
                   uint32_t xora, uint32_t xorb, uint32_t orb, uint32_t *ret_v,
                   uint32_t *ret_x) {
  /* cpu_reference.rs:434-439 */
  uint32_t a_eff = a_v ^ xora;
  uint32_t b_eff = (b_v ^ xorb) | orb;
  uint32_t b_eff_x = b_x & ~orb;
  *ret_v = a_eff & b_eff;
  *ret_x = (a_x | b_eff_x) & (a_eff | a_x) & (b_eff | b_eff_x);
}

void jqo_dff_commit(uint32_t old_v, uint32_t old_x, uint32_t new_v,
                    uint32_t new_x, uint32_t clken, uint32_t clken_x,
                    uint32_t *wo_v, uint32_t *wo_x) {
  /* kernel_v1_impl.cuh:517-525, cpu_reference.rs:659-664 */
  *wo_v = (old_v & ~clken) | (new_v & clken);
  *wo_x = (old_x & ~clken & ~clken_x) | (new_x & clken & ~clken_x) | clken_x;
}

int jqo_setup_violation(uint16_t arrival, uint16_t setup_ps,
                        uint32_t clock_period, int32_t *slack) {
  /* kernel_v1_impl.cuh:544-545 (u32 sum, arrival 0 skipped) */
  if (arrival > 0 && (uint32_t)arrival + (uint32_t)setup_ps > clock_period) {
    *slack = (int32_t)clock_period - (int32_t)arrival - (int32_t)setup_ps;
    return 1;
  }
  return 0;
}

int jqo_hold_violation(uint16_t arrival, uint16_t hold_ps, int32_t *slack) {
  /* kernel_v1_impl.cuh:551-552 (no arrival guard) */
  if (arrival < hold_ps) {
    *slack = (int32_t)arrival - (int32_t)hold_ps;
    return 1;
  }
  return 0;
}

static void push_event(event_sink *sink, uint32_t type, uint32_t msg,
                       uint32_t cycle, uint32_t d0, uint32_t d1, uint32_t d2,
                       uint32_t d3) {
  /* event_buffer.h:89-111: the counter always advances; the record is kept
   * only while below capacity. */
  uint64_t idx = __atomic_fetch_add(sink->count, 1, __ATOMIC_RELAXED);
  if (idx < sink->cap && sink->events) {
    jqo_event *e = &sink->events[idx];
    e->event_type = type;
    e->message_id = msg;
    e->cycle = cycle;
    e->reserved = 0;
    e->data[0] = d0;
    e->data[1] = d1;
    e->data[2] = d2;
    e->data[3] = d3;
  }
}

static inline uint32_t gather16(const uint32_t *src, const uint32_t *chunk,
                                 int t) {
  /* The 16-pair bit shuffle of kernel_v1_impl.cuh:159-189 (also :368-402 and
   * :449-479): chunk k_outer holds, for thread t, four u32 words at
   * [k_outer*1024 + t*4 + k_inner]; each packs two 13-bit source indices. */
  uint32_t r = 0;
  for (int ko = 0; ko < 4; ++ko) {
    const uint32_t *w4 = chunk + ko * 1024 + t * 4;
    for (int ki = 0; ki < 4; ++ki) {
      uint32_t w = w4[ki];
      uint32_t k = (uint32_t)(ko * 4 + ki);
      uint32_t i1 = w & 0xffffu, i2 = w >> 16;
      r |= ((src[(i1 >> 5) & 255] >> (i1 & 31)) & 1u) << (k * 2);
      r |= ((src[(i2 >> 5) & 255] >> (i2 & 31)) & 1u) << (k * 2 + 1);
    }
  }
  return r;
}

static inline uint16_t arr_step(int is_pass, uint16_t a, uint16_t b,
                                uint16_t delay) {
  /* kernel_v1_impl.cuh:224-228: pass-through takes a; else max; u16 wrap. */
  uint16_t base = is_pass ? a : (a > b ? a : b);
  return (uint16_t)(base + delay);
}

/*
 * One block's partition list for one (cycle, major stage).
 * kernel_v1_impl.cuh:32-563 with the CPU loop bodies of cpu_reference.rs.
 * `state_words` bounds every state access (SIZE_MAX disables the check).
 */
static long run_block(const uint32_t *script, size_t script_size,
                      const uint32_t *in_state, uint32_t *out_state,
                      size_t state_words, uint32_t *sram, uint32_t *sram_x,
                      size_t sram_words, blk_persist *P,
                      const uint32_t *constraints, uint32_t clock_ps,
                      event_sink *sink, uint32_t cycle, int32_t arr_off,
                      int track_arr, uint32_t flags) {
  size_t pi = 0;
  int quirk_two_state = 0;
  uint32_t S[NT], SX[NT], hin[NT], hinx[NT];
  uint32_t xora[NT], xorb[NT], orb[NT];
  uint16_t dly[NT], arr[NT];
  uint16_t hooks[NT];
  uint32_t sd[NT], sdx[NT], cp[NT], cpx[NT];

  for (;;) {
    if (pi + NT > script_size) return E_SCRIPT_OVERRUN;
    const uint32_t *meta = script + pi;
    uint32_t num_stages = meta[0];
    pi += NT;
    if (!num_stages) break; /* empty block (flatten.rs:1316-1319) */
    uint32_t is_last = meta[1];
    uint32_t num_ios = meta[2];
    uint32_t io_off = meta[3];
    uint32_t num_srams = meta[4];
    uint32_t sram_off = meta[5];
    uint32_t R = meta[6];
    uint32_t num_dup = meta[7];
    int is_x = meta[8] != 0;
    uint32_t xoff = meta[9];
    if ((flags & JQO_FLAG_CPU_XPROP_QUIRK) && !is_x) quirk_two_state = 1;
    if (quirk_two_state) is_x = 0;
    for (int t = 0; t < NT; ++t) {
      uint32_t w = meta[128 + t / 2];
      hooks[t] = (uint16_t)((t & 1) ? (w >> 16) : (w & 0xffffu));
    }
    if (num_ios > NT || num_srams * 4 + num_dup > NT ||
        num_srams + num_dup > num_ios)
      return E_SCRIPT_OVERRUN;
    size_t need = (size_t)2 * NT * R + (size_t)STAGE_WORDS * (num_stages + 2);
    if (pi + need > script_size) return E_SCRIPT_OVERRUN;

    /* ---- global read: kernel_v1_impl.cuh:92-154, cpu_reference.rs:47-71 */
    for (int t = 0; t < NT; ++t) S[t] = SX[t] = 0;
    for (uint32_t r = 0; r < R; ++r) {
      const uint32_t *rd = script + pi;
      for (int t = 0; t < NT; ++t) {
        uint32_t idx = rd[2 * t], mask = rd[2 * t + 1];
        if (!mask) continue;
        const uint32_t *base = (idx >> 31) ? out_state : in_state;
        size_t w = idx & 0x7fffffffu;
        if (w >= state_words) return E_STATE_OOB;
        uint32_t value = base[w];
        uint32_t xv = 0;
        if (is_x) {
          if ((size_t)xoff + w >= state_words) return E_STATE_OOB;
          xv = base[(size_t)xoff + w];
        }
        uint32_t cur = S[t], curx = SX[t], m = mask;
        while (m) {
          uint32_t low = m & (0u - m);
          cur = (cur << 1) | ((value & low) ? 1u : 0u);
          curx = (curx << 1) | ((xv & low) ? 1u : 0u);
          m ^= low;
        }
        S[t] = cur;
        SX[t] = curx;
      }
      pi += 2 * NT;
    }
    for (int t = 0; t < NT; ++t) arr[t] = 0;

    /* ---- boomerang stages: kernel_v1_impl.cuh:156-362 */
    for (uint32_t bs = 0; bs < num_stages; ++bs) {
      const uint32_t *ch = script + pi;
      pi += STAGE_WORDS;
      for (int t = 0; t < NT; ++t) {
        hin[t] = gather16(S, ch, t);
        hinx[t] = is_x ? gather16(SX, ch, t) : 0;
        xora[t] = ch[4096 + 4 * t];
        xorb[t] = ch[4096 + 4 * t + 1];
        orb[t] = ch[4096 + 4 * t + 2];
        dly[t] = (uint16_t)(ch[4096 + 4 * t + 3] & 0xffffu);
      }
      for (int t = 0; t < NT; ++t) {
        S[t] = hin[t];
        SX[t] = hinx[t];
        arr[t] = 0; /* arrivals reset at every stage (cuh:202) */
      }
      /* level 0: threads 128..255 (cuh:206-230) */
      for (int t = 128; t < NT; ++t) {
        uint32_t rv, rx;
        jqo_xprop_and(S[t - 128], SX[t - 128], S[t], SX[t], xora[t], xorb[t],
                      orb[t], &rv, &rx);
        S[t] = rv;
        if (is_x) SX[t] = rx;
        if (track_arr)
          arr[t] = arr_step(orb[t] == 0xffffffffu, arr[t - 128], arr[t], dly[t]);
      }
      /* levels 1..7: width 64..1, thread t in [w,2w) reads t+w and t+2w
       * (smem levels cuh:236-266, warp levels cuh:270-293) */
      for (int hi = 1; hi <= 7; ++hi) {
        int w = 1 << (7 - hi);
        for (int t = w; t < 2 * w; ++t) {
          uint32_t rv, rx;
          jqo_xprop_and(S[t + w], SX[t + w], S[t + 2 * w], SX[t + 2 * w],
                        xora[t], xorb[t], orb[t], &rv, &rx);
          S[t] = rv;
          if (is_x) SX[t] = rx;
          if (track_arr)
            arr[t] = arr_step(orb[t] == 0xffffffffu, arr[t + w], arr[t + 2 * w],
                              dly[t]);
        }
      }
      /* levels 8..12: bit-level inside thread 0 (cuh:294-347); thread 0's
       * arrival is never updated and stays 0 (cuh:269, :350). */
      {
        uint32_t v1 = S[1], v1x = SX[1];
        uint32_t xa = xora[0], xb = xorb[0], ob = orb[0];
        uint32_t r8 = ((v1 << 16) ^ xa) & ((v1 ^ xb) | ob) & 0xffff0000u;
        uint32_t r9 = ((r8 >> 8) ^ xa) & (((r8 >> 16) ^ xb) | ob) & 0xff00u;
        uint32_t r10 = ((r9 >> 4) ^ xa) & (((r9 >> 8) ^ xb) | ob) & 0xf0u;
        uint32_t r11 = ((r10 >> 2) ^ xa) & (((r10 >> 4) ^ xb) | ob) & 0xcu;
        uint32_t r12 = ((r11 >> 1) ^ xa) & (((r11 >> 2) ^ xb) | ob) & 0x2u;
        S[0] = r8 | r9 | r10 | r11 | r12;
        if (is_x) {
          uint32_t d, x8, x9, x10, x11, x12;
          jqo_xprop_and(v1 << 16, v1x << 16, v1, v1x, xa, xb, ob, &d, &x8);
          x8 &= 0xffff0000u;
          jqo_xprop_and(r8 >> 8, x8 >> 8, r8 >> 16, x8 >> 16, xa, xb, ob, &d, &x9);
          x9 &= 0xff00u;
          jqo_xprop_and(r9 >> 4, x9 >> 4, r9 >> 8, x9 >> 8, xa, xb, ob, &d, &x10);
          x10 &= 0xf0u;
          jqo_xprop_and(r10 >> 2, x10 >> 2, r10 >> 4, x10 >> 4, xa, xb, ob, &d,
                        &x11);
          x11 &= 0xcu;
          jqo_xprop_and(r11 >> 1, x11 >> 1, r11 >> 2, x11 >> 2, xa, xb, ob, &d,
                        &x12);
          x12 &= 0x2u;
          SX[0] = x8 | x9 | x10 | x11 | x12;
        } else {
          SX[0] = 0;
        }
        arr[0] = 0;
      }
      /* writeout hooks (cuh:355-361) */
      for (int t = 0; t < NT; ++t) {
        uint32_t h = hooks[t];
        if ((h >> 8) == bs) {
          P->wo[t] = S[h & 255];
          if (is_x) P->wo_x[t] = SX[h & 255];
          if (track_arr) P->wo_arr[t] = arr[h & 255];
        }
      }
    }

    /* ---- SRAM & duplicate permutation (cuh:365-409, cpu:171-193) */
    {
      const uint32_t *ch = script + pi;
      pi += STAGE_WORDS;
      for (int t = 0; t < NT; ++t) {
        uint32_t inv = ch[4096 + 4 * t], set0 = ch[4096 + 4 * t + 1];
        sd[t] = (gather16(P->wo, ch, t) & ~set0) ^ inv;
        sdx[t] = is_x ? (gather16(P->wo_x, ch, t) & ~set0) : 0;
      }
    }
    /* SRAM ports, read-before-write (cuh:411-443, :483-496; cpu:195-211) */
    for (uint32_t i = 0; i < num_srams; ++i) {
      uint32_t addrs = sd[4 * i];
      uint32_t en = sd[4 * i + 1], data = sd[4 * i + 2], data_x = sdx[4 * i + 2];
      uint32_t ra = addrs & 0xffffu, wa = addrs >> 16;
      size_t st = (size_t)sram_off + (size_t)i * SRAM_WORDS;
      if (st + ra >= sram_words || st + wa >= sram_words) return E_SRAM_OOB;
      uint32_t r = sram[st + ra], w0 = sram[st + wa];
      uint32_t rx = 0, w0x = 0;
      int have_x = is_x && sram_x != NULL;
      if (have_x) {
        rx = sram_x[st + ra];
        w0x = sram_x[st + wa];
      }
      P->wo[num_ios - num_srams + i] = r;
      sram[st + wa] = (w0 & ~en) | (data & en);
      if (is_x) {
        P->wo_x[num_ios - num_srams + i] = rx;
        if (have_x) sram_x[st + wa] = (w0x & ~en) | (data_x & en);
      }
    }
    for (uint32_t i = 0; i < num_dup; ++i) {
      uint32_t slot = num_ios - num_srams - num_dup + i;
      P->wo[slot] = sd[num_srams * 4 + i];
      if (is_x) P->wo_x[slot] = sdx[num_srams * 4 + i];
    }

    /* ---- clock-enable permutation + DFF commit (cuh:446-534, cpu:234-269) */
    {
      const uint32_t *ch = script + pi;
      pi += STAGE_WORDS;
      for (int t = 0; t < NT; ++t) {
        uint32_t inv = ch[4096 + 4 * t], set0 = ch[4096 + 4 * t + 1];
        cp[t] = (gather16(P->wo, ch, t) & ~set0) ^ inv;
        cpx[t] = is_x ? (gather16(P->wo_x, ch, t) & ~set0) : 0;
      }
      for (uint32_t t = 0; t < num_ios; ++t) {
        uint32_t dinv = ch[4096 + 4 * t + 2];
        uint32_t wv = P->wo[t] ^ dinv;
        size_t o = (size_t)io_off + t;
        if (o >= state_words) return E_STATE_OOB;
        uint32_t old = in_state[o];
        out_state[o] = (old & ~cp[t]) | (wv & cp[t]);
        if (is_x) {
          size_t ox = (size_t)xoff + o;
          if (ox >= state_words) return E_STATE_OOB;
          uint32_t wx, dummy;
          jqo_dff_commit(old, in_state[ox], wv, P->wo_x[t], cp[t], cpx[t],
                         &dummy, &wx);
          out_state[ox] = wx;
        }
        if (arr_off != 0) {
          size_t oa = (size_t)(uint32_t)arr_off + o;
          if (oa >= state_words) return E_STATE_OOB;
          out_state[oa] = (uint32_t)P->wo_arr[t];
        }
        /* setup / hold check per writeout word (cuh:536-558) */
        if (cp[t] != 0 && constraints != NULL) {
          uint32_t c = constraints[o];
          if (c != 0) {
            uint16_t setup = (uint16_t)(c >> 16), hold = (uint16_t)(c & 0xffffu);
            uint16_t a = P->wo_arr[t];
            int32_t slack;
            if (jqo_setup_violation(a, setup, clock_ps, &slack))
              push_event(sink, 4, (uint32_t)o, cycle, (uint32_t)o,
                         (uint32_t)slack, a, setup);
            if (jqo_hold_violation(a, hold, &slack))
              push_event(sink, 5, (uint32_t)o, cycle, (uint32_t)o,
                         (uint32_t)slack, a, hold);
          }
        }
      }
    }
    if (is_last) break;
  }
  if (pi != script_size) return E_SIZE_MISMATCH; /* cuh:562 */
  return (long)pi;
}

long jqo_simulate_block(const uint32_t *script, size_t script_size,
                        const uint32_t *input_state, uint32_t *output_state,
                        uint32_t *sram_data, uint32_t *sram_xmask,
                        uint32_t flags) {
  blk_persist P;
  memset(&P, 0, sizeof(P));
  uint64_t cnt = 0;
  event_sink sink = {NULL, 0, &cnt};
  return run_block(script, script_size, input_state, output_state, (size_t)-1,
                   sram_data, sram_xmask, (size_t)-1, &P, NULL, 0, &sink, 0, 0,
                   (flags & JQO_FLAG_FORCE_ARRIVALS) != 0, flags);
}

/* Work shared by the host threads of jqo_simulate: every thread walks the
 * same (cycle, major stage) sequence and takes blocks from an atomic counter;
 * a barrier separates major stages, as grid.sync() does in the kernel. */
typedef struct {
  size_t num_blocks, num_major_stages, num_cycles, state_size;
  const size_t *blocks_start;
  const uint32_t *blocks_data;
  uint32_t *sram, *sram_x, *states;
  const uint32_t *cons;
  uint32_t clock_ps;
  event_sink *sink;
  int32_t arr_off;
  int track;
  uint32_t flags;
  blk_persist *P;
  pthread_barrier_t bar;
  size_t next; /* block ticket */
  int err;
  int nthreads;
  int nthreads_started;
} sim_job;

static void *sim_worker(void *arg) {
  sim_job *J = (sim_job *)arg;
  int lead = 0;
  if (__atomic_fetch_add(&J->nthreads_started, 1, __ATOMIC_RELAXED) == 0)
    lead = 1;
  for (size_t c = 0; c < J->num_cycles; ++c) {
    const uint32_t *in = J->states + c * J->state_size;
    uint32_t *out = J->states + (c + 1) * J->state_size;
    for (size_t s = 0; s < J->num_major_stages; ++s) {
      for (;;) {
        size_t b = __atomic_fetch_add(&J->next, 1, __ATOMIC_RELAXED);
        if (b >= J->num_blocks) break;
        if (__atomic_load_n(&J->err, __ATOMIC_RELAXED)) continue;
        size_t st = J->blocks_start[s * J->num_blocks + b];
        size_t ed = J->blocks_start[s * J->num_blocks + b + 1];
        long r = run_block(J->blocks_data + st, ed - st, in, out, J->state_size,
                           J->sram, J->sram_x, (size_t)-1, &J->P[b], J->cons,
                           J->clock_ps, J->sink, (uint32_t)c, J->arr_off,
                           J->track, J->flags);
        if (r < 0) {
          int zero = 0;
          __atomic_compare_exchange_n(&J->err, &zero, (int)r, 0,
                                      __ATOMIC_RELAXED, __ATOMIC_RELAXED);
        }
      }
      /* stage boundary: everyone finished, one thread re-arms the tickets */
      if (J->nthreads > 1) pthread_barrier_wait(&J->bar);
      if (lead) __atomic_store_n(&J->next, 0, __ATOMIC_RELAXED);
      if (J->nthreads > 1) pthread_barrier_wait(&J->bar);
    }
  }
  return NULL;
}

int jqo_simulate(size_t num_blocks, size_t num_major_stages,
                 const size_t *blocks_start, const uint32_t *blocks_data,
                 uint32_t *sram_data, uint32_t *sram_xmask, size_t num_cycles,
                 size_t state_size, uint32_t *states,
                 const uint32_t *timing_constraints, jqo_event *events,
                 size_t event_cap, uint64_t *event_count,
                 int32_t arrival_state_offset, uint32_t flags,
                 int num_threads) {
  if (num_major_stages > 32) return E_TOO_MANY_STAGES; /* cuh:593 */
  uint64_t local_cnt = 0;
  event_sink sink = {events, event_cap, event_count ? event_count : &local_cnt};
  sim_job J;
  memset(&J, 0, sizeof(J));
  J.num_blocks = num_blocks;
  J.num_major_stages = num_major_stages;
  J.num_cycles = num_cycles;
  J.state_size = state_size;
  J.blocks_start = blocks_start;
  J.blocks_data = blocks_data;
  J.sram = sram_data;
  J.sram_x = sram_xmask;
  J.states = states;
  J.clock_ps = timing_constraints ? timing_constraints[0] : 0;
  J.cons = timing_constraints ? timing_constraints + 1 : NULL;
  J.sink = &sink;
  J.arr_off = arrival_state_offset;
  J.track = arrival_state_offset != 0 || timing_constraints != NULL ||
            (flags & JQO_FLAG_FORCE_ARRIVALS);
  J.flags = flags;
  J.P = (blk_persist *)calloc(num_blocks ? num_blocks : 1, sizeof(blk_persist));
  if (!J.P) return -100;
  if (num_threads < 1) num_threads = 1;
  if ((size_t)num_threads > num_blocks && num_blocks > 0)
    num_threads = (int)num_blocks;
  J.nthreads = num_threads;
  if (num_threads == 1) {
    sim_worker(&J);
  } else {
    pthread_t *th = (pthread_t *)calloc((size_t)num_threads, sizeof(pthread_t));
    pthread_barrier_init(&J.bar, NULL, (unsigned)num_threads);
    for (int i = 1; i < num_threads; ++i)
      pthread_create(&th[i], NULL, sim_worker, &J);
    sim_worker(&J);
    for (int i = 1; i < num_threads; ++i) pthread_join(th[i], NULL);
    pthread_barrier_destroy(&J.bar);
    free(th);
  }
  free(J.P);
  return J.err;
}

/* ---------------------------------------------------------------- netlist */
#define REC_WORDS (13 + 1 + 32 + 13 + 32 + 32)

int jqo_aig_simulate(uint32_t num_pins, const uint8_t *kind, const uint32_t *fa,
                     const uint32_t *fb, size_t n_dff, const uint32_t *dff_d,
                     const uint32_t *dff_en, const uint32_t *dff_q, size_t n_sram,
                     const uint32_t *sram_rec, size_t n_in, const uint32_t *in_pins,
                     size_t num_cycles, const uint8_t *in_vals, uint8_t *dff_state,
                     size_t n_po, const uint32_t *po_iv, uint8_t *po_vals,
                     uint32_t *sram_words, uint8_t *sram_rd) {
  uint8_t *v = (uint8_t *)calloc((size_t)num_pins + 1, 1);
  if (!v) return -100;
#define VAL(iv) ((uint8_t)(v[(iv) >> 1] ^ ((iv)&1u)))
  for (size_t c = 0; c < num_cycles; ++c) {
    const uint8_t *inr = in_vals + c * n_in;
    for (size_t i = 0; i < n_in; ++i) v[in_pins[i]] = inr[i] & 1;
    for (size_t i = 0; i < n_dff; ++i) v[dff_q[i]] = dff_state[c * n_dff + i] & 1;
    for (size_t s = 0; s < n_sram; ++s) {
      const uint32_t *rd = sram_rec + s * REC_WORDS + 14;
      for (int k = 0; k < 32; ++k)
        if (rd[k] && rd[k] != 0xffffffffu) v[rd[k]] = sram_rd[(c * n_sram + s) * 32 + k] & 1;
    }
    v[0] = 0;
    for (uint32_t p = 1; p <= num_pins; ++p)
      if (kind[p] == 1) v[p] = VAL(fa[p]) & VAL(fb[p]);
    for (size_t i = 0; i < n_dff; ++i) {
      uint8_t en = VAL(dff_en[i]);
      dff_state[(c + 1) * n_dff + i] = en ? VAL(dff_d[i]) : (dff_state[c * n_dff + i] & 1);
    }
    for (size_t i = 0; i < n_po; ++i) po_vals[(c + 1) * n_po + i] = VAL(po_iv[i]);
    for (size_t s = 0; s < n_sram; ++s) {
      const uint32_t *R = sram_rec + s * REC_WORDS;
      const uint32_t *raddr = R, *ren = R + 13, *waddr = R + 46, *wen = R + 59,
                     *wdat = R + 91;
      uint32_t ra = 0, wa = 0, en = 0, dat = 0;
      for (int k = 0; k < 13; ++k) {
        ra |= (uint32_t)VAL(raddr[k]) << k;
        wa |= (uint32_t)VAL(waddr[k]) << k;
      }
      for (int k = 0; k < 32; ++k) {
        en |= (uint32_t)VAL(wen[k]) << k;
        dat |= (uint32_t)VAL(wdat[k]) << k;
      }
      uint32_t *ram = sram_words + s * 8192;
      uint32_t r = ram[ra];
      uint8_t *rdn = sram_rd + ((c + 1) * n_sram + s) * 32;
      uint8_t *rdo = sram_rd + (c * n_sram + s) * 32;
      uint8_t ren_v = VAL(ren[0]);
      for (int k = 0; k < 32; ++k) rdn[k] = ren_v ? (uint8_t)((r >> k) & 1) : rdo[k];
      ram[wa] = (ram[wa] & ~en) | (dat & en);
    }
  }
#undef VAL
  free(v);
  return 0;
}
