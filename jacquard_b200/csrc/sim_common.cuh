// Shared device helpers of the interpreter kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/jacquard_b200.h"

namespace jqk {

constexpr int NT = 256;             // threads per block (src/flatten.rs:24)
constexpr uint32_t STAGE_WORDS = 5120;
constexpr uint32_t SRAM_WORDS = 8192;  // AIGPDK_SRAM_SIZE
constexpr int BAR_SLOTS = 64;
constexpr uint64_t DEFAULT_BARRIER_TIMEOUT = 2000000000ull;  // ~1 s at 2 GHz

// Grid barrier state lives in module memory (no allocation on the call path);
// each translation unit that includes this header has its own copy.  One slot
// per stream a launch is issued on (launch_slot); launches on one slot run in
// stream order and never overlap.  g_bar_count returns to 0 after every
// completed barrier.
static __device__ unsigned int g_bar_count[BAR_SLOTS];
static __device__ unsigned int g_bar_gen[BAR_SLOTS];
static __device__ int g_status[BAR_SLOTS];

// Slot of the (current device, stream) pair (launch_slots.cu): assigns a free
// one when `assign` and the pair has none yet; -1 when the table is full or,
// without `assign`, when nothing was launched on the pair.
int launch_slot(void *stream, bool assign);

__device__ __forceinline__ uint4 ldg4(const uint32_t *p) {
  return __ldg(reinterpret_cast<const uint4 *>(p));
}
__device__ __forceinline__ uint2 ldg2(const uint32_t *p) {
  return __ldg(reinterpret_cast<const uint2 *>(p));
}
// State and SRAM reads bypass L1: other SMs write them between barriers.
__device__ __forceinline__ uint32_t ldcg(const uint32_t *p) { return __ldcg(p); }

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Sense-free generation barrier with a bounded wait.  Returns false (and
// records JQ_ERR_BARRIER_TIMEOUT) when the wait runs out; every thread of the
// block gets the same answer.
__device__ __forceinline__ bool grid_barrier(int slot, unsigned nblocks,
                                             uint64_t timeout_cycles) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    unsigned gen = ld_acquire(&g_bar_gen[slot]);
    __threadfence();
    unsigned arrived = atomicAdd(&g_bar_count[slot], 1u);
    if (arrived == nblocks - 1) {
      g_bar_count[slot] = 0;
      __threadfence();
      atomicAdd(&g_bar_gen[slot], 1u);
    } else {
      uint64_t t0 = clock64();
      while (ld_acquire(&g_bar_gen[slot]) == gen) {
        __nanosleep(64);
        if ((uint64_t)(clock64() - t0) > timeout_cycles) {
          ok = 0;
          atomicExch(&g_status[slot], JQ_ERR_BARRIER_TIMEOUT);
          break;
        }
      }
    }
    // a peer that timed out makes everyone stop at the next barrier
    if (ok && *((volatile int *)&g_status[slot]) != 0) ok = 0;
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// The 16-pair bit shuffle (kernel ABI: four uint4 words per thread, each u32
// packs two 13-bit source indices; bit 2k / 2k+1 of the result).
__device__ __forceinline__ uint32_t gather16(const uint32_t *src, uint4 a, uint4 b,
                                             uint4 c, uint4 d) {
  uint32_t r = 0;
#define JQ_G(w, k)                                                        \
  {                                                                       \
    uint32_t i1 = (w)&0xffffu, i2 = (w) >> 16;                            \
    r |= ((src[(i1 >> 5) & 255] >> (i1 & 31)) & 1u) << (2 * (k));         \
    r |= ((src[(i2 >> 5) & 255] >> (i2 & 31)) & 1u) << (2 * (k) + 1);     \
  }
  JQ_G(a.x, 0) JQ_G(a.y, 1) JQ_G(a.z, 2) JQ_G(a.w, 3)
  JQ_G(b.x, 4) JQ_G(b.y, 5) JQ_G(b.z, 6) JQ_G(b.w, 7)
  JQ_G(c.x, 8) JQ_G(c.y, 9) JQ_G(c.z, 10) JQ_G(c.w, 11)
  JQ_G(d.x, 12) JQ_G(d.y, 13) JQ_G(d.z, 14) JQ_G(d.w, 15)
#undef JQ_G
  return r;
}

__device__ __forceinline__ void xand(uint32_t a, uint32_t ax, uint32_t b, uint32_t bx,
                                     uint32_t xa, uint32_t xb, uint32_t ob, uint32_t &r,
                                     uint32_t &rx) {
  uint32_t ae = a ^ xa, be = (b ^ xb) | ob, bex = bx & ~ob;
  r = ae & be;
  rx = (ax | bex) & (ae | ax) & (be | bex);
}

__device__ __forceinline__ uint16_t arr_step(bool pass, uint16_t a, uint16_t b, uint16_t d) {
  uint16_t base = pass ? a : (a > b ? a : b);
  return (uint16_t)(base + d);
}

// Append rule of the reference's write_event (csrc/event_buffer.h:89-111):
// the counter always advances; records past `cap` are dropped and flagged.
__device__ __forceinline__ void push_event(jq_event_buffer *eb, uint32_t cap, uint32_t type,
                                           uint32_t word, uint32_t cycle, uint32_t slack,
                                           uint32_t arr, uint32_t c) {
  uint32_t idx = atomicAdd(&eb->count, 1u);
  if (idx < cap) {
    jq_event *e = &eb->events[idx];
    e->event_type = type;
    e->message_id = word;
    e->cycle = cycle;
    e->data[0] = word;
    e->data[1] = slack;
    e->data[2] = arr;
    e->data[3] = c;
  } else {
    atomicExch(&eb->overflow, 1u);
  }
}

}  // namespace jqk
