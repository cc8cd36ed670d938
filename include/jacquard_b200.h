/*
 * jacquard_b200.h -- C ABI of the B200 (sm_100a) Boolean-processor
 * interpreter (libjacquard_b200.so).
 *
 * Drop-in boundary: the first two symbols have exactly the names, argument
 * order and meaning of the reference's kernel wrappers in csrc/kernel_v1.cu,
 * which the reference's Rust side binds through bindgen (build.rs:69) and
 * calls from sim_cuda (src/bin/jacquard.rs:1135-1147):
 *   simulate_v1_noninteractive_simple_scan_cuda  <- csrc/kernel_v1.cu:17-46
 *   simulate_v1_noninteractive_timed_cuda        <- csrc/kernel_v1.cu:49-78
 * All pointers are caller-owned DEVICE pointers; the launch runs on the
 * legacy default stream.  Like the reference, a launch failure prints the
 * CUDA error and exits the process (csrc/kernel_v1.cu:6-14).  Unlike the
 * reference's grid.sync(), this interpreter's grid barrier has a bounded
 * wait; a launch that ran out of it has left the snapshots half-written, so
 * the wrappers wait for the launch, and print and exit on that error too.
 * They therefore return with the work done (the reference returns right
 * after the launch; its caller synchronizes next, src/bin/jacquard.rs:1131,
 * 1149).
 *
 * The jq_* entry points below have no counterpart symbol in the reference:
 * they return a status instead of exiting, take an explicit stream, report
 * barrier timeouts and event-buffer overflow, and add the bit-lane batched
 * interpreter (many stimulus streams per launch).
 */
#ifndef JACQUARD_B200_H
#define JACQUARD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------ */
/* Reference-compatible entry points (types: usize = size_t, u32, i32, u8). */

/* Runs num_cycles cycles of the script.  states_noninteractive holds
 * (num_cycles+1) snapshots of state_size u32: snapshot 0 is the initial
 * state, snapshot c+1 is pre-filled by the caller with edge c+1's inputs and
 * receives the partitions' outputs.  blocks_start has
 * num_major_stages*num_blocks+1 entries.  sram_xmask must be a valid device
 * pointer even when no partition is X-capable.  arrival_state_offset != 0
 * writes per-word arrival times at that offset of each output snapshot. */
void simulate_v1_noninteractive_simple_scan_cuda(
    size_t num_blocks, size_t num_major_stages, const size_t *blocks_start,
    const uint32_t *blocks_data, uint32_t *sram_data, uint32_t *sram_xmask,
    size_t num_cycles, size_t state_size, uint32_t *states_noninteractive,
    int32_t arrival_state_offset);

/* Same, with setup/hold checking.  timing_constraints = [clock_period_ps,
 * one u32 per state word: setup<<16 | hold]; event_buffer points to the
 * reference's EventBuffer (csrc/event_buffer.h:45-50: u32 count, u32
 * overflow, u32 reserved[2], then 1024 events of 8 u32). */
void simulate_v1_noninteractive_timed_cuda(
    size_t num_blocks, size_t num_major_stages, const size_t *blocks_start,
    const uint32_t *blocks_data, uint32_t *sram_data, uint32_t *sram_xmask,
    size_t num_cycles, size_t state_size, uint32_t *states_noninteractive,
    const uint32_t *timing_constraints, uint8_t *event_buffer,
    int32_t arrival_state_offset);

/* ------------------------------------------------------------------------ */
/* Status-returning interface. */

#define JQ_OK 0
#define JQ_ERR_INVALID_ARG -1
#define JQ_ERR_LAUNCH -2          /* CUDA launch / occupancy failure */
#define JQ_ERR_BARRIER_TIMEOUT -3 /* a grid barrier wait ran out */
#define JQ_ERR_CUDA -4            /* asynchronous CUDA error */
#define JQ_ERR_TOO_MANY_BLOCKS -5 /* grid larger than co-resident capacity */
#define JQ_ERR_NOALLOC_LIMIT -6   /* request exceeds a fixed built-in workspace */
#define JQ_ERR_TOO_MANY_STREAMS -7 /* launches on more streams than barrier slots */
#define JQ_ERR_EVENT_OVERFLOW 1   /* positive: events were dropped */

/* Event record: identical to the reference's Event (32 bytes). */
typedef struct {
  uint32_t event_type, message_id, cycle, reserved;
  uint32_t data[4];
} jq_event;

/* Event sink with a caller-chosen capacity (the reference's fixed 1024-slot
 * EventBuffer is the legacy layout).  `count` counts every event, also those
 * dropped past `capacity`. */
typedef struct {
  uint32_t count, overflow, capacity, reserved;
  jq_event events[];  /* capacity entries follow */
} jq_event_buffer;

typedef struct {
  size_t num_blocks, num_major_stages;
  const size_t *blocks_start; /* device */
  const uint32_t *blocks_data; /* device */
  uint32_t *sram_data, *sram_xmask; /* device; sram_xmask may be NULL */
  size_t num_cycles, state_size;
  uint32_t *states; /* device, (num_cycles+1) x state_size */
  const uint32_t *timing_constraints; /* device or NULL */
  jq_event_buffer *events; /* device or NULL (required with constraints) */
  uint32_t event_capacity; /* records that fit in `events` */
  int32_t arrival_state_offset;
  uint32_t first_cycle; /* cycle number reported in events */
  uint64_t barrier_timeout_cycles; /* 0 = default (about a second) */
  void *stream; /* cudaStream_t, NULL = legacy default stream */
  /* Optional stage-depth tables from jq_plain_prepare (both or neither,
   * device): levels of a boomerang stage whose outputs nothing reads are
   * skipped.  NULL runs every level. */
  const uint8_t *stage_depth;
  const uint32_t *stage_depth_base;
} jq_sim_args;

/* Barrier slots.  Each interpreter (plain, batched) keeps its grid-barrier
 * counters and its error status in module memory, 64 slots per device.  A
 * launch takes the slot of the (device, stream) it is issued on: launches on
 * one stream share it and run in stream order, launches on different streams
 * get different slots, so they may overlap on the GPU.  Slots are never
 * released; the 65th distinct stream of a process gets
 * JQ_ERR_TOO_MANY_STREAMS.  NULL and cudaStreamLegacy are one stream;
 * cudaStreamPerThread is one handle for all host threads, so launches on it
 * from several threads must not overlap.  A launch captured in a CUDA graph
 * keeps the slot of the stream it was captured on. */

/* Plain interpreter (reference layout, one stimulus stream).  Asynchronous;
 * returns JQ_OK or a launch error.  Kernel-side status (barrier timeout) is
 * read back with jq_sim_status on the same stream. */
int jq_simulate(const jq_sim_args *a);

/* Synchronizes `stream` and returns JQ_OK, JQ_ERR_BARRIER_TIMEOUT or
 * JQ_ERR_CUDA for the plain launches made so far on it, and clears the
 * recorded error. */
int jq_sim_status(void *stream);

/* Stage depth of a script for the plain interpreter (no counterpart in the
 * reference): for every boomerang stage, the deepest tree level whose
 * outputs a writeout hook or a needed gather of the next stage reads
 * (0: only the first AND level, positions 4096..8191; 1: nothing below
 * position 512; 2: any).  stage_depth_base (device, num_blocks *
 * num_major_stages words) receives each (major stage, block) entry's first
 * code; stage_depth (device, depth_capacity bytes) the codes, partitions in
 * script order.  With stage_depth NULL only *num_stages (the size needed) is
 * computed.  JQ_ERR_INVALID_ARG when depth_capacity is too small.
 * Synchronizes `stream`.  The legacy wrappers compute these tables on every
 * call into a device buffer the library keeps per device (allocated on the
 * first call, grown for larger scripts). */
int jq_plain_prepare(const size_t *blocks_start, const uint32_t *blocks_data, size_t num_blocks,
                     size_t num_major_stages, uint32_t *stage_depth_base, uint8_t *stage_depth,
                     size_t depth_capacity, size_t *num_stages, void *stream);

/* Largest grid the plain interpreter can keep co-resident on `device`. */
int jq_max_blocks(int device, size_t *max_blocks);

/* ------------------------------------------------------------------------ */
/* Bit-lane batched interpreter: 32*lanes independent stimulus streams run the
 * same script in one persistent launch.  A lane word holds one signal (a bit
 * position of the reference layout, word*32+bit, X plane at metadata word
 * 9 * 32) for streams 32l..32l+31.  The state buffers interleave lane groups
 * (jq_batched_state_words words; lanes rounded up to even):
 *   x_interleaved = 1, lane-pair quads (V = signals_per_snapshot / 2 value
 *     signals, signal V + s the X of s): word ((l >> 1) * V + s mod V) * 4 +
 *     2 * (l & 1) + (s >= V), i.e. (value, X) of the even lane, then of the
 *     odd lane;
 *   x_interleaved = 2, lane octets (lanes a multiple of 8): word
 *     ((l >> 3) * V + s mod V) * 16 + 2 * (l & 7) + (s >= V), i.e. the 64
 *     bytes (value, X) of 8 lane words for one signal are adjacent; it runs
 *     octet work items (lanes_per_item 8) only;
 *   x_interleaved = 0: word ((l >> 1) * signals + s) * 2 + (l & 1).
 * jq_batched_pack_state / jq_batched_unpack_state convert from / to the
 * lane-major form [l][signal] that `stimulus`, `wave` and `record` use.
 * Two snapshot buffers ping-pong: cycle c reads state_a when c
 * is even (state_b when odd) and writes the other; after num_cycles cycles the
 * final state is in state_a if num_cycles is even, else state_b.  Both buffers
 * must start with snapshot 0 (values, X template).  Words that no partition
 * writes (inputs aside, which come from `stimulus`) keep their snapshot-0
 * value in every cycle, where the plain interpreter keeps each snapshot's
 * host pre-fill; the two agree when every snapshot carries the same pre-fill
 * (the X template).  Arrivals are not written into the state (they are the
 * same for every stream: see arrival_first / arrival_steady). */
typedef struct {
  size_t num_blocks, num_major_stages;
  const size_t *blocks_start;  /* device */
  const uint32_t *blocks_data; /* device, 16-byte aligned, prepared by
                                  jq_batched_prepare */
  uint32_t lanes;              /* lane words (32 streams each) */
  uint32_t *sram_data, *sram_xmask; /* device: [stream][sram_words_per_stream] */
  size_t sram_words_per_stream;
  size_t num_cycles;
  size_t signals_per_snapshot; /* effective state words * 32 */
  uint32_t *state_a, *state_b;
  const uint32_t *stimulus;    /* [num_cycles+1][lanes][input_signals] or NULL */
  size_t input_signals;        /* stimulus signals per lane and cycle */
  const uint32_t *input_regions; /* device: (state signal, stimulus signal, count)
                                    triples, or NULL for one region at 0 (used
                                    when several designs share one state) */
  uint32_t n_input_regions;
  const uint32_t *po_signals;  /* signals recorded each cycle */
  uint32_t n_po;
  uint32_t *wave;              /* [num_cycles][n_po][lanes] */
  uint32_t *record;            /* optional [num_cycles+1][lanes][signals] */
  uint32_t wo_slots;           /* >= the script's largest num_ios (<= 256) */
  const uint32_t *block_list;  /* device: blocks with work, per major stage
                                  (any order; heaviest first is best), or NULL
                                  for all blocks */
  const uint32_t *block_list_start; /* device: num_major_stages+1 offsets */
  unsigned long long *part_cycles; /* optional device output: SM clocks spent
                                      per partition, summed over work items
                                      (a lane-pair item counts once) and
                                      cycles (partition order of the script:
                                      major stage, block, position in block);
                                      the grid-barrier wait an item takes
                                      over from the previous stage is not
                                      counted */
  const uint32_t *part_base;   /* device: index of the first partition of each
                                  (major stage, block), from jq_batched_prepare */
  const uint32_t *gr_sources;  /* device: global-read sources, from
                                  jq_batched_prepare */
  size_t grid;                 /* CTAs; 0 = all that fit */
  uint64_t barrier_timeout_cycles;
  void *stream;
  uint32_t lanes_per_item;     /* lane words one work item runs: 0 = automatic
                                  (8 in the octet layout; otherwise 2 when
                                  lanes is even and the shared memory of a
                                  lane pair fits the writeouts, else 1), 1, 2,
                                  or 8 (JQ_ERR_INVALID_ARG when it does not
                                  fit, lanes does not divide, or the layout
                                  differs).  Octet items need every partition
                                  in the compact form the prepare step writes
                                  and within jq_batched_oct_capacity slots
                                  (jq_batched_slot_need); a partition that is
                                  not gives JQ_ERR_INVALID_ARG in the status */
  int32_t x_interleaved;       /* state layout (above): 1 (lane-pair quads) or
                                  2 (lane octets) when signals [S/2, S) are
                                  the X planes of [0, S/2) (S =
                                  signals_per_snapshot; required when any
                                  partition is X-capable, and then every such
                                  partition's X offset, metadata word 9, is
                                  S/64 words), 0 for scripts without X */
  /* Setup/hold checks (timing_constraints NULL: none).  The predicate is the
   * plain interpreter's (and the reference kernel's,
   * csrc/kernel_v1_impl.cuh:536-558), applied per stream: a word's arrival
   * does not depend on the stream, only the clock-enable gate does.  The
   * arrivals come from two tables of one u32 per state word (low 16 bits):
   * arrival_first for the first cycle of a launch, arrival_steady for the
   * others.  They are the arrival sections of snapshots 1 and 2 of a
   * two-cycle jq_simulate run of the same script with an arrival section
   * (any stimulus): the plain interpreter's per-block writeout arrivals
   * start at zero in each launch and repeat from the second cycle on.
   * Events are the reference's records with `reserved` = the stream
   * (32 * lane + bit), `cycle` = first_cycle + the cycle in the launch. */
  const uint32_t *timing_constraints; /* device [clock_ps, state words...] */
  const uint32_t *arrival_first, *arrival_steady; /* device, state words each */
  jq_event_buffer *events;     /* device; count/overflow as for jq_simulate */
  uint32_t event_capacity;
  uint32_t first_cycle;
} jq_batch_args;

/* Prepares a script (FlattenedScriptV1, device arrays) for the batched
 * interpreter; run once per script, synchronizes `stream`.  Outputs (device):
 *   out         blocks_data_len words, 16-byte aligned: the script in the
 *               batched layout (same size and partition offsets, boomerang
 *               chunks reordered per thread);
 *   part_base   num_blocks * num_major_stages words: index of the first
 *               partition of each (major stage, block), partitions numbered
 *               in script order;
 *   gr_sources  jq_batched_gr_words(num_partitions) words: the source signal
 *               of each global-read position of each partition.
 * JQ_ERR_INVALID_ARG when the script holds other than num_partitions
 * partitions. */
size_t jq_batched_gr_words(size_t num_partitions);
int jq_batched_prepare(const size_t *blocks_start, const uint32_t *blocks_data,
                       size_t blocks_data_len, size_t num_blocks, size_t num_major_stages,
                       size_t num_partitions, uint32_t *out, uint32_t *part_base,
                       uint32_t *gr_sources, void *stream);
int jq_simulate_batched(const jq_batch_args *a);
/* Words of one batched state buffer. */
size_t jq_batched_state_words(uint32_t lanes, size_t signals);
/* Lane-major [lanes][signals] (device) <-> batched state layout (device),
 * asynchronous on `stream`. */
int jq_batched_pack_state(const uint32_t *lane_major, uint32_t lanes, size_t signals,
                          int32_t x_interleaved, uint32_t *state, void *stream);
int jq_batched_unpack_state(const uint32_t *state, uint32_t lanes, size_t signals,
                            int32_t x_interleaved, uint32_t *lane_major, void *stream);
/* Synchronizes `stream`; JQ_OK or the recorded error of the batched launches
 * made on it (cleared by the read).  Barrier slots as for jq_simulate. */
int jq_batched_status(void *stream);
int jq_batched_max_blocks(int device, uint32_t wo_slots, size_t *max_blocks);
int jq_batched_smem_bytes(uint32_t wo_slots);
/* Octet work items (no counterpart in the reference): the 64-byte tree slots
 * one item holds in shared memory on the current device, and, into the
 * device word *need (asynchronous on `stream`), the most slots any partition
 * of a prepared script needs (0xffffffff when some partition cannot run as an
 * octet item).  Octet items run a script when need <= capacity. */
int jq_batched_oct_capacity(uint32_t *slots);
int jq_batched_slot_need(const size_t *blocks_start, const uint32_t *prepared, size_t num_blocks,
                         size_t num_major_stages, uint32_t *need, void *stream);

/* ------------------------------------------------------------------------ */
/* Partition cost model (no counterpart in the reference): an MLP
 * JQ_MLP_FEATURES -> 128 -> 128 -> 1 (ReLU) predicting log kernel time of a
 * partition from its features.  BF16 weights/activations, FP32 accumulation.
 * theta is the fp32 master parameter vector (JQ_MLP_PARAMS floats:
 * W1[128][24] b1[128] W2[128][128] b2[128] W3[128] b3), theta16 its bf16 copy
 * (uint16 storage).  X holds normalised features as bf16 [n][24]. */
#define JQ_MLP_FEATURES 24
#define JQ_MLP_HIDDEN 128
#define JQ_MLP_PARAMS (128 * 24 + 128 + 128 * 128 + 128 + 128 + 1)

/* theta16 <- bf16(theta). */
int jq_mlp_sync_bf16(const float *theta, uint16_t *theta16, void *stream);
/* y[i] = model(X[i]) for n rows. */
int jq_mlp_forward(const float *theta, const uint16_t *theta16, const uint16_t *X, size_t n,
                   float *y, void *stream);

typedef struct {
  float *theta;          /* device fp32 master parameters (updated when apply) */
  uint16_t *theta16;     /* device bf16 copy (updated when apply) */
  float *adam_m, *adam_v; /* device Adam moments (JQ_MLP_PARAMS each) */
  const uint16_t *X;     /* device bf16 features [rows][24] */
  const float *T;        /* device targets [rows] */
  const uint32_t *batch_index; /* device row indices of this mini-batch */
  uint32_t batch;
  uint32_t step;         /* Adam step, 1-based */
  float lr;
  int32_t apply;         /* 0: gradient only (grad_out), 1: Adam update */
  float *grad_out;       /* optional device [JQ_MLP_PARAMS] summed gradient */
  float *loss_out;       /* optional device scalar: mean squared error */
  float *scratch;        /* device workspace, jq_mlp_scratch_floats(scratch_ctas) */
  uint32_t scratch_ctas; /* CTAs that split the batch (one gradient row each) */
  void *stream;
} jq_mlp_step_args;

/* Floats of workspace jq_mlp_train_step needs for `ctas` CTAs. */
size_t jq_mlp_scratch_floats(uint32_t ctas);
/* One mini-batch: forward, backward of the mean squared error, gradient
 * reduction and (apply=1) an Adam step (beta1 0.9, beta2 0.999, eps 1e-8). */
int jq_mlp_train_step(const jq_mlp_step_args *a);

/* No counterpart in the reference.  Same as jq_mlp_train_step but allocates
 * nothing and ignores a->scratch: the per-CTA gradient workspace is a
 * file-scope device array of JQ_MLP_NOALLOC_MAX_CTAS rows (about 1.3 MB, held
 * on every GPU that loads the library until exit).  For hosts that cannot
 * allocate device memory once running: an embedding host with one device
 * pool sized at start-up, or one whose latency limits rule out an allocation
 * that may synchronize the device.  a->scratch_ctas must be
 * 1..JQ_MLP_NOALLOC_MAX_CTAS, otherwise JQ_ERR_NOALLOC_LIMIT; a NULL `a` is
 * JQ_ERR_INVALID_ARG.  Every call resolves the array's address for the
 * current device and context (cudaGetSymbolAddress, which allocates
 * nothing); the first call on a device may also load the library's module
 * there, so make it before any stream capture.  All calls on a device share
 * the array: calls that overlap on the GPU race.  Nothing in it needs
 * clearing; each call writes every entry it reads. */
#define JQ_MLP_NOALLOC_MAX_CTAS 16
int jq_mlp_train_step_noalloc(const jq_mlp_step_args *a);

/* ------------------------------------------------------------------------ */
/* Output transitions for waveform writers (no counterpart in the reference,
 * whose writer walks every output of every snapshot on the host,
 * src/sim/vcd_io.rs:758-946).  Walks snapshots first_snapshot ..
 * first_snapshot+num_snapshots-1 of `states` (device, snapshot_words words
 * each).  Each output j has a code: 3 when its X bit is set (X word
 * xmask_offset words after its value word, when xmask_offset != 0), else its
 * value bit.  Constant outputs, with out_pos[j] = 0xFFFFFFFF, take
 * out_const[j] (0 when out_const is NULL).  A transition is a code that
 * differs from the previous snapshot's (2 = unknown before the first).
 *
 * Outputs (device):
 *   counts[s]    transitions of walk step s;
 *   offsets[s]   their start, with offsets[num_snapshots] = total;
 *   transitions  j | code << 30, in (snapshot, output) order, capacity entries;
 *   arrivals     (optional) the low 16 bits of each transition's arrival
 *                word, arrival_offset words after the value word.
 * *total gets the number of transitions.  Returns JQ_ERR_EVENT_OVERFLOW when
 * it exceeds capacity (capacity 0 only counts).  Synchronizes `stream`. */
int jq_output_transitions(const uint32_t *states, size_t first_snapshot, size_t num_snapshots,
                          size_t snapshot_words, size_t xmask_offset, size_t arrival_offset,
                          const uint32_t *out_pos, const uint32_t *out_const, uint32_t n_out,
                          uint32_t *counts, unsigned long long *offsets, uint32_t *transitions,
                          uint32_t *arrivals, size_t capacity, size_t *total, void *stream);

/* Set bits for the display / assertion post-scan (no counterpart in the
 * reference, whose post-scan probes every condition of every snapshot on the
 * host, src/bin/jacquard.rs:1152-1253).  Same walk and outputs as
 * jq_output_transitions.  Each entry j | 1 << 30 is a condition bit
 * bit_pos[j] that is 1 in that snapshot. */
int jq_set_bits(const uint32_t *states, size_t first_snapshot, size_t num_snapshots,
                size_t snapshot_words, const uint32_t *bit_pos, uint32_t n_bits, uint32_t *counts,
                unsigned long long *offsets, uint32_t *hits, size_t capacity, size_t *total,
                void *stream);

/* ------------------------------------------------------------------------ */
/* RepCut hypergraph build (src/repcut.rs:58-176) on the device, from the
 * arrays of jqf_repcut_slice and the design arrays (kind, fa, fb).  All
 * pointers are device memory except the two level-start arrays, which the
 * host walks to launch one pass per level:
 *   rlevel_nodes: pins 1..num_pins ordered by reverse level,
 *     rlevel_start_host[num_rlevels+1];
 *   flevel_nodes: likewise by forward level;
 *   nfe[pin]: number of endpoint-input occurrences of the pin;
 *   supp_start_host / supp_edges / wsupp: the traversal-order exceptions of
 *     jqf_repcut_slice;
 *   sets, cone, supp_bits: workspace of (num_pins+1) * 64 u64,
 *     (num_pins+1) bytes and num_fanouts / 32 + 2 words.
 * Outputs per pin: fingerprint[2*(num_pins+1)] (equal endpoint sets give
 * equal fingerprints), popcount (endpoints reached), node_weight (f32, 0
 * outside the cone); endpoint_weight[num_endpoints].  Asynchronous on
 * `stream`. */
int jq_repcut_build(uint32_t num_pins, const uint8_t *kind, const uint32_t *fa, const uint32_t *fb,
                    const uint32_t *fanout_start, const uint32_t *fanouts, const uint8_t *staged,
                    uint32_t num_endpoints, const uint32_t *ep_start, const uint32_t *ep_pins,
                    const uint32_t *nfe, const uint32_t *rlevel_nodes,
                    const uint32_t *rlevel_start_host, uint32_t num_rlevels,
                    const uint32_t *flevel_nodes, const uint32_t *flevel_start_host,
                    uint32_t num_flevels, const uint32_t *supp_start_host,
                    const uint32_t *supp_edges, const uint8_t *wsupp, uint32_t num_fanouts,
                    uint32_t *supp_bits, unsigned long long *sets, uint8_t *cone,
                    unsigned long long *fingerprint, uint32_t *popcount, float *node_weight,
                    unsigned long long *endpoint_weight, void *stream);

/* Human-readable text for a status code. */
const char *jq_strerror(int code);

#ifdef __cplusplus
}
#endif

#endif
