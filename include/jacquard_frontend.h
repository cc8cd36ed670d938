/*
 * jacquard_frontend.h -- host-side script front end (libjq_frontend.so).
 *
 * Builds the reference's FlattenedScriptV1 instruction stream from a design:
 *   design (AIG) -> major stages -> partitions -> boomerang stages -> script.
 * It takes the place of the reference's Rust front end
 * (src/sim/setup.rs:75-326 load_design, src/staging.rs, src/repcut.rs,
 * src/pe.rs, src/flatten.rs), which cannot be built here.  The script it emits
 * is consumed unchanged by the interpreter entry points in jacquard_b200.h.
 * Pure host code: no CUDA calls.
 */
#ifndef JACQUARD_FRONTEND_H
#define JACQUARD_FRONTEND_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Seeded synthetic design (aigpdk semantics).  See generate.cpp. */
typedef struct {
  uint64_t seed;
  uint32_t n_clusters;        /* 1 = flat levelized logic */
  uint32_t nodes_per_cluster; /* AND nodes per cluster */
  uint32_t depth;             /* logic levels */
  uint32_t fanin_window;      /* fanins drawn from the previous N levels */
  double intra_frac;          /* probability a fanin stays in its cluster */
  uint32_t n_dff, n_pi, n_po, n_sram;
  uint32_t sram_addr_bits;    /* used address bits of each SRAM (<= 13) */
  int32_t with_reset;         /* input 0 is a synchronous reset of every DFF */
} jqf_gen_params;

typedef struct {
  uint64_t num_pins, num_and, num_dffs, num_pos, num_srams;
  uint32_t clock_flag_pin, reset_pin;
} jqf_design_info_t;

#define JQF_SRAM_RECORD_WORDS (13 + 1 + 32 + 13 + 32 + 32)

void *jqf_generate(const jqf_gen_params *p, uint64_t *num_and);
void jqf_free_design(void *design);

/* AIG builder for designs read from a gate-level netlist (the handle is a
 * design: free it with jqf_free_design).  Signals are "iv" = pin << 1 |
 * invert; pin 0 is constant 0, so iv 0 / 1 are the constants.  Sources can
 * be added at any time.  jqf_builder_and folds constants and reuses an
 * existing gate for the same fanins (src/aig.rs:327-345), and returns the
 * gate's iv.  jqf_builder_output appends a primary output (unique) and
 * returns its index.  jqf_builder_finish checks the design and records its
 * clock-flag / reset pins for the stimulus helpers. */
void *jqf_builder_new(void);
uint32_t jqf_builder_input(void *b);
uint32_t jqf_builder_clock_flag(void *b);
uint32_t jqf_builder_dff(void *b);
int jqf_builder_set_dff(void *b, uint32_t index, uint32_t d_iv, uint32_t en_iv);
uint32_t jqf_builder_and(void *b, uint32_t a_iv, uint32_t b_iv);
int64_t jqf_builder_output(void *b, uint32_t iv);
int jqf_builder_finish(void *b, uint32_t clock_flag_pin, uint32_t reset_pin);
int jqf_design_info(void *design, jqf_design_info_t *out);
/* Copy one design array (see capi.cpp for `which`); returns its byte size. */
int64_t jqf_design_array(void *design, int which, void *dst, size_t cap);
/* Per-pin gate delays in ps (num_pins + 1 entries each), injected into the
 * script's padding slots at build time (src/flatten.rs:1812-1846). */
int jqf_set_delays(void *design, const uint32_t *rise, const uint32_t *fall, size_t n);

typedef struct {
  size_t num_blocks;           /* CTAs of the interpreter launch */
  int32_t xprop;               /* classify X-capable partitions, words 8/9 */
  uint32_t n_level_split;
  const uint32_t *level_split; /* cumulative global levels (--level-split) */
  uint32_t target_cone;        /* partitioner: AND nodes per chunk (0 = default) */
  uint32_t target_endpoint_bits;
  int32_t num_threads;         /* 0 = all host threads */
  int32_t merge_passes;
  /* Optional learned partition cost model (JQF_COST_MODEL_FLOATS floats:
   * W1[128][24] b1[128] W2[128][128] b2[128] W3[128] b3, then feature mean[24]
   * and 1/std[24]).  When set, partition merges are accepted when the
   * predicted kernel time of the merged partition is below the sum of the
   * two; otherwise the stage-count rule is used. */
  const float *cost_model;
  /* Partitioner: when non-zero, each major stage's endpoints are cut into at
   * most this many chunks of balanced cone size (the smallest bound on a
   * chunk's AND count that gives that many) instead of chunks of
   * target_cone, and merges keep every partition within that bound.  The
   * batched kernel runs one work item per (partition, lane-word group) per
   * CTA, so grid / groups partitions per stage keep every stage to one
   * round of items. */
  uint32_t target_parts;
  /* Balanced mode without a cost model: a chunk's cost adds input_weight16 /
   * 16 gates per distinct chunk input (the batched kernel's global read
   * loads one slot per input); 0 counts gates and SRAMs only. */
  uint32_t input_weight16;
} jqf_build_params;

#define JQF_FEATURES 24
#define JQF_COST_MODEL_FLOATS (128 * 24 + 128 + 128 * 128 + 128 + 128 + 1 + 24 + 24)

typedef struct {
  uint64_t num_blocks, num_major_stages, blocks_data_len;
  uint32_t reg_io_state_size, sram_storage_size;
  uint32_t xprop_enabled, xprop_state_offset;
  uint64_t num_partitions, num_delay_patches, total_boomerang_stages;
} jqf_script_info_t;

void *jqf_build_script(void *design, const jqf_build_params *bp, char *err, size_t errlen);
void jqf_free_script(void *script);
int jqf_script_info(void *script, jqf_script_info_t *out);
int64_t jqf_script_array(void *script, int which, void *dst, size_t cap);

/* Features of every partition of a built script, in script order (major
 * stage, block, position): num_partitions x JQF_FEATURES floats. */
int jqf_script_features(void *design, void *script, float *out);
/* Host inference of a cost model on `n` feature rows (log kernel cycles). */
int jqf_cost_model_predict(const float *model, const float *features, size_t n, float *out);

/* RepCut hypergraph inputs of staged slice `slice` of the design under the
 * given level split (src/repcut.rs:58-176).  Outputs:
 *   - the fanout CSR of the AIG and the endpoint-group input pins (CSR);
 *   - staged-input flags;
 *   - the reverse / forward levels that schedule the propagation;
 *   - the traversal-order exceptions of the reference: per block of 4096
 *     endpoints the fanout edges that do not propagate (supp_start /
 *     supp_edges), and per-pin fanin weights that are skipped (wsupp).
 * Arrays may be NULL, which returns sizes only:
 *   fanout_start[num_pins+2], ep_start[E+1], supp_start[blocks+1];
 *   staged / rlevel / flevel / wsupp [num_pins+1];
 *   sizes = {E, fanouts length, ep_pins length, supp_edges length}.
 * Returns the number of slices, or -1. */
int jqf_repcut_slice(void *design, const uint32_t *level_split, size_t n_split, uint32_t slice,
                     uint32_t *fanout_start, uint32_t *fanouts, uint32_t *ep_start,
                     uint32_t *ep_pins, uint8_t *staged, uint32_t *rlevel, uint32_t *flevel,
                     uint32_t *supp_start, uint32_t *supp_edges, uint8_t *wsupp,
                     uint64_t *sizes);

/* Host-side script validator (same walk as the kernel). 0 = valid. */
int jqf_validate(const uint64_t *blocks_start, size_t num_blocks, size_t num_major_stages,
                 const uint32_t *blocks_data, size_t blocks_data_len,
                 uint32_t reg_io_state_size, uint32_t sram_storage_size,
                 size_t state_words, char *err, size_t errlen);

/* Timing constraint buffer, build_timing_constraint_buffer
 * (src/flatten.rs:1891-1924) with the clock-arrival fold of :97-123. */
int jqf_constraint_buffer(uint32_t num_words, uint64_t clock_period_ps, size_t n,
                          const uint16_t *setup_ps, const uint16_t *hold_ps,
                          const int16_t *clock_arrival_ps, const uint32_t *data_state_pos,
                          uint32_t *out_clock_ps, uint32_t *out_words);

/* Delay injection on explicit patch arrays (src/flatten.rs:1812-1846). */
int jqf_inject_delays(uint32_t *blocks_data, size_t blocks_data_len, size_t n_patches,
                      const uint64_t *offsets, const uint32_t *pins_start, const uint32_t *pins,
                      const uint16_t *rise, const uint16_t *fall, size_t n_pins);

#ifdef __cplusplus
}
#endif

#endif
