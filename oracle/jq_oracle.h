/*
 * jq_oracle.h -- CPU oracle for the Boolean-processor interpreter.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA path is
 * compared against; it is never linked into, called by, or used as a fallback
 * for the product library (libjacquard_b200.so).  Only tests/, the smoke check
 * and the CPU-baseline leg of bench.py load it.
 *
 * What it restates (reference paths are relative to the Jacquard tree):
 *   - src/sim/cpu_reference.rs:17-289   simulate_block_v1        (2-state)
 *   - src/sim/cpu_reference.rs:299-674  simulate_block_v1_xprop  (X lanes)
 *   - src/sim/cpu_reference.rs:679-790  sanity_check_cpu[_xprop] (loop order,
 *                                       next-snapshot pre-seed)
 *   - csrc/kernel_v1_impl.cuh:32-626    the CUDA kernel's per-partition X
 *                                       dispatch, u16 arrival tracking and
 *                                       setup/hold event emission, including
 *                                       the per-CTA persistent shared arrays
 *                                       (writeouts, writeout X, writeout
 *                                       arrival) that carry values across
 *                                       partitions, major stages and cycles.
 *   - csrc/event_buffer.h:35-50,89-111  event record layout and append rule.
 */
#ifndef JQ_ORACLE_H
#define JQ_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* One violation / event record; identical layout to the reference's Event
 * (csrc/event_buffer.h:35-40): 8 x u32 = 32 bytes. */
typedef struct {
  uint32_t event_type;
  uint32_t message_id;
  uint32_t cycle;
  uint32_t reserved;
  uint32_t data[4];
} jqo_event;

/* Flags for jqo_simulate. */
#define JQO_FLAG_CPU_XPROP_QUIRK 1u /* reproduce cpu_reference.rs:335-348: in an
                                       X run, the first non-X-capable partition
                                       of a block hands the REST of the block to
                                       the 2-state routine and returns. */
#define JQO_FLAG_FORCE_ARRIVALS 2u  /* track arrivals even when neither an
                                       arrival section nor constraints are
                                       requested (no observable effect). */

/*
 * Run num_cycles cycles of the flattened script over the snapshot buffer, in
 * the kernel's order: for cycle, for major stage, for block.  Semantics are
 * those of simulate_v1_noninteractive_simple_scan (kernel_v1_impl.cuh:565).
 *
 *   states               (num_cycles+1)*state_size u32, in/out; snapshot 0 is
 *                        the initial state, later snapshots are pre-filled by
 *                        the caller with that edge's inputs.
 *   sram_xmask           may be NULL when no partition is X-capable.
 *   timing_constraints   [clock_ps, one word per state word] or NULL.
 *   events/event_cap     event sink (may be NULL with cap 0); *event_count
 *                        counts every violation seen, like the reference's
 *                        atomic counter, even past the cap.
 *   num_threads          >1 runs the blocks of one major stage on that many
 *                        host threads (blocks are independent within a stage).
 * Returns 0, or a negative code on a malformed script (see jq_oracle.c).
 */
int jqo_simulate(size_t num_blocks, size_t num_major_stages,
                 const size_t *blocks_start, const uint32_t *blocks_data,
                 uint32_t *sram_data, uint32_t *sram_xmask, size_t num_cycles,
                 size_t state_size, uint32_t *states,
                 const uint32_t *timing_constraints, jqo_event *events,
                 size_t event_cap, uint64_t *event_count,
                 int32_t arrival_state_offset, uint32_t flags, int num_threads);

/*
 * One block's partition list against explicit input/output state (the unit the
 * reference CPU tests drive, cpu_reference.rs:17 and :299).  `x_input` /
 * `x_output` follow the kernel convention: the X-mask words live at
 * state + xmask_state_offset (metadata word 9), so pass the same arrays.
 * Persistent per-block arrays start zeroed.  Returns script words consumed or
 * a negative error.
 */
long jqo_simulate_block(const uint32_t *script, size_t script_size,
                        const uint32_t *input_state, uint32_t *output_state,
                        uint32_t *sram_data, uint32_t *sram_xmask,
                        uint32_t flags);

/* The X-propagation AND of cpu_reference.rs:434-439 / kernel_v1_impl.cuh:214-220. */
void jqo_xprop_and(uint32_t a_v, uint32_t a_x, uint32_t b_v, uint32_t b_x,
                   uint32_t xora, uint32_t xorb, uint32_t orb, uint32_t *ret_v,
                   uint32_t *ret_x);

/* DFF commit with clock-enable gating, kernel_v1_impl.cuh:515-527. */
void jqo_dff_commit(uint32_t old_v, uint32_t old_x, uint32_t new_v,
                    uint32_t new_x, uint32_t clken, uint32_t clken_x,
                    uint32_t *wo_v, uint32_t *wo_x);

/* Setup / hold predicates of kernel_v1_impl.cuh:543-556 (restated as test
 * helpers in src/flatten.rs:3076-3094).  Return 1 and write the slack when the
 * check fires. */
int jqo_setup_violation(uint16_t arrival, uint16_t setup_ps,
                        uint32_t clock_period, int32_t *slack);
int jqo_hold_violation(uint16_t arrival, uint16_t hold_ps, int32_t *slack);

/*
 * Netlist-level checker, independent of any script: evaluates the AIG gate
 * by gate in pin (topological) order, one cycle at a time, with the clocked
 * semantics the script encodes -- Q(next) = en ? D : Q; SRAM read data
 * (next) = r_en ? ram[r_addr] : previous; then ram[w_addr] takes wr_data on
 * the bits of wr_en (read before write).  Used to check that a script built
 * by the front end computes the design it came from.
 *   in_vals   (num_cycles+1) x n_in bytes (0/1): input_layout pin values.
 *   dff_state (num_cycles+1) x n_dff bytes: row 0 is the initial state (in),
 *             rows 1.. are written.
 *   po_vals   (num_cycles+1) x n_po bytes: row c+1 = outputs computed from
 *             row c's inputs and state (row 0 untouched).
 *   sram_words n_sram * 8192 u32 (in/out); sram_rd n_sram*32 bytes per row
 *             (num_cycles+1 rows, row 0 in).
 * Two-state only.  Returns 0.
 */
int jqo_aig_simulate(uint32_t num_pins, const uint8_t *kind, const uint32_t *fa,
                     const uint32_t *fb, size_t n_dff, const uint32_t *dff_d,
                     const uint32_t *dff_en, const uint32_t *dff_q, size_t n_sram,
                     const uint32_t *sram_rec, size_t n_in, const uint32_t *in_pins,
                     size_t num_cycles, const uint8_t *in_vals, uint8_t *dff_state,
                     size_t n_po, const uint32_t *po_iv, uint8_t *po_vals,
                     uint32_t *sram_words, uint8_t *sram_rd);

/* RepCut endpoint-set clusters and endpoint weights of one staged slice
 * (src/repcut.rs:58-176), from the arrays of jqf_repcut_slice.  Returns the
 * number of clusters (class_of_pin, cluster_first, cluster_count filled in
 * first-occurrence order), or -1. */
int jqo_repcut(uint32_t num_pins, const uint8_t *kind, const uint32_t *fa, const uint32_t *fb,
               const uint32_t *fanout_start, const uint32_t *fanouts, const uint8_t *staged,
               uint32_t num_endpoints, const uint32_t *ep_start, const uint32_t *ep_pins,
               int32_t *class_of_pin, uint32_t *cluster_first, uint32_t *cluster_count,
               uint64_t *endpoint_weight);

#ifdef __cplusplus
}
#endif

#endif
