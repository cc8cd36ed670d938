// Script front end: synthetic design -> staged AIG -> partitions -> boomerang
// stages -> flattened script (the reference's FlattenedScriptV1 layout).
#pragma once
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "aig.hpp"

namespace jq {

constexpr int BOOM_STAGES = 13;                  // src/pe.rs:27
constexpr uint32_t NT = 1u << (BOOM_STAGES - 5);  // 256 threads, src/flatten.rs:24
constexpr uint32_t MAX_WRITEOUTS = NT;           // src/pe.rs:29

// ---------------------------------------------------------------- generator
struct GenParams {
  uint64_t seed = 1;
  uint32_t n_clusters = 1;
  uint32_t nodes_per_cluster = 16384;
  uint32_t depth = 32;
  uint32_t fanin_window = 4;
  double intra_frac = 1.0;
  uint32_t n_dff = 1024, n_pi = 32, n_po = 32, n_sram = 0;
  uint32_t sram_addr_bits = 10;
  int with_reset = 0;
};
struct GenInfo {
  uint64_t num_and = 0;
  uint32_t clock_flag_pin = 0, reset_pin = 0;
};
AIG generate_design(const GenParams &p, GenInfo *info);

// ---------------------------------------------------------------- staging
// StagedAIG (src/staging.rs:12-21): a horizontal slice of the AIG between two
// global level splits.  Endpoint e < staged_outputs.size() is a staged IO pin;
// otherwise it is original endpoint group endpoints[e - staged_outputs.size()].
struct StagedAIG {
  std::vector<uint8_t> is_staged_input;  // per pin: produced by an earlier slice
  bool has_staged_inputs = false;
  std::vector<uint32_t> staged_outputs;  // pins
  std::vector<uint32_t> endpoints;       // original endpoint-group ids
  size_t num_endpoint_groups() const { return staged_outputs.size() + endpoints.size(); }
  template <class F>
  void for_each_input(const AIG &g, size_t e, F &&f) const {
    if (e < staged_outputs.size()) {
      f(staged_outputs[e]);
    } else {
      g.for_each_endpoint_input(endpoints[e - staged_outputs.size()], f);
    }
  }
  bool is_leaf(const AIG &g, uint32_t pin) const {
    return g.kind[pin] != DRV_AND || (has_staged_inputs && is_staged_input[pin]);
  }
};
std::vector<StagedAIG> build_staged_aigs(const AIG &g, const std::vector<uint32_t> &level_split);

// ---------------------------------------------------------------- packer
struct BoomStage {
  // hier[l][j]: pin at level l slot j (size 8192 >> l), NONE = unused.
  std::vector<uint32_t> hier[BOOM_STAGES + 1];
  std::vector<uint16_t> write_outs;  // word indices into the `after` layout
};
struct Partition {
  std::vector<uint32_t> endpoints;  // staged endpoint ids
  std::vector<BoomStage> stages;
  uint32_t cone_ands = 0;  // AND gates in the partition's cone
  uint32_t targets = 0;    // distinct endpoint input pins
};
struct PackOptions {
  int max_stages = 64;
  // every gate at tree level 1 (one logic level per boomerang stage): the
  // form the batched kernel evaluates as dense slot lists
  bool flat = false;
};
// Builds one partition; returns false when the endpoint set does not fit the
// 256-thread boomerang resources (the caller splits it).
bool build_partition(const AIG &g, const StagedAIG &st,
                     const std::vector<uint32_t> &endpoints, Partition &out,
                     const PackOptions &opt);

struct CostModel;

// ---------------------------------------------------------------- partitioner
struct PartitionOptions {
  uint32_t target_cone = 3000;     // AND nodes per initial chunk
  uint32_t target_endpoint_bits = 2048;
  int num_threads = 0;             // 0 = hardware concurrency
  int merge_passes = 1;
  // when non-zero, each stage is cut into at most this many chunks of
  // balanced cone size instead of chunks of target_cone, and merges keep
  // every partition's cone within the balanced bound
  uint32_t target_parts = 0;
  // balanced mode without a cost model: cut cost per distinct chunk input,
  // in 1/16 of an AND gate (the cost model picks this weight per stage)
  uint32_t input_weight16 = 0;
  // when set, balanced cuts are chosen and merges accepted on predicted
  // kernel time instead of the fixed weights and the stage-count rule
  const CostModel *cost_model = nullptr;
  const std::vector<uint8_t> *xpins = nullptr;
};
std::vector<Partition> partition_stage(const AIG &g, const StagedAIG &st,
                                       const PartitionOptions &opt);

// ---------------------------------------------------------------- flattener
struct FlatScript {
  size_t num_blocks = 0, num_major_stages = 0;
  std::vector<size_t> blocks_start;
  std::vector<uint32_t> blocks_data;
  uint32_t reg_io_state_size = 0;
  uint32_t sram_storage_size = 0;  // u32 words
  std::vector<uint32_t> input_layout;
  // (pin, state bit position) pairs, insertion order of the reference maps
  std::vector<std::pair<uint32_t, uint32_t>> input_map;   // pin -> pos
  std::vector<std::pair<uint32_t, uint32_t>> output_map;  // pin_iv -> pos
  std::vector<std::pair<uint32_t, uint32_t>> staged_io_map;
  std::vector<std::vector<std::vector<uint32_t>>> stages_blocks_parts;
  // per partition in (major stage, block, part) order
  std::vector<uint8_t> partition_x_capable;
  std::vector<uint32_t> part_num_stages;
  bool xprop_enabled = false;
  uint32_t xprop_state_offset = 0;
  // delay patch map: (blocks_data offset, AIG pins at that thread position)
  std::vector<size_t> delay_patch_offset;
  std::vector<uint32_t> delay_patch_pins_start;  // CSR into delay_patch_pins
  std::vector<uint32_t> delay_patch_pins;
  // DFF constraints (one per DFF): position of D in state, effective values
  std::vector<uint32_t> dff_data_pos;
  // the partitions in script order (major stage, block, position), pointing
  // into the caller's partition vectors
  std::vector<const Partition *> part_ptrs;
  std::vector<uint32_t> part_major_stage;
};
struct FlattenOptions {
  size_t num_blocks = 148;
  bool xprop = false;
};
bool flatten_script(const AIG &g, const std::vector<StagedAIG> &stageds,
                    const std::vector<std::vector<Partition>> &parts,
                    const FlattenOptions &opt, FlatScript &out, std::string *err);

// src/flatten.rs:1812-1846: per-thread-position max gate delay into padding.
void inject_timing(FlatScript &s, const std::vector<uint32_t> &rise,
                   const std::vector<uint32_t> &fall);

// ---------------------------------------------------------------- cost model
// Partition features for the learned cost model (24 per partition); computed
// identically for built partitions (training) and merge candidates.
constexpr int NFEAT = 24;
void partition_features(const AIG &g, const StagedAIG &st, const Partition &p,
                        const std::vector<uint8_t> *xpins, float *f);

// A small MLP (NFEAT -> 128 -> 128 -> 1, ReLU) evaluated on the host with
// bf16-rounded weights and fp32 accumulation; predicts log(kernel cycles).
struct CostModel {
  std::vector<float> w1, b1, w2, b2, w3;  // row-major [out][in]
  float b3 = 0;
  std::vector<float> mean, inv_std;       // feature normalisation
  bool valid() const { return !w1.empty(); }
  float predict(const float *feat) const;
};

// ---------------------------------------------------------------- checker
// Walks blocks_data the way the kernel does and checks every index against
// the state/SRAM sizes (src/flatten.rs:1526-1532 layout).  Returns "" if ok.
std::string validate_script(const FlatScript &s, size_t state_words_per_snapshot);

}  // namespace jq
