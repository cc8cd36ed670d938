// AIG (and-inverter graph) for the script front end.
//
// Conventions follow the reference's AIG (src/aig.rs:173-289):
//   * pins are numbered 1..num_pins in topological order, pin 0 is Tie0;
//   * a signal reference "iv" is (pin << 1) | invert;
//   * an AND gate stores its two fanins (a_iv, b_iv) with a_iv < b_iv and is
//     structurally hashed (add_and_gate, src/aig.rs:327-345);
//   * endpoint groups are enumerated as [primary outputs][DFFs][SRAMs]
//     (src/aig.rs:2715-2743), each with the input pins of
//     EndpointGroup::for_each_input (src/aig.rs:129-168).
#pragma once
#include <cstdint>
#include <string>
#include <unordered_map>
#include <vector>

namespace jq {

constexpr uint32_t NONE = 0xffffffffu;
constexpr int SRAM_ADDR_BITS = 13;  // AIGPDK_SRAM_ADDR_WIDTH (src/aigpdk.rs:20)
constexpr uint32_t SRAM_WORDS = 1u << SRAM_ADDR_BITS;

enum DriverKind : uint8_t {
  DRV_TIE0 = 0,
  DRV_AND = 1,
  DRV_INPUT = 2,    // primary input port
  DRV_CLKFLAG = 3,  // clock edge flag (posedge / negedge of a clock port)
  DRV_DFF = 4,      // DFF Q output
  DRV_SRAM = 5,     // SRAM read-data bit
};

struct DFF {
  uint32_t d_iv = 0;   // data input with invert bit
  uint32_t en_iv = 0;  // clock enable (clock edge flag, set/reset overlay)
  uint32_t q = 0;      // Q pin (no invert)
};

// A synchronous single-clock RAM with the `$__RAMGEM_SYNC_` interface
// (src/aig.rs:95-108): 13-bit read/write addresses, 32 data bits.
struct RAMBlock {
  uint32_t r_addr_iv[SRAM_ADDR_BITS];
  uint32_t r_en_iv = 0;
  uint32_t r_data[32];  // read-data pins (no invert); NONE = unused
  uint32_t w_addr_iv[SRAM_ADDR_BITS];
  uint32_t w_en_iv[32];
  uint32_t w_data_iv[32];
};

struct AIG {
  uint32_t num_pins = 0;
  std::vector<uint8_t> kind{DRV_TIE0};
  std::vector<uint32_t> fa{0}, fb{0};  // AND fanins (iv) ; aux index for others
  std::unordered_map<uint64_t, uint32_t> and_cache;
  std::vector<uint32_t> primary_outputs;  // unique pin_iv, insertion order
  std::vector<DFF> dffs;
  std::vector<RAMBlock> srams;
  // Per-pin gate delay in ps (rise, fall); empty when no timing is loaded.
  std::vector<uint32_t> delay_rise, delay_fall;

  uint32_t add_pin(DriverKind k, uint32_t aux = 0) {
    ++num_pins;
    kind.push_back(k);
    fa.push_back(aux);
    fb.push_back(0);
    return num_pins;
  }
  // src/aig.rs:327-345: constant folding, (min,max) order, structural hash.
  uint32_t add_and(uint32_t a, uint32_t b) {
    if (a == 0 || b == 0) return 0;
    if (a == 1) return b;
    if (b == 1) return a;
    if (a > b) std::swap(a, b);
    uint64_t key = (uint64_t)a << 32 | b;
    auto it = and_cache.find(key);
    if (it != and_cache.end()) return it->second << 1;
    uint32_t p = add_pin(DRV_AND);
    fa[p] = a;
    fb[p] = b;
    and_cache.emplace(key, p);
    return p << 1;
  }
  bool is_and(uint32_t p) const { return kind[p] == DRV_AND; }

  size_t num_endpoint_groups() const {
    return primary_outputs.size() + dffs.size() + srams.size();
  }
  // EndpointGroup::for_each_input (src/aig.rs:129-168): pins (no invert),
  // zero skipped, duplicates possible.
  template <class F>
  void for_each_endpoint_input(size_t e, F &&f) const {
    auto g = [&](uint32_t pin) {
      if (pin >= 1) f(pin);
    };
    size_t npo = primary_outputs.size(), nd = dffs.size();
    if (e < npo) {
      g(primary_outputs[e] >> 1);
    } else if (e < npo + nd) {
      const DFF &d = dffs[e - npo];
      g(d.en_iv >> 1);
      g(d.d_iv >> 1);
    } else {
      const RAMBlock &r = srams[e - npo - nd];
      g(r.r_en_iv >> 1);
      for (int i = 0; i < SRAM_ADDR_BITS; ++i) {
        g(r.r_addr_iv[i] >> 1);
        g(r.w_addr_iv[i] >> 1);
      }
      for (int i = 0; i < 32; ++i) {
        g(r.w_en_iv[i] >> 1);
        g(r.w_data_iv[i] >> 1);
      }
    }
  }
  // Input layout (src/sim/setup.rs:211-216): every InputPort and
  // InputClockFlag pin, in pin order.
  std::vector<uint32_t> input_layout() const {
    std::vector<uint32_t> v;
    for (uint32_t p = 1; p <= num_pins; ++p)
      if (kind[p] == DRV_INPUT || kind[p] == DRV_CLKFLAG) v.push_back(p);
    return v;
  }
  // X sources and X-capable pins (src/aig.rs:3277-3366).
  std::vector<uint8_t> x_capable_pins(int *iterations = nullptr) const;
};

}  // namespace jq
