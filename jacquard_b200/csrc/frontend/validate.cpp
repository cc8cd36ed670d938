// Script validator: walks blocks_data exactly as the interpreter does
// (partition size = 256 + 512*R + 5120*S + 2*5120, src/flatten.rs:1526-1532)
// and checks every offset and index the kernel will dereference, so that a
// malformed script is rejected on the host before any launch.
#include "frontend.hpp"

#include <sstream>

namespace jq {

std::string validate_script(const FlatScript &s, size_t state_words) {
  std::ostringstream err;
  const size_t nb = s.num_blocks, nms = s.num_major_stages;
  if (nms > 32) return "more than 32 major stages";
  if (s.blocks_start.size() != nb * nms + 1) return "blocks_start size";
  if (s.blocks_start.back() + 8 * NT > s.blocks_data.size()) return "missing tail padding";
  const uint32_t rio = s.reg_io_state_size;
  for (size_t bi = 0; bi < nb * nms; ++bi) {
    size_t pi = s.blocks_start[bi], end = s.blocks_start[bi + 1];
    if (end < pi) return "blocks_start not monotone";
    for (;;) {
      if (pi + NT > end) { err << "block " << bi << ": truncated metadata"; return err.str(); }
      const uint32_t *m = &s.blocks_data[pi];
      uint32_t ns = m[0];
      if (!ns) { pi += NT; break; }
      uint32_t nio = m[2], io = m[3], nsr = m[4], sro = m[5], R = m[6], nd = m[7];
      uint32_t isx = m[8], xo = m[9];
      if (nio > NT || nsr * 4 + nd > NT || nsr + nd > nio) { err << "block " << bi << ": io counts"; return err.str(); }
      if ((size_t)io + nio > rio) { err << "block " << bi << ": io range past state"; return err.str(); }
      if ((size_t)sro + (size_t)nsr * SRAM_WORDS > s.sram_storage_size) { err << "block " << bi << ": sram range"; return err.str(); }
      if (isx && (size_t)xo + rio > state_words) { err << "block " << bi << ": xmask offset"; return err.str(); }
      for (int t = 0; t < (int)NT; ++t) {
        uint32_t w = m[128 + t / 2];
        uint32_t h = (t & 1) ? w >> 16 : w & 0xffff;
        if (h != 0xffff && (h >> 8) >= ns) { err << "block " << bi << ": hook stage"; return err.str(); }
      }
      size_t need = NT + 2 * (size_t)NT * R + 5120 * ((size_t)ns + 2);
      if (pi + need > end) { err << "block " << bi << ": partition overruns block"; return err.str(); }
      const uint32_t *g = m + NT;
      for (uint32_t t = 0; t < NT; ++t) {
        uint32_t bits = 0;
        for (uint32_t r = 0; r < R; ++r) {
          uint32_t idx = g[r * 2 * NT + 2 * t], mask = g[r * 2 * NT + 2 * t + 1];
          if (!mask) continue;
          bits += (uint32_t)__builtin_popcount(mask);
          if ((idx & 0x7fffffffu) >= rio) { err << "block " << bi << ": global read index"; return err.str(); }
        }
        // a thread appends at most 32 bits (one state word)
        if (bits > 32) { err << "block " << bi << ": global read bits per thread"; return err.str(); }
      }
      const uint32_t *st = g + 2 * (size_t)NT * R;
      for (uint32_t k = 0; k < ns + 2; ++k) {
        const uint32_t *ch = st + 5120 * (size_t)k;
        for (int q = 0; q < 4096; ++q) {
          uint32_t w = ch[q];
          if ((w & 0xffff) >= 8192 || (w >> 16) >= 8192) { err << "block " << bi << ": shuffle index"; return err.str(); }
        }
      }
      // SRAM/duplicate and clock-enable permutations read writeout slots:
      // every used entry must point below num_ios * 32
      for (uint32_t k = ns; k < ns + 2; ++k) {
        const uint32_t *ch = st + 5120 * (size_t)k;
        const uint32_t nq = (k == ns ? nsr * 4 + nd : nio) * 32;
        for (uint32_t q = 0; q < nq; ++q) {
          const uint32_t T = q >> 5, kk = q & 31;
          const uint32_t w = ch[(kk >> 3) * 1024 + T * 4 + ((kk >> 1) & 3)];
          const uint32_t e = (kk & 1) ? (w >> 16) : (w & 0xffff);
          if (e >= nio * 32) { err << "block " << bi << ": writeout permutation index"; return err.str(); }
        }
      }
      // SRAM port addresses are 13 bits: bits 13..15 of the read and write
      // address words must be forced to 0 (set0 on, inversion off)
      {
        const uint32_t *F = st + 5120 * (size_t)ns + 4096;
        for (uint32_t i = 0; i < nsr; ++i) {
          const uint32_t inv = F[4 * (4 * i) + 0], set0 = F[4 * (4 * i) + 1];
          const uint32_t hi = 0xe000e000u;
          if ((set0 & hi) != hi || (inv & hi) != 0) { err << "block " << bi << ": SRAM address bits"; return err.str(); }
        }
      }
      pi += need;
      if (m[1]) break;
    }
    if (pi != end) { err << "block " << bi << ": size mismatch"; return err.str(); }
  }
  return "";
}

}  // namespace jq
