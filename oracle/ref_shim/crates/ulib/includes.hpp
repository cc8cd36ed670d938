// Type shim so the reference kernel sources compile on their own.
// The reference includes <crates/ulib/includes.hpp> from its vendored `ulib`
// crate (empty in this checkout); the kernel only needs these fixed-width
// aliases.  Used by oracle/build_ref.sh, never by the product library.
#pragma once
#include <cstddef>
#include <cstdint>
typedef std::uint8_t u8;
typedef std::uint16_t u16;
typedef std::uint32_t u32;
typedef std::uint64_t u64;
typedef std::int32_t i32;
typedef std::size_t usize;
