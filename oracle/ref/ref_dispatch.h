// Build shim for compiling the reference's own CPU sources (src/cpu/*.cpp, src/*.cpp) in
// place. The reference's FAST_FSS_DISPATCH_INTEGRAL_TYPES (src/impl/def.h:38-45) also
// instantiates wideint::uint<2..4>, whose library is absent from the reference tree; this
// shim re-defines the macro with the same switch over elementSize restricted to the four
// built-in widths (1, 2, 4, 8 bytes). Any other elementSize takes the reference's own
// default case (FAST_FSS_INVALID_ELEMENT_SIZE_ERROR / size 0).
#pragma once
#include "impl/def.h"

#undef FAST_FSS_DISPATCH_INTEGRAL_TYPES
#define FAST_FSS_DISPATCH_INTEGRAL_TYPES(ELEMENT_SIZE, DEFAULT_CASE, ...)                             \
    _FAST_FSS_DISPATCH_SWITCH(ELEMENT_SIZE, DEFAULT_CASE,                                          \
                              _FAST_FSS_DISPATCH_CASE(std::uint8_t, __VA_ARGS__);                  \
                              _FAST_FSS_DISPATCH_CASE(std::uint16_t, __VA_ARGS__);                 \
                              _FAST_FSS_DISPATCH_CASE(std::uint32_t, __VA_ARGS__);                 \
                              _FAST_FSS_DISPATCH_CASE(std::uint64_t, __VA_ARGS__);)                \
    ()
