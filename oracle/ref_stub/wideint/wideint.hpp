// Minimal stand-in for the wideint library (github.com/oldprincess/wideint), which the
// reference tree references as an empty git submodule. It declares only the names the
// reference's <=64-bit code paths mention (src/impl/def.h:42-44, src/impl/number.h:17-28,74);
// no wide-integer arithmetic is provided, so only elementSize 1/2/4/8 are built.
#pragma once
#include <cstddef>

namespace wideint {
namespace detail {
template <std::size_t N, bool Signed>
class basic_int;
} // namespace detail

template <std::size_t N>
using uint = detail::basic_int<N, false>;

template <class T>
int countl_zero(const T &) noexcept;
} // namespace wideint
