// Stand-in for the absent `cth` utility library, used only to compile the
// reference's CPU path in place (oracle/_ref). It provides the one facility
// the hot-path headers need: unary operator* on an enum yields its underlying
// value. The generator macro becomes a no-op because the template covers it.
#pragma once
#include <type_traits>

template<class E>
    requires std::is_enum_v<E>
constexpr auto operator*(E e) noexcept { return static_cast<std::underlying_type_t<E>>(e); }

#define CTH_GEN_ENUM_DEREF_OVERLOAD(E)
