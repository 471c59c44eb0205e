/* ORACLE PIN — test infrastructure only; never linked into the product.
 *
 * Stand-in for the two boost::math::ccmath functions that the reference's
 * corelib/internal/common/math/math_acos_lt.cpp names (boost is an empty submodule in the reference
 * tree).  They are only used by math::acos_approx, which the pinned path does not call; acos_lt,
 * the table lookup the CPU environment lookup uses, needs neither. */
#pragma once
#include <cmath>

namespace boost::math::ccmath {
template<class T> constexpr T abs(T x) { return x < T(0) ? -x : x; }
template<class T> inline T sqrt(T x) { return std::sqrt(x); }
}  // namespace boost::math::ccmath
