// Minimal stand-in for boost/math/constants: only the two constants the
// reference's hot path uses. Values are the exact mathematical constants,
// rounded to T by the conversion, as Boost does for float/double.
#pragma once
namespace boost { namespace math { namespace constants {
template <class T> inline T pi() { return static_cast<T>(3.141592653589793238462643383279502884L); }
template <class T> inline T one_div_two_pi() { return static_cast<T>(0.159154943091895335768883763372514362L); }
}}}
