#pragma once
#include "tape.hpp"
namespace boost {
template<class T = int> struct uniform_int {
  T lo, hi;
  uniform_int(T lo = 0, T hi = 9) : lo(lo), hi(hi) {}
  template<class E> T operator()(E&) const {
    double u = random_tape::next_uniform();
    T span = hi - lo;
    T k = static_cast<T>(u*(double(span) + 1.0));
    return lo + (k < span ? k : span);
  }
};
}
