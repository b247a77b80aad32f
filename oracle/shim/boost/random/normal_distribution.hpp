#pragma once
#include "tape.hpp"
namespace boost {
template<class T = double> struct normal_distribution {
  T m, s;
  normal_distribution(T m = T(0), T s = T(1)) : m(m), s(s) {}
  template<class E> T operator()(E&) const { return m + s*T(random_tape::next_normal()); }
};
}
