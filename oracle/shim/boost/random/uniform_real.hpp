#pragma once
#include "tape.hpp"
namespace boost {
template<class T = double> struct uniform_real {
  T a, b;
  uniform_real(T a = T(0), T b = T(1)) : a(a), b(b) {}
  template<class E> T operator()(E&) const { return a + (b - a)*T(random_tape::next_uniform()); }
};
}
