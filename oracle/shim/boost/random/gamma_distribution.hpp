// Oracle test infrastructure: declared only so the reference headers compile;
// the oracle never draws from this distribution.
#pragma once
#include <stdexcept>
namespace boost {
template<class A = double, class B = double> struct gamma_distribution {
  template<class... X> gamma_distribution(X...) {}
  template<class E> A operator()(E&) const { throw std::runtime_error("gamma_distribution not on the oracle path"); }
};
}
