#pragma once
namespace boost {
template<class E, class D> struct variate_generator {
  E e; D d;
  variate_generator(E e, D d) : e(e), d(d) {}
  auto operator()() { return d(e); }
};
}
