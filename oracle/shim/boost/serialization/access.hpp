// Oracle test infrastructure: serialization is not exercised by the oracle;
// these declarations only let the reference's State headers compile.
#pragma once
namespace boost { namespace serialization {
class access {};
template<class B, class D> B& base_object(D& d) { return static_cast<B&>(d); }
template<class B, class D> const B& base_object(const D& d) { return static_cast<const B&>(d); }
template<class T> struct array_wrapper { T* p; std::size_t n; };
template<class T> array_wrapper<T> make_array(T* p, std::size_t n) { return array_wrapper<T>{p, n}; }
}}
#define BOOST_SERIALIZATION_SPLIT_MEMBER()
