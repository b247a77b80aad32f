// Oracle test infrastructure: minimal stand-in for boost::mpl::if_c / if_
// so that the reference's headers compile without Boost installed.
#pragma once
#include <type_traits>
namespace boost { namespace mpl {
template<bool C, class T1, class T2> struct if_c { typedef T1 type; };
template<class T1, class T2> struct if_c<false,T1,T2> { typedef T2 type; };
template<class C, class T1, class T2> struct if_ : if_c<bool(C::value),T1,T2> {};
}}
