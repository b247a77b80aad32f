// Oracle test infrastructure: BOOST_AUTO / BOOST_TYPEOF via C++11 keywords.
#pragma once
#define BOOST_AUTO(var, expr) auto var = (expr)
#define BOOST_AUTO_TPL(var, expr) auto var = (expr)
#define BOOST_TYPEOF(expr) decltype(expr)
#define BOOST_TYPEOF_TPL(expr) decltype(expr)
#define BOOST_TYPEOF_REGISTER_TEMPLATE(a, b)
#define BOOST_TYPEOF_INCREMENT_REGISTRATION_GROUP()
