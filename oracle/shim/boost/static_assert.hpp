// Oracle test infrastructure: BOOST_STATIC_ASSERT in terms of static_assert.
#pragma once
#define BOOST_STATIC_ASSERT(x) static_assert((x), #x)
