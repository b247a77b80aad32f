// Oracle test infrastructure: engine stand-in; all draws come from the tape.
#pragma once
#include "tape.hpp"
namespace boost {
struct mt19937 { void seed(unsigned) {} };
}
