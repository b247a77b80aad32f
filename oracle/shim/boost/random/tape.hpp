// Oracle test infrastructure: tape-replay random numbers.
//
// The reference draws every variate through boost::variate_generator over a
// distribution object.  This stand-in serves the draws from a caller-filled
// tape of uniforms on (0,1) instead, in the order the reference consumes them
// (one host thread), so that the reference's own resampler code can be run on
// exactly the uniforms the CUDA path uses:
//   uniform_real(a,b)        -> a + (b-a)*u
//   uniform_int(lo,hi)       -> lo + min(floor(u*(hi-lo+1)), hi-lo)
//   normal_distribution(m,s) -> m + s*u      (u then holds a standard normal)
#pragma once
#include <cstddef>
#include <stdexcept>
namespace boost { namespace random_tape {
struct Tape { const double* data = nullptr; std::size_t n = 0, pos = 0; };
inline Tape& tape() { static thread_local Tape t; return t; }
inline void set(const double* d, std::size_t n) { tape().data = d; tape().n = n; tape().pos = 0; }
inline std::size_t consumed() { return tape().pos; }
inline double next() {
  Tape& t = tape();
  if (t.pos >= t.n) throw std::runtime_error("random tape exhausted");
  return t.data[t.pos++];
}
}}
