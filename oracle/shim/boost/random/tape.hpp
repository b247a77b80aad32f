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
// Timing mode (no tape on this thread): draws cycle through process-wide
// tables of standard normals and of uniforms filled by the timing harness,
// each thread from its own position, at the cost of a load per draw.  Used
// only to time the reference's filter loop on many threads, never for parity.
struct Cycle { const double* nrm = nullptr; const double* uni = nullptr; std::size_t n = 0; };
inline Cycle& cycle() { static Cycle c; return c; }
inline std::size_t& cycle_pos() {
  static thread_local std::size_t p = reinterpret_cast<std::size_t>(&p) / 64 * 2654435761u;
  return p;
}
inline double next_normal() {
  if (tape().data) return next();
  const Cycle& c = cycle();
  if (!c.nrm) throw std::runtime_error("random tape unset");
  return c.nrm[cycle_pos()++ % c.n];
}
inline double next_uniform() {
  if (tape().data) return next();
  const Cycle& c = cycle();
  if (!c.uni) throw std::runtime_error("random tape unset");
  return c.uni[cycle_pos()++ % c.n];
}
}}
