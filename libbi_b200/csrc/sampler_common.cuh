// Host-side helpers shared by the samplers over the batched filter (PMMH in
// pmmh.cu, SMC^2 in smc2.cu): the priors' log-densities and the
// counter-based draws of their proposals.
#pragma once
#include "internal.cuh"
#include "../../include/bpf_math.h"

#include <cmath>

namespace bpf {
namespace sampler {

constexpr double kHalfLog2Pi = 0.91893853320467274178032973640562;

// log density of the prior of one parameter (the parameter block's
// log-density, e.g. share/tt/cpp/action/uniform.hpp.tt, gaussian.hpp.tt)
inline double log_prior(const bpf_pmmh_param& q, double x) {
  switch (q.prior) {
    case BPF_PRIOR_UNIFORM:
      return (x >= q.a && x <= q.b) ? -std::log(q.b - q.a) : -INFINITY;
    case BPF_PRIOR_LOG_NORMAL: {
      if (!(x > 0.0)) return -INFINITY;
      const double z = (std::log(x) - q.a) / q.b;
      return -0.5 * z * z - kHalfLog2Pi - std::log(q.b * x);
    }
    case BPF_PRIOR_GAUSSIAN: {
      const double z = (x - q.a) / q.b;
      return -0.5 * z * z - kHalfLog2Pi - std::log(q.b);
    }
    default:
      return -INFINITY;
  }
}

inline double normal_draw(uint64_t seed, int c, int r, int j) {
  bpf_u32x4 w = bpf_draw(seed, (uint32_t)c, (uint32_t)r, (uint32_t)(j / 2), BPF_RNG_PMMH);
  double z0, z1;
  bpf_normal_pair_d(w.v[0], w.v[1], &z0, &z1);
  return (j & 1) ? z1 : z0;
}

inline double uniform_draw(uint64_t seed, int c, int r, int blk) {
  bpf_u32x4 w = bpf_draw(seed, (uint32_t)c, (uint32_t)r, (uint32_t)blk, BPF_RNG_PMMH);
  return bpf_u01d(w.v[0], w.v[1]);
}

}  // namespace sampler
}  // namespace bpf
