// Block-then-grid log-sum-exp + ESS reduction (device functions).
//
// Replaces bi::ess_reduce and bi::logsumexp_reduce
// (share/src/bi/primitive/vector_primitive.hpp:933-974), which make two
// Thrust passes (max_element with nan_less_functor, then a transform_reduce of
// (e, e^2) with e = nanexp(lw - max)) and return scalars to the host.  Here
// each thread keeps an online (max, sum e, sum e^2) in FP64, blocks combine
// them with warp shuffles, and the last block to finish combines the block
// partials in a fixed order, so the result is deterministic and stays on the
// device.
#pragma once
#include "internal.cuh"

namespace bpf {

__device__ __forceinline__ LwPartial lw_combine(LwPartial a, LwPartial b) {
  LwPartial r;
  r.mx = nan_max(a.mx, b.mx);
  if (isinf(r.mx)) {  // both empty / all -inf, or a +inf log-weight
    r.s1 = 0.0; r.s2 = 0.0;
    return r;
  }
  double fa = a.s1 == 0.0 ? 0.0 : exp(a.mx - r.mx);
  double fb = b.s1 == 0.0 ? 0.0 : exp(b.mx - r.mx);
  r.s1 = a.s1 * fa + b.s1 * fb;
  r.s2 = a.s2 * fa * fa + b.s2 * fb * fb;
  return r;
}

__device__ __forceinline__ LwPartial lw_empty() {
  LwPartial r; r.mx = -INFINITY; r.s1 = 0.0; r.s2 = 0.0; return r;
}

// online update with one log-weight.  NaN contributes nothing (nanexp);
// -inf contributes exp(-inf) = 0; +inf becomes the max and, as
// nanexp(inf - inf) = 0 in the reference, leaves every weight zero.
__device__ __forceinline__ void lw_push(LwPartial& a, double x) {
  if (isnan(x)) return;
  if (isinf(a.mx) && a.mx > 0.0) return;
  if (isinf(x)) {
    if (x > 0.0) { a.mx = x; a.s1 = 0.0; a.s2 = 0.0; }
    return;
  }
  if (x > a.mx) {
    double f = a.s1 == 0.0 ? 0.0 : exp(a.mx - x);
    a.s1 = a.s1 * f + 1.0;
    a.s2 = a.s2 * f * f + 1.0;
    a.mx = x;
  } else {
    double e = exp(x - a.mx);
    a.s1 += e;
    a.s2 += e * e;
  }
}

__device__ __forceinline__ LwPartial warp_combine(LwPartial v) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) {
    LwPartial o;
    o.mx = __shfl_down_sync(0xffffffffu, v.mx, d);
    o.s1 = __shfl_down_sync(0xffffffffu, v.s1, d);
    o.s2 = __shfl_down_sync(0xffffffffu, v.s2, d);
    v = lw_combine(v, o);
  }
  return v;
}

// Combine one partial per thread across the block; result valid in thread 0.
__device__ __forceinline__ LwPartial block_combine(LwPartial v) {
  __shared__ LwPartial wp[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
  v = warp_combine(v);
  if (lane == 0) wp[warp] = v;
  __syncthreads();
  if (warp == 0) {
    v = lane < nw ? wp[lane] : lw_empty();
    v = warp_combine(v);
  }
  __syncthreads();
  return v;
}

enum FinalizeMode { kFinalizeReduce = 0, kFinalizeStep = 1, kFinalizeLogsumexp = 2 };

// Called by every thread of the last block: combine partials[0..np) in a
// fixed order and write the statistics.
__device__ __forceinline__ void finalize_partials(const LwPartial* partials, int np, int n,
                                                  StepStats* st, int mode, int observed) {
  LwPartial v = lw_empty();
  for (int i = threadIdx.x; i < np; i += blockDim.x) {
    LwPartial p;
    p.mx = __ldcg(&partials[i].mx);
    p.s1 = __ldcg(&partials[i].s1);
    p.s2 = __ldcg(&partials[i].s2);
    v = lw_combine(v, p);
  }
  v = block_combine(v);
  if (threadIdx.x == 0) {
    st->mx = v.mx;
    st->s1 = v.s1;
    st->s2 = v.s2;
    // ess_reduce: sum.first^2 / sum.second; lW = mx + log(sum.first) - log(n)
    st->ess = v.s1 * v.s1 / v.s2;
    st->lW = v.mx + log(v.s1) - log((double)n);
    if (mode == kFinalizeLogsumexp) {
      st->lW = v.mx + log(v.s1);
    } else if (mode == kFinalizeStep) {
      if (observed) {
        // BootstrapPF::correct, share/src/bi/filter/BootstrapPF.hpp:176-179
        st->inc = st->lW - st->ll;
        st->ll = st->lW;
        st->step += 1;
        // Resampler::resample trigger, share/src/bi/resampler/Resampler.hpp:168
        st->resample = st->ess < st->ess_rel * (double)n ? 1 : 0;
      } else {
        st->resample = 0;
      }
    }
  }
}

}  // namespace bpf
