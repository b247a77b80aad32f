/*
 * libbi_b200 — device-side pieces of the step statistics, for kernels
 * compiled outside the library (a model's own fused transition,
 * include/bpf_model.cuh) as well as the library's own.  CUDA C++ only.
 *
 * A filter step ends with the log-weight reduction of Resampler::reduce ->
 * ess_reduce (share/src/bi/resampler/Resampler.hpp:156-163,
 * share/src/bi/primitive/vector_primitive.hpp:960-974) and the bookkeeping
 * of BootstrapPF::correct (share/src/bi/filter/BootstrapPF.hpp:171-181).
 * Here each thread keeps an online (max, sum e, sum e^2) in FP64 for its
 * particles; a block takes the maximum of its threads' maxima, rescales each
 * thread's sums with one exp and adds them; the last block to finish
 * combines the block partials the same way in a fixed order, so the result
 * is deterministic, stays on the device and is identical whichever kernel
 * (built-in or compiled from a model class) produced the log-weights.
 */
#ifndef BPF_DEVICE_CUH
#define BPF_DEVICE_CUH

#include <cuda_runtime.h>
#include <stdint.h>
#include "libbi_b200.h"

namespace bpf {

// Programmatic dependent launch.  A kernel launched with the programmatic
// stream serialization attribute (bpf::launch_pdl) may be scheduled while the
// kernel before it on the stream is still running; pdl_wait() blocks until
// that kernel has completed and its memory operations are visible, and must
// come before any access to what it wrote (it returns at once for a kernel
// launched without the attribute).  pdl_trigger() lets the next such kernel
// be scheduled early; it is launched once every block of this kernel has
// triggered or exited, and still waits in pdl_wait() for this kernel to
// complete.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// One block's (or thread's) share of the reduction: max log-weight and the
// sums of e and e^2 with e = nanexp(lw - mx).
struct LwPartial {
  double mx, s1, s2;
};

// Device-side results of a reduction / filter step (one per filter).
struct StepStats {
  double mx;        // max log-weight
  double s1, s2;    // sum e, sum e^2 with e = nanexp(lw - mx)
  double ess;       // s1^2 / s2
  double lW;        // mx + log s1 - log N
  double ll;        // logLikelihood
  double inc;       // logIncrement of the latest correct
  int resample;     // next step resamples (ESS < essRel*N after an observed step)
  int resampled;    // this step resampled
  int status;       // BPF_OK / BPF_E_DEGENERATE / BPF_E_TIMEOUT
  int step;         // schedule index of the latest correct (0 = initial)
  double ess_rel;
  int n;
  int pad;
  // a whole-filter run's per-step record (inc, ess, resampled) at
  // hist[3 (step - 1)], written by the step's last block; null outside one
  double* hist;
  int hist_n;       // steps hist holds
  int pad2;
};


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

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, d));
  return v;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
  return v;
}

// Combine one partial per thread across the block (blockDim.x a multiple of
// 32, at most 1024); the result is valid in every thread.  Max first, then one
// rescaling exp per partial and plain sums, so the critical path holds a
// single exp.
__device__ __forceinline__ LwPartial block_combine(LwPartial v) {
  __shared__ double s_m[32], s_1[32], s_2[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = blockDim.x >> 5;
  double m = warp_max(v.mx);  // partial maxima are never NaN
  if (lane == 0) s_m[warp] = m;
  __syncthreads();
  double M = lane < nw ? s_m[lane] : -INFINITY;
  M = warp_max(M);
  // empty partials (s1 == 0) contribute nothing, also when M is infinite
  const double f = v.s1 == 0.0 ? 0.0 : exp(v.mx - M);
  double a = warp_sum(v.s1 * f), b = warp_sum(v.s2 * f * f);
  if (lane == 0) { s_1[warp] = a; s_2[warp] = b; }
  __syncthreads();
  a = lane < nw ? s_1[lane] : 0.0;
  b = lane < nw ? s_2[lane] : 0.0;
  LwPartial r;
  r.mx = M;
  r.s1 = warp_sum(a);
  r.s2 = warp_sum(b);
  if (isinf(M)) { r.s1 = 0.0; r.s2 = 0.0; }
  __syncthreads();
  return r;
}

enum FinalizeMode { kFinalizeReduce = 0, kFinalizeStep = 1, kFinalizeLogsumexp = 2 };

// Called by every thread of the last block: combine partials[0..np) in a
// fixed order and write the statistics.
__device__ __forceinline__ void finalize_partials(const LwPartial* partials, int np, int n,
                                                  StepStats* st, int mode, int observed) {
  // each thread folds a fixed, strided subset of the partials (max first,
  // then rescaled sums); loads are issued kBatch at a time so that the last
  // block waits for a few memory round trips, not one per partial
  constexpr int kBatch = 8;
  const int nt = blockDim.x;
  double m = -INFINITY;
  for (int base = 0; base < np; base += nt * kBatch) {
    double v[kBatch];
#pragma unroll
    for (int k = 0; k < kBatch; ++k) {
      const int i = base + k * nt + threadIdx.x;
      v[k] = i < np ? __ldcg(&partials[i].mx) : -INFINITY;
    }
#pragma unroll
    for (int k = 0; k < kBatch; ++k) m = fmax(m, v[k]);
  }
  LwPartial v;
  v.mx = m; v.s1 = 0.0; v.s2 = 0.0;
  if (!isinf(m)) {
    for (int base = 0; base < np; base += nt * kBatch) {
      double pm[kBatch], p1[kBatch], p2[kBatch];
#pragma unroll
      for (int k = 0; k < kBatch; ++k) {
        const int i = base + k * nt + threadIdx.x;
        pm[k] = i < np ? __ldcg(&partials[i].mx) : 0.0;
        p1[k] = i < np ? __ldcg(&partials[i].s1) : 0.0;
        p2[k] = i < np ? __ldcg(&partials[i].s2) : 0.0;
      }
#pragma unroll
      for (int k = 0; k < kBatch; ++k) {
        if (p1[k] == 0.0) continue;
        const double f = exp(pm[k] - m);
        v.s1 += p1[k] * f;
        v.s2 += p2[k] * f * f;
      }
    }
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

// ---------------------------------------------------------------------------
// the end of every transition block: this block's (max, sum e, sum e^2) to
// partials[pidx]; the last of the np blocks that share `counter` combines
// partials[pbase .. pbase + np) and writes the step statistics.  Returns true
// in the block that finalised.
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool transition_reduce_tail(LwPartial part, LwPartial* partials, int pidx, int pbase,
                                                       int np, unsigned* counter, int n, StepStats* st, bool ok,
                                                       int resampled, bool observed) {
  part = block_combine(part);
  if (threadIdx.x == 0) partials[pidx] = part;
  __shared__ bool am_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) am_last = atomicAdd(counter, 1u) == (unsigned)np - 1;
  __syncthreads();
  if (am_last) {
    __threadfence();
    if (ok) {
      finalize_partials(partials + pbase, np, n, st, kFinalizeStep, observed);
      if (threadIdx.x == 0) {
        st->resampled = resampled;
        double* h = st->hist;
        const int k = st->step;
        if (h && observed && k >= 1 && k <= st->hist_n) {
          h[3 * (k - 1) + 0] = st->inc;
          h[3 * (k - 1) + 1] = st->ess;
          h[3 * (k - 1) + 2] = (double)resampled;
        }
      }
    }
    if (threadIdx.x == 0) *counter = 0;
  }
  return am_last;
}


// Launch a kernel with the programmatic stream serialization attribute (its
// body starts with pdl_wait()).
template <class... KArgs, class... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                              Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, args...);
}

}  // namespace bpf

#endif
