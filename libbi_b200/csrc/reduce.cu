// Stand-alone log-weight reductions: ess_reduce and logsumexp_reduce
// (share/src/bi/primitive/vector_primitive.hpp:933-974), block-then-grid.
#include "internal.cuh"
#include "reduce.cuh"

namespace bpf {

// exp(d) by the table-driven method (P. T. P. Tang, "Table-driven
// implementation of the exponential function in IEEE floating-point
// arithmetic", ACM TOMS 15(2), 1989): d = (64 m + j) ln2/64 + r with
// |r| <= ln2/128, exp(d) = 2^m * 2^(j/64) * e^r, e^r by its degree-5 Taylor
// polynomial (truncation below 4e-17 relative).  tab[j] = 2^(j/64).  A few
// ulp from the correctly rounded value, against ~30 FP64 operations for the
// general exp about 12.  exp_table takes d in (-690, kLazyMargin]: 2^m then
// stays a normal number and is added to the exponent field of tab[j]
// (exact).  exp_nonpos also takes arguments below -690 (and NaN, -inf) and
// gives 0 for them: such a term cannot change a sum that holds exp(0) = 1,
// and every sum here holds the term of the value that set its reference.
constexpr double kInvLn2x64 = 92.33248261689366;     // 64 / ln 2
constexpr double kLn2d64Hi = 0.010830424696223417;   // ln 2 / 64, 36 significant bits
constexpr double kLn2d64Lo = 2.572804622327669e-14;  // ln 2 / 64 - kLn2d64Hi
constexpr double kRound52 = 6755399441055744.0;      // 1.5 * 2^52
// a thread's sums are kept relative to a reference c that is raised only when
// a value exceeds it by more than this, so the rescaling exp is rare; terms
// stay below e^(2 * 128) and the sums far from overflow
constexpr double kLazyMargin = 128.0;

__device__ __forceinline__ double exp_table(double d, const double* __restrict__ tab) {
  // k = rint(d * 64/ln2) by the 1.5 * 2^52 rounding constant: its low
  // mantissa bits hold k (two's complement), no conversion instruction
  const double t = fma(d, kInvLn2x64, kRound52);
  const double kf = t - kRound52;
  const int k = (int)__double2loint(t);  // in [-63710, 11818]
  double r = fma(-kf, kLn2d64Hi, d);
  r = fma(-kf, kLn2d64Lo, r);
  double p = fma(r, 1.0 / 120.0, 1.0 / 24.0);
  p = fma(p, r, 1.0 / 6.0);
  p = fma(p, r, 0.5);
  p = fma(p, r, 1.0);
  p = fma(p, r, 1.0);
  const double tj = tab[k & 63];
  const double ts = __hiloint2double(__double2hiint(tj) + (k >> 6) * (1 << 20), __double2loint(tj));
  return ts * p;
}

__device__ __forceinline__ double exp_nonpos(double d, const double* __restrict__ tab) {
  const bool keep = d > -690.0;  // false also for NaN and -inf
  const double e = exp_table(keep ? d : 0.0, tab);
  return keep ? e : 0.0;
}

// A thread's running statistics: maximum mx, and s1 = sum e^(x - c),
// s2 = sum e^(2 (x - c)) relative to the reference c (c <= mx < c + margin).
struct LwAcc {
  double mx, c, s1, s2;
};

__device__ __forceinline__ LwAcc acc_empty() {
  LwAcc a;
  a.mx = -INFINITY;
  a.c = -INFINITY;
  a.s1 = 0.0;
  a.s2 = 0.0;
  return a;
}

// The thread's statistics relative to its maximum, as a partial.
__device__ __forceinline__ LwPartial acc_partial(const LwAcc& a, const double* __restrict__ tab) {
  LwPartial v;
  v.mx = a.mx;
  v.s1 = a.s1;
  v.s2 = a.s2;
  if (a.s1 != 0.0 && a.c != a.mx) {
    const double f = exp_nonpos(a.c - a.mx, tab);
    v.s1 *= f;
    v.s2 *= f * f;
  }
  return v;
}

// Fold a batch of log-weights into a thread's statistics: one exp per
// element relative to the reference.  NaN contributes nothing, -inf
// contributes exp(-inf) = 0, +inf empties the sums (nanexp(inf - inf)).
// fmax ignores NaN, so the batch maximum is that of its non-NaN values.
template <int K>
__device__ __forceinline__ void lw_push_batch(LwAcc& a, const double (&x)[K], const double* __restrict__ tab) {
  double bm = -INFINITY;
#pragma unroll
  for (int k = 0; k < K; ++k) bm = fmax(bm, x[k]);
  if (bm == INFINITY || a.mx == INFINITY) {
    a.mx = INFINITY;
    a.s1 = 0.0;
    a.s2 = 0.0;
    return;
  }
  a.mx = fmax(a.mx, bm);
  if (bm > a.c + kLazyMargin) {  // also the first finite batch (c = -inf)
    if (a.s1 != 0.0) {
      const double f = exp_nonpos(a.c - bm, tab);
      a.s1 *= f;
      a.s2 *= f * f;
    }
    a.c = bm;
  }
  if (a.c == -INFINITY) return;  // nothing finite yet
  double d[K];
  bool fast = true;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    d[k] = x[k] - a.c;
    fast &= d[k] > -690.0;  // false for NaN and -inf
  }
  if (fast) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const double e = exp_table(d[k], tab);
      a.s1 += e;
      a.s2 += e * e;
    }
  } else {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const double e = exp_nonpos(d[k], tab);
      a.s1 += e;
      a.s2 += e * e;
    }
  }
}

// Each block folds a contiguous chunk of lw into one partial, eight values per
// thread per iteration with 16-byte loads; the last block to finish combines
// the partials in block order.
constexpr int kReduceBlocksPerSm = 3;

__global__ void __launch_bounds__(kBlock, kReduceBlocksPerSm)
k_lw_reduce(const double* __restrict__ lw, int n, int chunk, LwPartial* partials, StepStats* st,
            unsigned* counter, int mode) {
  constexpr int K = 8;
  __shared__ double s_tab[64];
  if (threadIdx.x < 64) s_tab[threadIdx.x] = exp2((double)threadIdx.x / 64.0);
  __syncthreads();
  const int b = blockIdx.x;
  const int begin = b * chunk;
  const int end = min(n, begin + chunk);
  LwAcc acc = acc_empty();
  const bool vec = ((reinterpret_cast<uintptr_t>(lw + begin) & 15) == 0);
  int i = begin + threadIdx.x * K;
  if (vec) {
    // the next batch's loads are issued before the current batch's exps, so
    // the memory latency overlaps the arithmetic
    const int stride = blockDim.x * K;
    double2 nxt[K / 2];
    if (i + K <= end) {
#pragma unroll
      for (int k = 0; k < K / 2; ++k) nxt[k] = __ldg(reinterpret_cast<const double2*>(lw + i) + k);
    }
    while (i + K <= end) {
      double x[K];
#pragma unroll
      for (int k = 0; k < K / 2; ++k) {
        x[2 * k] = nxt[k].x;
        x[2 * k + 1] = nxt[k].y;
      }
      i += stride;
      if (i + K <= end) {
#pragma unroll
        for (int k = 0; k < K / 2; ++k) nxt[k] = __ldg(reinterpret_cast<const double2*>(lw + i) + k);
      }
      lw_push_batch<K>(acc, x, s_tab);
    }
  }
  LwPartial v = acc_partial(acc, s_tab);
  // the tail (or an unaligned chunk) one element at a time
  for (; i < end; i += blockDim.x * K)
    for (int k = 0; k < K && i + k < end; ++k) lw_push(v, __ldg(lw + i + k));
  v = block_combine(v);
  if (threadIdx.x == 0) partials[b] = v;
  __shared__ bool am_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) am_last = atomicAdd(counter, 1u) == gridDim.x - 1;
  __syncthreads();
  if (am_last) {
    __threadfence();
    finalize_partials(partials, gridDim.x, n, st, mode, 0);
    if (threadIdx.x == 0) *counter = 0;
  }
}

static int lw_reduce_impl(const double* lw, int n, ResampleScratch& s, cudaStream_t st, int mode) {
  if (n <= 0 || lw == nullptr) return BPF_E_INVALID;
  // one wave of resident blocks, each folding at least 2048 values; chunks
  // are multiples of 8 so that every chunk stays 16-byte aligned when lw is
  int blocks = (n + 2047) / 2048;
  if (blocks > 148 * kReduceBlocksPerSm) blocks = 148 * kReduceBlocksPerSm;
  if (blocks > s.max_partials) blocks = s.max_partials;
  int chunk = (n + blocks - 1) / blocks;
  chunk = (chunk + 7) & ~7;
  blocks = (n + chunk - 1) / chunk;
  k_lw_reduce<<<blocks, kBlock, 0, st>>>(lw, n, chunk, s.partials, s.stats, s.counters + 3, mode);
  BPF_TRY(cudaGetLastError());
  return BPF_OK;
}

int launch_lw_reduce(const double* lw, int n, ResampleScratch& s, cudaStream_t st) {
  return lw_reduce_impl(lw, n, s, st, kFinalizeReduce);
}

int launch_logsumexp(const double* lw, int n, ResampleScratch& s, cudaStream_t st) {
  return lw_reduce_impl(lw, n, s, st, kFinalizeLogsumexp);
}

}  // namespace bpf
