// Stand-alone log-weight reductions: ess_reduce and logsumexp_reduce
// (share/src/bi/primitive/vector_primitive.hpp:933-974), block-then-grid.
#include "internal.cuh"
#include "reduce.cuh"

namespace bpf {

// exp(d) for d <= 0 by the table-driven method (P. T. P. Tang, "Table-driven
// implementation of the exponential function in IEEE floating-point
// arithmetic", ACM TOMS 15(2), 1989): d = (64 m + j) ln2/64 + r with
// |r| <= ln2/128, exp(d) = 2^m * 2^(j/64) * e^r, e^r by its degree-5 Taylor
// polynomial (truncation below 4e-17 relative).  tab[j] = 2^(j/64).  A few
// ulp from the correctly rounded value, against ~30 FP64 operations for the
// general exp about 12.  Arguments below -690 (and NaN, -inf) give 0: such a
// term cannot change a sum that holds exp(0) = 1, which every sum here does.
constexpr double kInvLn2x64 = 92.33248261689366;     // 64 / ln 2
constexpr double kLn2d64Hi = 0.010830424696223417;   // ln 2 / 64, 36 significant bits
constexpr double kLn2d64Lo = 2.572804622327669e-14;  // ln 2 / 64 - kLn2d64Hi
__device__ __forceinline__ double exp_nonpos(double d, const double* __restrict__ tab) {
  const bool keep = d > -690.0;  // false also for NaN and -inf
  const double dc = keep ? d : 0.0;
  // k = rint(dc * 64/ln2) by the 1.5 * 2^52 rounding constant: its low
  // mantissa bits hold k (two's complement), no conversion instruction
  const double t = fma(dc, kInvLn2x64, 6755399441055744.0);
  const double kf = t - 6755399441055744.0;
  const int k = (int)__double2loint(t);  // in [-63710, 0]
  double r = fma(-kf, kLn2d64Hi, dc);
  r = fma(-kf, kLn2d64Lo, r);
  double p = fma(r, 1.0 / 120.0, 1.0 / 24.0);
  p = fma(p, r, 1.0 / 6.0);
  p = fma(p, r, 0.5);
  p = fma(p, r, 1.0);
  p = fma(p, r, 1.0);
  const double e = tab[k & 63] * p * __hiloint2double(((k >> 6) + 1023) << 20, 0);
  return keep ? e : 0.0;
}

// Fold a batch of log-weights into a thread partial: the batch maximum
// first (one rescaling exp when it raises the running maximum), then one exp
// per element relative to the running maximum.  NaN contributes nothing,
// -inf contributes exp(-inf) = 0, +inf empties the sums (nanexp(inf - inf)).
template <int K>
__device__ __forceinline__ void lw_push_batch(LwPartial& a, const double (&x)[K], const double* __restrict__ tab) {
  double bm = -INFINITY;
  bool pinf = false;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    if (!isnan(x[k])) bm = fmax(bm, x[k]);
    pinf |= (x[k] == INFINITY);
  }
  if (pinf || (isinf(a.mx) && a.mx > 0.0)) { a.mx = INFINITY; a.s1 = 0.0; a.s2 = 0.0; return; }
  if (bm > a.mx) {
    const double f = a.s1 == 0.0 ? 0.0 : exp_nonpos(a.mx - bm, tab);
    a.s1 *= f;
    a.s2 *= f * f;
    a.mx = bm;
  }
  if (isinf(a.mx)) return;  // nothing finite yet
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const double e = exp_nonpos(x[k] - a.mx, tab);  // NaN -> 0
    a.s1 += e;
    a.s2 += e * e;
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
  LwPartial v = lw_empty();
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
      lw_push_batch<K>(v, x, s_tab);
    }
  }
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
