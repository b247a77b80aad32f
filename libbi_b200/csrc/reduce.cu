// Stand-alone log-weight reductions: ess_reduce and logsumexp_reduce
// (share/src/bi/primitive/vector_primitive.hpp:933-974), block-then-grid.
#include "internal.cuh"
#include "reduce.cuh"

namespace bpf {

// Fold a batch of log-weights into a thread partial: the batch maximum
// first (one rescaling exp when it raises the running maximum), then one exp
// per element relative to the running maximum.  NaN contributes nothing,
// -inf contributes exp(-inf) = 0, +inf empties the sums (nanexp(inf - inf)).
template <int K>
__device__ __forceinline__ void lw_push_batch(LwPartial& a, const double (&x)[K]) {
  double bm = -INFINITY;
  bool pinf = false;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    if (!isnan(x[k])) bm = fmax(bm, x[k]);
    pinf |= (x[k] == INFINITY);
  }
  if (pinf || (isinf(a.mx) && a.mx > 0.0)) { a.mx = INFINITY; a.s1 = 0.0; a.s2 = 0.0; return; }
  if (bm > a.mx) {
    const double f = a.s1 == 0.0 ? 0.0 : exp(a.mx - bm);
    a.s1 *= f;
    a.s2 *= f * f;
    a.mx = bm;
  }
  if (isinf(a.mx)) return;  // nothing finite yet
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const double e = isnan(x[k]) ? 0.0 : exp(x[k] - a.mx);
    a.s1 += e;
    a.s2 += e * e;
  }
}

// Each block folds a contiguous chunk of lw into one partial, eight values per
// thread per iteration with 16-byte loads; the last block to finish combines
// the partials in block order.
__global__ void __launch_bounds__(kBlock)
k_lw_reduce(const double* __restrict__ lw, int n, int chunk, LwPartial* partials, StepStats* st,
            unsigned* counter, int mode) {
  constexpr int K = 8;
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
      lw_push_batch<K>(v, x);
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
  // enough blocks to fill the GPU (8 per SM), each folding at least 2048
  // values; chunks are multiples of 8 so that every chunk stays 16-byte
  // aligned when lw is
  int blocks = (n + 2047) / 2048;
  if (blocks > 148 * 8) blocks = 148 * 8;
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
