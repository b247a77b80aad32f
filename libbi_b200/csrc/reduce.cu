// Stand-alone log-weight reductions: ess_reduce and logsumexp_reduce
// (share/src/bi/primitive/vector_primitive.hpp:933-974), block-then-grid.
#include "internal.cuh"
#include "reduce.cuh"

namespace bpf {

// Each block folds a contiguous chunk of lw into one partial; the last block
// to finish combines the partials in block order.
__global__ void __launch_bounds__(kBlock)
k_lw_reduce(const double* __restrict__ lw, int n, int chunk, LwPartial* partials, StepStats* st,
            unsigned* counter, int mode) {
  const int b = blockIdx.x;
  const int begin = b * chunk;
  const int end = min(n, begin + chunk);
  LwPartial v = lw_empty();
  const bool vec = ((reinterpret_cast<uintptr_t>(lw) & 15) == 0) && (chunk % 2 == 0);
  if (vec) {
    const double2* p = reinterpret_cast<const double2*>(lw + begin);
    const int pairs = (end - begin) / 2;
    for (int k = threadIdx.x; k < pairs; k += blockDim.x) {
      double2 t = __ldg(p + k);
      lw_push(v, t.x);
      lw_push(v, t.y);
    }
    if (((end - begin) & 1) && threadIdx.x == 0) lw_push(v, __ldg(lw + end - 1));
  } else {
    for (int i = begin + threadIdx.x; i < end; i += blockDim.x) lw_push(v, __ldg(lw + i));
  }
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
  // enough blocks to fill the GPU, each folding at least one tile
  int blocks = (n + kTile - 1) / kTile;
  if (blocks > 148 * 4) blocks = 148 * 4;
  if (blocks > s.max_partials) blocks = s.max_partials;
  int chunk = (n + blocks - 1) / blocks;
  chunk = (chunk + 1) & ~1;
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
