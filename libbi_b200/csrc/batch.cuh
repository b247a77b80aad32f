// A batch of independent filters in shared structure-of-arrays buffers
// (batch.cu): the per-filter layout the batch kernels index through, and
// the per-step history record.  The guided step of a batch (guided.cu) uses
// the same layout.
#pragma once
#include "internal.cuh"

namespace bpf {

struct BatchFilter {
  int n;          // particles
  int off;        // first column in the shared buffers
  int block0;     // first transition block (and partial)
  int nblocks;    // transition blocks
  int resampler;  // BPF_RESAMPLER_*
  int B;          // Metropolis steps
  uint64_t seed;
  int tile0;      // first 128-particle tile of the guided step
  int ntiles;     // 128-particle tiles of the guided step
};

// the finalising block of filter f appends (logIncrement, ESS, resampled)
__device__ __forceinline__ void batch_record(const StepStats* st, double* hist, int nf, int f, int k) {
  if (hist && threadIdx.x == 0) {
    double* h = hist + 3 * ((size_t)k * nf + f);
    h[0] = st->inc;
    h[1] = st->ess;
    h[2] = (double)st->resampled;
  }
}

// the batched resampler (batch.cu): one CTA of `threads` threads per filter
int launch_batch_resample(const double* lw, int* as, const BatchFilter* filt, const int* order, int nf,
                          int max_n, StepStats* stats, double* lu_buf, int* os_buf, int step, cudaStream_t st,
                          int threads);
int configure_batch_resample(int max_n);
int tune_batch_resample(const BatchFilter* filt, const int* order, int nf, int max_n, int ld, cudaStream_t st,
                        int* best, double* us);

}  // namespace bpf
