// Many independent bootstrap particle filters advanced together.
//
// LibBi runs the filters of a particle-marginal Metropolis-Hastings chain or
// of SMC^2's parameter particles one after another, each a full
// Filter<BootstrapPF>::filter (share/src/bi/sampler/MarginalMH.hpp:230-271,
// share/src/bi/sampler/MarginalSIR.hpp:283-420).  Here a batch holds F
// filters of one model (each with its own particle count, constants, seed and
// resampler) in shared structure-of-arrays buffers, and one filter step of
// the whole batch is two launches:
//   k_batch_resample      one 1024-thread CTA per filter that resamples
//                         (gated on the filter's own ESS flag): the permuted
//                         systematic, multinomial or Metropolis ancestors of
//                         the single-filter path, computed on chip
//   k_batch_*_transition  one thread per particle over all filters' blocks;
//                         the last block of each filter finalises that
//                         filter's ESS, lW, logLikelihood and resample flag
// Filter f's particles occupy columns [off_f, off_f + n_f) of every state
// row; its transition blocks never straddle another filter.  Filter f draws
// from the same random streams as a single filter with its seed, so a batch
// reproduces F single filters bit for bit.
#include "internal.cuh"
#include "reduce.cuh"
#include "model_body.cuh"
#include "resample_common.cuh"
#include "batch.cuh"
#include "../../include/bpf_math.h"
#include "proposal.cuh"

#include <algorithm>
#include <cmath>
#include <new>
#include <vector>

namespace bpf {

constexpr int kBatchThreads = 1024;

// ---------------------------------------------------------------------------
// initial draws (Simulator::init -> Model::initialSamples) and statistics
// ---------------------------------------------------------------------------
__device__ __forceinline__ void batch_stats_init(StepStats* st, int n, double ess_rel) {
  StepStats z{};
  z.mx = 0.0; z.s1 = 0.0; z.s2 = 0.0; z.ess = 0.0; z.lW = 0.0; z.ll = 0.0; z.inc = 0.0;
  z.resample = 0; z.resampled = 0; z.status = BPF_OK; z.step = 0; z.ess_rel = ess_rel; z.n = n;
  *st = z;
}

template <class T>
__global__ void k_batch_l96_init(T* x, int ld, int D, double* lw, const BatchFilter* filt, const L96Params* prms,
                                 const int* blk2f, StepStats* stats, double ess_rel) {
  const int f = __ldg(blk2f + blockIdx.x);
  const BatchFilter fd = filt[f];
  const int p = (blockIdx.x - fd.block0) * blockDim.x + threadIdx.x;
  if (p == 0) batch_stats_init(stats + f, fd.n, ess_rel);
  if (p >= fd.n) return;
  const T mean = (T)prms[f].x0_mean, sd = (T)prms[f].x0_std;
  const size_t col = (size_t)fd.off + p;
  for (int b = 0; b < (D + 3) / 4; ++b) {
    bpf_u32x4 r = bpf_draw(fd.seed, (uint32_t)p, 0u, (uint32_t)b, BPF_RNG_INIT);
    T z[4];
    box_muller(r.v[0], r.v[1], z[0], z[1]);
    box_muller(r.v[2], r.v[3], z[2], z[3]);
    for (int j = 0; j < 4; ++j) {
      const int i = 4 * b + j;
      if (i < D) x[(size_t)i * ld + col] = Prec<T>::fma_(sd, z[j], mean);
    }
  }
  lw[col] = 0.0;
}

template <class T>
__global__ void k_batch_pz_init(T* x, int ld, double* lw, const BatchFilter* filt, const PZParams* prms,
                                const int* blk2f, StepStats* stats, double ess_rel) {
  const int f = __ldg(blk2f + blockIdx.x);
  const BatchFilter fd = filt[f];
  const int p = (blockIdx.x - fd.block0) * blockDim.x + threadIdx.x;
  if (p == 0) batch_stats_init(stats + f, fd.n, ess_rel);
  if (p >= fd.n) return;
  const PZParams& prm = prms[f];
  const size_t col = (size_t)fd.off + p;
  bpf_u32x4 r = bpf_draw(fd.seed, (uint32_t)p, 0u, 0u, BPF_RNG_INIT);
  T z0, z1;
  box_muller(r.v[0], r.v[1], z0, z1);
  x[col] = Prec<T>::exp_(Prec<T>::fma_((T)prm.p0_sigma, z0, (T)prm.p0_mu));
  x[(size_t)ld + col] = Prec<T>::exp_(Prec<T>::fma_((T)prm.z0_sigma, z1, (T)prm.z0_mu));
  lw[col] = 0.0;
}

// ---------------------------------------------------------------------------
// transitions: the single-filter bodies, indexed through the block's filter
// ---------------------------------------------------------------------------
template <class T, int D>
__global__ void __launch_bounds__(kL96Block, l96_min_blocks(sizeof(T)))
k_batch_l96_transition(const T* __restrict__ x_in, T* __restrict__ x_out, int ld, int* __restrict__ as,
                       double* __restrict__ lw, const T* __restrict__ y, double t1d, double t2d, int step,
                       const BatchFilter* __restrict__ filt, const L96Params* __restrict__ prms,
                       const int* __restrict__ blk2f, StepStats* stats, LwPartial* partials, unsigned* counters,
                       double* hist, int nf, int k) {
  __shared__ T sx[D][kL96Block];
  const int f = __ldg(blk2f + blockIdx.x);
  const BatchFilter fd = filt[f];
  StepStats* st = stats + f;
  const int p = (blockIdx.x - fd.block0) * kL96Block + threadIdx.x;
  const int resampled = st->resample;
  const bool ok = st->status == BPF_OK;
  const T* yf = y ? y + (size_t)f * D : nullptr;
  LwPartial part = lw_empty();
  if (ok && p < fd.n) {
    const int col = fd.off + p;
    const int src = resampled ? min(max(as[col], 0), fd.n - 1) : p;
    T x0[D];
#pragma unroll
    for (int i = 0; i < D; ++i) x0[i] = __ldg(x_in + (size_t)i * ld + fd.off + src);
    l96_rk4<T, D>(x0, t1d, t2d, (T)prms[f].F, (T)prms[f].h);
#pragma unroll
    for (int i = 0; i < D; ++i) sx[i][threadIdx.x] = x0[i];
    // the filter's constants and log-likelihood are read after the ODE (not
    // held across it); the last block rewrites st->ll only after every
    // block has arrived
    const L96Params prm = prms[f];
    const double l = l96_noise_obs<T, D>(sx, x_out, (size_t)ld, col, yf, fd.seed, (uint32_t)p, step, prm,
                                         resampled ? st->ll : lw[col]);
    lw[col] = l;
    if (resampled) as[col] = src;
    lw_push(part, l);
  }
  if (transition_reduce_tail(part, partials, blockIdx.x, fd.block0, fd.nblocks, counters + f, fd.n, st, ok,
                             resampled, y != nullptr))
    batch_record(st, hist, nf, f, k);
}

template <class T>
__global__ void __launch_bounds__(kPZBlock)
k_batch_pz_transition(const T* __restrict__ x_in, T* __restrict__ x_out, int ld, int* __restrict__ as,
                      double* __restrict__ lw, const T* __restrict__ y, double t1d, double t2d, int step,
                      const BatchFilter* __restrict__ filt, const PZParams* __restrict__ prms,
                      const int* __restrict__ blk2f, StepStats* stats, LwPartial* partials, unsigned* counters,
                      double* hist, int nf, int k) {
  const int f = __ldg(blk2f + blockIdx.x);
  const BatchFilter fd = filt[f];
  StepStats* st = stats + f;
  const int p = (blockIdx.x - fd.block0) * kPZBlock + threadIdx.x;
  const int resampled = st->resample;
  const bool ok = st->status == BPF_OK;
  const PZParams prm = prms[f];
  LwPartial part = lw_empty();
  if (ok && p < fd.n) {
    const int col = fd.off + p;
    const int src = resampled ? min(max(as[col], 0), fd.n - 1) : p;
    T P = __ldg(x_in + fd.off + src), Z = __ldg(x_in + (size_t)ld + fd.off + src);
    const T alpha = pz_alpha<T>(fd.seed, (uint32_t)p, step, prm);
    pz_advance<T>(P, Z, alpha, t1d, t2d, prm);
    double l = resampled ? st->ll : lw[col];
    if (y) l += pz_obs_term<T>(P, __ldg(y + f), prm);
    x_out[col] = P;
    x_out[(size_t)ld + col] = Z;
    lw[col] = l;
    if (resampled) as[col] = src;
    lw_push(part, l);
  }
  if (transition_reduce_tail(part, partials, blockIdx.x, fd.block0, fd.nblocks, counters + f, fd.n, st, ok,
                             resampled, y != nullptr))
    batch_record(st, hist, nf, f, k);
}

// ---------------------------------------------------------------------------
// resampling, one CTA per filter
// ---------------------------------------------------------------------------
template <int NT>
__device__ __forceinline__ int block_exclusive_max_int_nt(int v, int* total) {
  __shared__ int wt[NT / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int inc = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    int o = __shfl_up_sync(0xffffffffu, inc, d);
    if (lane >= d) inc = max(inc, o);
  }
  const int excl_in_warp = __shfl_up_sync(0xffffffffu, inc, 1);
  if (lane == 31) wt[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    int t = lane < NT / 32 ? wt[lane] : 0;
#pragma unroll
    for (int d = 1; d < NT / 32; d <<= 1) {
      int o = __shfl_up_sync(0xffffffffu, t, d);
      if (lane >= d) t = max(t, o);
    }
    if (lane < NT / 32) wt[lane] = t;
  }
  __syncthreads();
  int r = warp > 0 ? wt[warp - 1] : 0;
  if (lane > 0) r = max(r, excl_in_warp);
  *total = wt[NT / 32 - 1];
  __syncthreads();
  return r;
}

__device__ __forceinline__ unsigned long long batch_q(const double* lwf, int i, double mx) {
  return weight_to_fixed(nanexp(__dsub_rn(__ldg(lwf + i), mx)));
}

__device__ __forceinline__ u128 u128_of(unsigned long long q) {
  u128 r; r.lo = q; r.hi = 0; return r;
}

// Number of entries of the nondecreasing lu[0..n) below x: a binary search
// over every 32nd entry (in shared memory), then over one run of 32 in L2.
__device__ __forceinline__ int count_below(const double* lu, const double* s_coarse, int nc, int n, double x) {
  int lo = 0, hi = nc;  // first coarse c with lu[32c] >= x
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (s_coarse[mid] < x) lo = mid + 1; else hi = mid;
  }
  // answer in (32(lo-1), 32 lo], clipped to [0, n]
  int a = lo > 0 ? 32 * (lo - 1) + 1 : 0;
  int b = min(n, 32 * lo);
  while (a < b) {
    const int mid = (a + b) >> 1;
    if (__ldcg(lu + mid) < x) a = mid + 1; else b = mid;
  }
  return a;
}

// Shared memory: marks (one int per particle), childless flags (one byte per
// particle), coarse multinomial index (kBatchThreads doubles).
inline size_t batch_resample_smem(int max_n) {
  return (size_t)max_n * sizeof(int) + (size_t)max_n + (size_t)kBatchThreads * sizeof(double) + 16;
}

// Batches whose largest filter has at most kBatchOsSmemMax particles keep
// the cumulative offspring in shared memory too (the SMEM_OS kernels): the
// CTA's passes over them then cost shared-memory latency instead of L2
// round trips
constexpr int kBatchOsSmemMax = 12288;
inline size_t batch_resample_smem_os(int max_n) { return batch_resample_smem(max_n) + (size_t)max_n * sizeof(int); }

template <bool SMEM_OS>
__device__ __forceinline__ int ld_os(const int* p) {
  if constexpr (SMEM_OS) return *p;
  else return __ldcg(p);
}

// Permuted ancestors of filter blockIdx.x, the rule of
// ResamplerHost::cumulativeOffspringToAncestorsPermute
// (share/src/bi/host/resampler/ResamplerHost.hpp:134-168) in closed form:
// survivors in place, extra copies by ancestor into the childless slots in
// ascending order.  Cumulative offspring of
//   systematic   SystematicResampler::cumulativeOffspring (SystematicResampler.hpp:111-130)
//   multinomial  MultinomialResamplerHost::ancestors (MultinomialResamplerHost.hpp:29-65)
//   Metropolis   MetropolisResamplerHost::ancestors (MetropolisResamplerHost.hpp:32-62)
// computed exactly as the single-filter kernels compute them.
template <int NT, bool SMEM_OS>
__global__ void __launch_bounds__(NT, 1)
k_batch_resample(const double* __restrict__ lw, int* __restrict__ as, const BatchFilter* __restrict__ filt,
                 const int* __restrict__ order, StepStats* stats, double* lu_buf, int* os_buf, int step) {
  extern __shared__ __align__(16) unsigned char s_raw[];
  pdl_trigger();  // a single filter's transition, a programmatic dependent, may be scheduled
  const int f = order[blockIdx.x];
  const BatchFilter fd = filt[f];
  StepStats* st = stats + f;
  if (st->resample == 0 || st->status != BPF_OK) return;  // uniform over the block
  const int n = fd.n;
  const double* lwf = lw + fd.off;
  int* asf = as + fd.off;
  double* s_coarse = reinterpret_cast<double*>(s_raw);
  int* marks = reinterpret_cast<int*>(s_raw + kBatchThreads * sizeof(double));  // layout for the largest NT
  // the cumulative offspring: after the marks in shared memory, or the
  // filter's columns of the global buffer
  int* osf = SMEM_OS ? marks + n : os_buf + fd.off;
  unsigned char* flags = reinterpret_cast<unsigned char*>(SMEM_OS ? osf + n : marks + n);
  const int IT = (n + NT - 1) / NT;
  const int i0 = min(n, threadIdx.x * IT);
  const int i1 = min(n, i0 + IT);
  const double mx = st->mx;
  const double nd = (double)n;

  // ---- cumulative offspring Os of this thread's particles, into osf ----
  if (fd.resampler == BPF_RESAMPLER_SYSTEMATIC || fd.resampler == BPF_RESAMPLER_MULTINOMIAL) {
    const bool mult = fd.resampler == BPF_RESAMPLER_MULTINOMIAL;
    u128 acc = u128_zero(), vacc = u128_zero();
    for (int i = i0; i < i1; ++i) {
      acc = u128_add(acc, u128_of(batch_q(lwf, i, mx)));
      if (mult) vacc = u128_add(vacc, spacing_to_fixed(multinomial_spacing(nullptr, i, n, fd.seed, step)));
    }
    u128 Wtot;
    const u128 texcl = block_exclusive_scan_u128_nt<NT>(acc, &Wtot);
    const double W = u128_to_weight(Wtot);
    // SystematicResampler::cumulativeOffspring throws
    // ParticleFilterDegeneratedException unless W > 0
    // (share/src/bi/resampler/SystematicResampler.hpp:118-129)
    if (!(W > 0.0)) {
      if (threadIdx.x == 0) st->status = BPF_E_DEGENERATE;
      return;
    }
    if (!mult) {
      bpf_u32x4 r = bpf_draw(fd.seed, 0u, (uint32_t)step, 0u, BPF_RNG_SYSTEMATIC);
      const double a = bpf_u01d(r.v[0], r.v[1]);
      const double yW = __ddiv_rn(1.0, W);
      u128 Q = texcl;
      for (int i = i0; i < i1; ++i) {
        Q = u128_add(Q, u128_of(batch_q(lwf, i, mx)));
        osf[i] = systematic_Os(u128_to_weight(Q), W, yW, nd, a, n);
      }
    } else {
      u128 Vtot;
      const u128 vexcl = block_exclusive_scan_u128_nt<NT>(vacc, &Vtot);
      const double lW = log(W);
      double* luf = lu_buf + fd.off;
      // lu_s = lW + lMax_s, lMax_s = -(sum of the spacings of slots >= s)
      u128 V = vexcl;
      for (int s = i0; s < i1; ++s) {
        const double lu = __dadd_rn(lW, -fixed_to_spacing(u128_sub(Vtot, V)));
        luf[s] = lu;
        if ((s & 31) == 0) s_coarse[s >> 5] = lu;
        V = u128_add(V, spacing_to_fixed(multinomial_spacing(nullptr, s, n, fd.seed, step)));
      }
      __syncthreads();
      const int nc = (n + 31) >> 5;
      // slot s takes the number of m with log(Ws_m) <= lu_s (clamped to n-1),
      // so Os_m = #{s : lu_s < log(Ws_m)} for m < n-1 and Os_{n-1} = n
      u128 Q = texcl;
      for (int m = i0; m < i1; ++m) {
        Q = u128_add(Q, u128_of(batch_q(lwf, m, mx)));
        osf[m] = m == n - 1 ? n : count_below(luf, s_coarse, nc, n, log(u128_to_weight(Q)));
      }
    }
  } else {
    // Metropolis: B steps per particle, then offspring counts and their
    // cumulative sums in place
    for (int i = i0; i < i1; ++i) osf[i] = 0;
    __syncthreads();
    for (int p = i0; p < i1; ++p) {
      const int a = metropolis_ancestor(lwf, n, fd.B, nullptr, fd.seed, step, p);
      atomicAdd(osf + a, 1);
    }
    __syncthreads();
    int loc = 0;
    for (int i = i0; i < i1; ++i) loc += ld_os<SMEM_OS>(osf + i);
    int tot;
    int run = block_exclusive_scan_int_nt<NT>(loc, &tot);
    for (int i = i0; i < i1; ++i) { run += ld_os<SMEM_OS>(osf + i); osf[i] = run; }
  }
  __syncthreads();

  // ---- permutation: childless counts, survivors, extra-copy marks ----
  const int before0 = i0 == 0 ? 0 : ld_os<SMEM_OS>(osf + i0 - 1);
  int zl = 0;
  {
    int prev = before0;
    for (int i = i0; i < i1; ++i) {
      const int o = ld_os<SMEM_OS>(osf + i);
      zl += (o == prev);
      prev = o;
    }
  }
  int ztot;
  const int zexcl = block_exclusive_scan_int_nt<NT>(zl, &ztot);
  for (int r = threadIdx.x; r < ztot; r += NT) marks[r] = 0;
  __syncthreads();
  {
    int prev = before0, Z = zexcl;
    for (int i = i0; i < i1; ++i) {
      const int o = ld_os<SMEM_OS>(osf + i);
      const bool zero = o == prev;
      flags[i] = zero;
      if (!zero) {
        asf[i] = i;
        // E_i = Os_{i-1} - i + Z_i extra copies precede particle i's
        const int e = prev - i + Z;
        if (o - prev >= 2 && e >= 0 && e < ztot) marks[e] = i + 1;
      }
      Z += zero;
      prev = o;
    }
  }
  __syncthreads();
  // inclusive max-scan of marks[0..ztot): rank r -> 1 + the ancestor whose
  // extra copies cover r
  {
    const int CH = (ztot + NT - 1) / NT;
    const int r0 = min(ztot, threadIdx.x * CH), r1 = min(ztot, r0 + CH);
    int m = 0;
    for (int r = r0; r < r1; ++r) m = max(m, marks[r]);
    int mtot;
    const int mexcl = block_exclusive_max_int_nt<NT>(m, &mtot);
    int run = mexcl;
    for (int r = r0; r < r1; ++r) { run = max(run, marks[r]); marks[r] = run; }
  }
  __syncthreads();
  {
    int Z = zexcl;
    for (int i = i0; i < i1; ++i)
      if (flags[i]) {
        // a consistent Os gives 1 <= marks[Z] <= n; anything else stays in range
        const int a = Z < ztot ? marks[Z] - 1 : i;
        asf[i] = a >= 0 && a < n ? a : i;
        ++Z;
      }
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
int launch_batch_init(const ModelArgs& m, void* x, int ld, double* lw, const BatchFilter* filt, const void* prms,
                      const int* blk2f, int blocks, StepStats* stats, double ess_rel, cudaStream_t st) {
  if (m.kind == BPF_MODEL_L96) {
    if (m.precision == BPF_F64)
      k_batch_l96_init<double><<<blocks, kL96Block, 0, st>>>((double*)x, ld, m.dim, lw, filt,
                                                             (const L96Params*)prms, blk2f, stats, ess_rel);
    else
      k_batch_l96_init<float><<<blocks, kL96Block, 0, st>>>((float*)x, ld, m.dim, lw, filt, (const L96Params*)prms,
                                                            blk2f, stats, ess_rel);
  } else {
    k_batch_pz_init<double><<<blocks, kPZBlock, 0, st>>>((double*)x, ld, lw, filt, (const PZParams*)prms, blk2f,
                                                         stats, ess_rel);
  }
  BPF_TRY(cudaGetLastError());
  return BPF_OK;
}

#define BATCH_L96_CASE(TT, DD)                                                                              \
  case DD:                                                                                                  \
    k_batch_l96_transition<TT, DD><<<blocks, kL96Block, 0, st>>>(                                           \
        (const TT*)x_in, (TT*)x_out, ld, as, lw, (const TT*)y, t1, t2, step, filt, (const L96Params*)prms, \
        blk2f, stats, partials, counters, hist, nf, k);                                                     \
    break;

int launch_batch_transition(const ModelArgs& m, const void* x_in, void* x_out, int ld, int* as, double* lw,
                            const void* y, double t1, double t2, int step, const BatchFilter* filt,
                            const void* prms, const int* blk2f, int blocks, StepStats* stats, LwPartial* partials,
                            unsigned* counters, double* hist, int nf, int k, cudaStream_t st) {
  if (m.kind == BPF_MODEL_L96) {
    if (m.precision == BPF_F64) {
      switch (m.dim) {
        BATCH_L96_CASE(double, 4) BATCH_L96_CASE(double, 8) BATCH_L96_CASE(double, 16)
        BATCH_L96_CASE(double, 32) BATCH_L96_CASE(double, 40)
        default: return BPF_E_INVALID;
      }
    } else {
      switch (m.dim) {
        BATCH_L96_CASE(float, 4) BATCH_L96_CASE(float, 8) BATCH_L96_CASE(float, 16)
        BATCH_L96_CASE(float, 32) BATCH_L96_CASE(float, 40)
        default: return BPF_E_INVALID;
      }
    }
  } else {
    k_batch_pz_transition<double><<<blocks, kPZBlock, 0, st>>>(
        (const double*)x_in, (double*)x_out, ld, as, lw, (const double*)y, t1, t2, step, filt,
        (const PZParams*)prms, blk2f, stats, partials, counters, hist, nf, k);
  }
  BPF_TRY(cudaGetLastError());
  return BPF_OK;
}

// threads per filter CTA of the batched resampler: 256, 512 or 1024 (the
// in-CTA arithmetic is exact, so the count changes the speed only)
int launch_batch_resample(const double* lw, int* as, const BatchFilter* filt, const int* order, int nf,
                          int max_n, StepStats* stats, double* lu_buf, int* os_buf, int step, cudaStream_t st,
                          int threads) {
  if (max_n <= kBatchOsSmemMax) {
    const size_t smem = batch_resample_smem_os(max_n);
    switch (threads) {
      case 256:
        k_batch_resample<256, true><<<nf, 256, smem, st>>>(lw, as, filt, order, stats, lu_buf, os_buf, step);
        break;
      case 512:
        k_batch_resample<512, true><<<nf, 512, smem, st>>>(lw, as, filt, order, stats, lu_buf, os_buf, step);
        break;
      case 1024:
        k_batch_resample<1024, true><<<nf, 1024, smem, st>>>(lw, as, filt, order, stats, lu_buf, os_buf, step);
        break;
      default: return BPF_E_INVALID;
    }
  } else {
    const size_t smem = batch_resample_smem(max_n);
    switch (threads) {
      case 256:
        k_batch_resample<256, false><<<nf, 256, smem, st>>>(lw, as, filt, order, stats, lu_buf, os_buf, step);
        break;
      case 512:
        k_batch_resample<512, false><<<nf, 512, smem, st>>>(lw, as, filt, order, stats, lu_buf, os_buf, step);
        break;
      case 1024:
        k_batch_resample<1024, false><<<nf, 1024, smem, st>>>(lw, as, filt, order, stats, lu_buf, os_buf, step);
        break;
      default: return BPF_E_INVALID;
    }
  }
  BPF_TRY(cudaGetLastError());
  return BPF_OK;
}

// The limit is a property of the kernel, shared by every batch: it is raised
// to what the largest allowed filter needs (a smaller batch created later
// must not lower it under a larger one), once per device.
int configure_batch_resample(int max_n) {
  if (max_n > BPF_BATCH_MAX_PARTICLES) return BPF_E_INVALID;
  static unsigned c256 = 0, c512 = 0, c1024 = 0, d256 = 0, d512 = 0, d1024 = 0;
  const int smem = (int)batch_resample_smem(BPF_BATCH_MAX_PARTICLES);
  BPF_TRY(set_dyn_smem_once(k_batch_resample<256, false>, smem, c256));
  BPF_TRY(set_dyn_smem_once(k_batch_resample<512, false>, smem, c512));
  BPF_TRY(set_dyn_smem_once(k_batch_resample<1024, false>, smem, c1024));
  const int smem_os = (int)batch_resample_smem_os(kBatchOsSmemMax);
  BPF_TRY(set_dyn_smem_once(k_batch_resample<256, true>, smem_os, d256));
  BPF_TRY(set_dyn_smem_once(k_batch_resample<512, true>, smem_os, d512));
  BPF_TRY(set_dyn_smem_once(k_batch_resample<1024, true>, smem_os, d1024));
  return BPF_OK;
}

// synthetic log-weights 2 N(0, 1) over the whole buffer, for the autotuner
__global__ void k_batch_synthetic_lw(double* lw, int ld) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ld) return;
  const bpf_u32x4 r = bpf_draw(0x7a11ull, (uint32_t)i, 0u, 0u, BPF_RNG_DATA);
  double z0, z1;
  bpf_normal_pair_d(r.v[0], r.v[1], &z0, &z1);
  lw[i] = 2.0 * z0;
}

// statistics that open every filter's resampling gate, with each filter's
// maximum log-weight
__global__ void k_batch_tune_stats(const double* lw, const BatchFilter* filt, StepStats* st, int nf) {
  const int f = blockIdx.x;
  if (f >= nf) return;
  const BatchFilter fd = filt[f];
  double m = -INFINITY;
  for (int i = threadIdx.x; i < fd.n; i += blockDim.x) m = fmax(m, lw[fd.off + i]);
  m = warp_max(m);
  __shared__ double s_m[32];
  if ((threadIdx.x & 31) == 0) s_m[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, s_m[w]);
    m = fmax(m, s_m[0]);
    StepStats z{};
    z.mx = m;
    z.resample = 1;
    z.status = BPF_OK;
    z.n = fd.n;
    st[f] = z;
  }
}

// Time the three thread counts on synthetic log-weights laid out as the
// batch's filters (scratch buffers: the batch's own state is untouched) and
// return the fastest; the medians go to us[3] (256, 512, 1024).
int tune_batch_resample(const BatchFilter* filt, const int* order, int nf, int max_n, int ld, cudaStream_t st,
                        int* best, double* us) {
  *best = kBatchThreads;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  BPF_TRY(cudaStreamIsCapturing(st, &cs));
  if (cs != cudaStreamCaptureStatusNone) return BPF_OK;  // no timing inside a capture: keep the default
  double* lw = nullptr;
  double* lu = nullptr;
  int *as = nullptr, *os = nullptr;
  StepStats* stats = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = BPF_OK;
  auto A = [&](void** p, size_t b) {
    if (!rc && cudaMalloc(p, b) != cudaSuccess) rc = BPF_E_NOMEM;
  };
  A((void**)&lw, (size_t)ld * sizeof(double));
  A((void**)&lu, (size_t)ld * sizeof(double));
  A((void**)&as, (size_t)ld * sizeof(int));
  A((void**)&os, (size_t)ld * sizeof(int));
  A((void**)&stats, (size_t)nf * sizeof(StepStats));
  if (!rc && (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)) rc = BPF_E_CUDA;
  if (!rc) {
    k_batch_synthetic_lw<<<(ld + 255) / 256, 256, 0, st>>>(lw, ld);
    k_batch_tune_stats<<<nf, 256, 0, st>>>(lw, filt, stats, nf);
    if (cudaGetLastError() != cudaSuccess) rc = BPF_E_CUDA;
  }
  // the sizes take turns, round after round, so that a drift of clocks or
  // caches during the tuning reaches every size alike; each size's median
  // decides
  const int counts[3] = {256, 512, 1024};
  constexpr int kReps = 9;
  float t[3][kReps];
  for (int r = -2; !rc && r < kReps; ++r) {  // two untimed rounds first
    for (int c = 0; !rc && c < 3; ++c) {
      if (r >= 0 && cudaEventRecord(e0, st) != cudaSuccess) { rc = BPF_E_CUDA; break; }
      rc = launch_batch_resample(lw, as, filt, order, nf, max_n, stats, lu, os, 1, st, counts[c]);
      if (!rc && r >= 0 &&
          (cudaEventRecord(e1, st) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
           cudaEventElapsedTime(&t[c][r], e0, e1) != cudaSuccess))
        rc = BPF_E_CUDA;
    }
  }
  double best_us = 0.0;
  for (int c = 0; !rc && c < 3; ++c) {
    std::sort(t[c], t[c] + kReps);
    const double med = 1e3 * t[c][kReps / 2];
    if (us) us[c] = med;
    if (c == 0 || med < best_us) {
      best_us = med;
      *best = counts[c];
    }
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  void* ps[] = {lw, lu, as, os, stats};
  for (void* q : ps)
    if (q) cudaFree(q);
  if (rc) {
    cudaGetLastError();
    *best = kBatchThreads;
  }
  return rc;
}

}  // namespace bpf

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
struct bpf_batch {
  bpf::ModelArgs model;
  int nf = 0, ld = 0, blocks = 0, max_n = 0, esz = 0, nobs = 0, bs = 0;
  int tiles = 0;               // 128-particle tiles over all filters (guided step)
  int rs_threads = 1024;       // threads per filter CTA of the resampler (autotuned at create)
  double rs_us[3] = {0.0, 0.0, 0.0};  // its tuning medians for 256, 512, 1024 threads
  bpf_proposal* prop = nullptr;  // learned proposal (bpf_batch_set_proposal), owned by the caller
  int* tile2f = nullptr;       // tile -> filter, allocated with the proposal
  // the PZ guided step's network outputs (ld entries), allocated with a PZ proposal
  float2* gO = nullptr;
  double ess_rel = 0.0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::vector<bpf::BatchFilter> filt;
  std::vector<double> theta;  // nf x BPF_MAX_THETA
  void* x[2] = {nullptr, nullptr};
  int cur = 0;
  double* lw = nullptr;
  int* as = nullptr;
  bpf::StepStats* stats = nullptr;
  bpf::LwPartial* partials = nullptr;
  unsigned* counters = nullptr;
  bpf::BatchFilter* filt_dev = nullptr;
  void* prm_dev = nullptr;
  int* blk2f = nullptr;
  int* order = nullptr;
  double* lu = nullptr;
  int* os = nullptr;
  void* y_dev = nullptr;
  size_t y_cap = 0;
  double* hist = nullptr;
  size_t hist_cap = 0;
  int step = 0;
  // bpf_filter_batch: the captured init + T steps, reused while T, t0, dt
  // and the buffers stay the same
  cudaGraphExec_t graph = nullptr;
  int g_T = 0;
  double g_t0 = 0.0, g_dt = 0.0;
  const void* g_y = nullptr;
  const void* g_hist = nullptr;
  // optional device timing: events around every step_device call's kernels
  // and around every filter run's graph launch
  bool timing = false;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  double timed_ms = 0.0;
  int timed_steps = 0;
};

namespace {

template <class P>
int upload_params(bpf_batch* b, const std::vector<P>& v) {
  BPF_TRY(cudaMemcpyAsync(b->prm_dev, v.data(), v.size() * sizeof(P), cudaMemcpyHostToDevice, b->stream));
  BPF_TRY(cudaStreamSynchronize(b->stream));  // v is a temporary
  return BPF_OK;
}

int batch_upload_params(bpf_batch* b) {
  const int nf = b->nf;
  const double* th = b->theta.data();
  if (b->model.kind == BPF_MODEL_L96) {
    std::vector<bpf::L96Params> v((size_t)nf);
    for (int f = 0; f < nf; ++f)
      v[f] = b->model.precision == BPF_F64 ? bpf::l96_params<double>(th + (size_t)f * BPF_MAX_THETA, b->model.h)
                                           : bpf::l96_params<float>(th + (size_t)f * BPF_MAX_THETA, b->model.h);
    return upload_params(b, v);
  }
  std::vector<bpf::PZParams> v((size_t)nf);
  for (int f = 0; f < nf; ++f)
    v[f] = bpf::pz_params<double>(th + (size_t)f * BPF_MAX_THETA, b->model.h, b->model.atoler, b->model.rtoler);
  return upload_params(b, v);
}

int batch_check_theta(const bpf_model_desc* m, const double* th) {
  if (m->kind == BPF_MODEL_L96) {
    if (!(th[1] >= 0.0) || !(th[2] > 0.0)) return BPF_E_INVALID;
  } else {
    if (!(th[5] >= 0.0) || !(th[6] > 0.0)) return BPF_E_INVALID;
  }
  return BPF_OK;
}

void batch_free(bpf_batch* b) {
  if (b->graph) cudaGraphExecDestroy(b->graph);
  for (cudaEvent_t e : b->ev)
    if (e) cudaEventDestroy(e);
  void* ptrs[] = {b->x[0], b->x[1], b->lw, b->as, b->stats, b->partials, b->counters, b->filt_dev,
                  b->prm_dev, b->blk2f, b->order, b->lu, b->os, b->y_dev, b->hist, b->tile2f,
                  b->gO};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (b->own_stream && b->stream) cudaStreamDestroy(b->stream);
}

template <class P>
int dalloc(P** p, size_t bytes) {
  if (cudaMalloc((void**)p, bytes) != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return BPF_E_NOMEM;
  }
  return BPF_OK;
}

int batch_enqueue_init(bpf_batch* b) {
  b->cur = 0;
  b->step = 0;
  return bpf::launch_batch_init(b->model, b->x[0], b->ld, b->lw, b->filt_dev, b->prm_dev, b->blk2f, b->blocks,
                                b->stats, b->ess_rel, b->stream);
}

int batch_enqueue_step(bpf_batch* b, double t1, double t2, const void* y_dev, double* hist, int k) {
  const int step = b->step + 1;
  int rc = bpf::launch_batch_resample(b->lw, b->as, b->filt_dev, b->order, b->nf, b->max_n, b->stats, b->lu,
                                      b->os, step, b->stream, b->rs_threads);
  if (rc) return rc;
  if (b->prop && y_dev && b->model.kind == BPF_MODEL_PZ) {
    // guided step of the PZ model: the proposal over the log-noise
    const double dt = bpf::proposal_dt(b->prop);
    if (std::fabs((t2 - t1) - dt) > 1e-9 * dt) return BPF_E_INVALID;
    bpf::BatchPZGuidedArgs g;
    g.x_in = (const double*)b->x[b->cur];
    g.x_out = (double*)b->x[b->cur ^ 1];
    g.ld = b->ld;
    g.as = b->as;
    g.lw = b->lw;
    g.y = (const double*)y_dev;
    g.t1 = t1;
    g.t2 = t2;
    g.step = step;
    g.filt = b->filt_dev;
    g.prms = (const bpf::PZParams*)b->prm_dev;
    g.blk2f = b->blk2f;
    g.blocks = b->blocks;
    g.stats = b->stats;
    g.partials = b->partials;
    g.counters = b->counters;
    g.hist = hist;
    g.nf = b->nf;
    g.k = k;
    g.O = b->gO;
    rc = bpf::launch_batch_pz_guided(*bpf::proposal_net(b->prop), g, b->stream);
  } else if (b->prop && y_dev) {
    // guided step: the learned proposal, trained for one interval
    const double dt = bpf::proposal_dt(b->prop);
    if (std::fabs((t2 - t1) - dt) > 1e-9 * dt) return BPF_E_INVALID;
    bpf::BatchGuidedArgs g;
    g.x_in = (const float*)b->x[b->cur];
    g.x_out = (float*)b->x[b->cur ^ 1];
    g.ld = b->ld;
    g.as = b->as;
    g.lw = b->lw;
    g.y = (const float*)y_dev;
    g.t1 = t1;
    g.t2 = t2;
    g.step = step;
    g.filt = b->filt_dev;
    g.prms = (const bpf::L96Params*)b->prm_dev;
    g.tile2f = b->tile2f;
    g.tiles = b->tiles;
    g.stats = b->stats;
    g.partials = b->partials;
    g.counters = b->counters;
    g.hist = hist;
    g.nf = b->nf;
    g.k = k;
    rc = bpf::launch_batch_guided(*bpf::proposal_net(b->prop), g, b->stream);
  } else {
    rc = bpf::launch_batch_transition(b->model, b->x[b->cur], b->x[b->cur ^ 1], b->ld, b->as, b->lw, y_dev, t1,
                                      t2, step, b->filt_dev, b->prm_dev, b->blk2f, b->blocks, b->stats,
                                      b->partials, b->counters, hist, b->nf, k, b->stream);
  }
  if (rc) return rc;
  b->cur ^= 1;
  b->step = step;
  return BPF_OK;
}

int batch_read(bpf_batch* b, double* ll, double* ess, int* status) {
  std::vector<bpf::StepStats> s((size_t)b->nf);
  BPF_TRY(cudaMemcpyAsync(s.data(), b->stats, s.size() * sizeof(bpf::StepStats), cudaMemcpyDeviceToHost,
                          b->stream));
  BPF_TRY(cudaStreamSynchronize(b->stream));
  int rc = BPF_OK;
  for (int f = 0; f < b->nf; ++f) {
    if (ll) ll[f] = s[f].status == BPF_OK ? s[f].ll : -INFINITY;
    if (ess) ess[f] = s[f].ess;
    if (status) status[f] = s[f].status;
    if (s[f].status != BPF_OK && rc == BPF_OK) rc = s[f].status;
  }
  return rc;
}

}  // namespace

extern "C" {

int bpf_batch_create(const bpf_model_desc* model, int nfilters, const bpf_batch_filter* filters, double ess_rel,
                     void* stream, bpf_batch** out) {
  if (!out) return BPF_E_INVALID;
  *out = nullptr;
  if (!model || !filters || nfilters <= 0 || !(ess_rel >= 0.0 && ess_rel <= 1.0)) return BPF_E_INVALID;
  if (model->kind == BPF_MODEL_L96) {
    const int ok_dims[] = {4, 8, 16, 32, 40};
    bool ok = false;
    for (int d : ok_dims) ok |= (model->dim == d);
    if (!ok || model->integrator != BPF_ODE_RK4 || !(model->h > 0.0)) return BPF_E_INVALID;
    if (model->precision != BPF_F32 && model->precision != BPF_F64) return BPF_E_INVALID;
  } else if (model->kind == BPF_MODEL_PZ) {
    if (model->dim != 2 || model->integrator != BPF_ODE_RK43 || model->precision != BPF_F64) return BPF_E_INVALID;
    if (!(model->h > 0.0) || !(model->atoler > 0.0) || !(model->rtoler >= 0.0)) return BPF_E_INVALID;
  } else {
    return BPF_E_INVALID;
  }
  for (int f = 0; f < nfilters; ++f) {
    const bpf_batch_filter& bf = filters[f];
    if (bf.nparticles <= 0 || bf.nparticles > BPF_BATCH_MAX_PARTICLES) return BPF_E_INVALID;
    if (bf.resampler < BPF_RESAMPLER_SYSTEMATIC || bf.resampler > BPF_RESAMPLER_METROPOLIS) return BPF_E_INVALID;
    if (bf.metropolis_steps < 0) return BPF_E_INVALID;
    if (batch_check_theta(model, bf.theta)) return BPF_E_INVALID;
  }
  bpf_batch* b = new (std::nothrow) bpf_batch();
  if (!b) return BPF_E_NOMEM;
  b->model.kind = model->kind;
  b->model.dim = model->dim;
  b->model.precision = model->precision;
  b->model.integrator = model->integrator;
  b->model.h = model->h;
  b->model.atoler = model->atoler;
  b->model.rtoler = model->rtoler;
  for (int i = 0; i < BPF_MAX_THETA; ++i) b->model.theta[i] = model->theta[i];
  b->nf = nfilters;
  b->ess_rel = ess_rel;
  b->esz = model->precision == BPF_F64 ? 8 : 4;
  b->nobs = model->kind == BPF_MODEL_L96 ? model->dim : 1;
  b->bs = model->kind == BPF_MODEL_L96 ? bpf::kL96Block : bpf::kPZBlock;
  b->filt.resize((size_t)nfilters);
  b->theta.resize((size_t)nfilters * BPF_MAX_THETA);
  std::vector<int> blk2f;
  int off = 0;
  for (int f = 0; f < nfilters; ++f) {
    const bpf_batch_filter& bf = filters[f];
    bpf::BatchFilter& d = b->filt[f];
    d.n = bf.nparticles;
    d.off = off;
    d.block0 = off / b->bs;
    d.nblocks = (bf.nparticles + b->bs - 1) / b->bs;
    d.resampler = bf.resampler;
    d.B = bf.metropolis_steps;
    d.seed = bf.seed;
    d.tile0 = b->tiles;
    d.ntiles = (bf.nparticles + 127) / 128;
    b->tiles += d.ntiles;
    for (int i = 0; i < BPF_MAX_THETA; ++i) b->theta[(size_t)f * BPF_MAX_THETA + i] = bf.theta[i];
    for (int k = 0; k < d.nblocks; ++k) blk2f.push_back(f);
    off += d.nblocks * b->bs;
    b->max_n = std::max(b->max_n, d.n);
  }
  b->ld = off;
  b->blocks = (int)blk2f.size();
  // largest filters resample first
  std::vector<int> order((size_t)nfilters);
  for (int f = 0; f < nfilters; ++f) order[f] = f;
  std::stable_sort(order.begin(), order.end(), [&](int i, int j) { return b->filt[i].n > b->filt[j].n; });

  int rc = BPF_OK;
  if (stream) {
    b->stream = (cudaStream_t)stream;
  } else {
    // graphs cannot be captured on the legacy default stream; a blocking
    // stream stays ordered with it
    if (cudaStreamCreate(&b->stream) != cudaSuccess) rc = BPF_E_CUDA;
    b->own_stream = rc == BPF_OK;
  }
  const size_t L = (size_t)b->ld;
  const size_t xb = (size_t)b->model.dim * L * b->esz;
  const size_t prm_b = b->model.kind == BPF_MODEL_L96 ? sizeof(bpf::L96Params) : sizeof(bpf::PZParams);
  if (!rc) rc = dalloc(&b->x[0], xb);
  if (!rc) rc = dalloc(&b->x[1], xb);
  if (!rc) rc = dalloc(&b->lw, L * sizeof(double));
  if (!rc) rc = dalloc(&b->as, L * sizeof(int));
  if (!rc) rc = dalloc(&b->stats, (size_t)nfilters * sizeof(bpf::StepStats));
  if (!rc) rc = dalloc(&b->partials, (size_t)b->blocks * sizeof(bpf::LwPartial));
  if (!rc) rc = dalloc(&b->counters, (size_t)nfilters * sizeof(unsigned));
  if (!rc) rc = dalloc(&b->filt_dev, (size_t)nfilters * sizeof(bpf::BatchFilter));
  if (!rc) rc = dalloc(&b->prm_dev, (size_t)nfilters * prm_b);
  if (!rc) rc = dalloc(&b->blk2f, (size_t)b->blocks * sizeof(int));
  if (!rc) rc = dalloc(&b->order, (size_t)nfilters * sizeof(int));
  if (!rc) rc = dalloc(&b->lu, L * sizeof(double));
  if (!rc) rc = dalloc(&b->os, L * sizeof(int));
  if (!rc && (cudaMemsetAsync(b->counters, 0, (size_t)nfilters * sizeof(unsigned), b->stream) != cudaSuccess ||
              cudaMemsetAsync(b->as, 0, L * sizeof(int), b->stream) != cudaSuccess ||
              cudaMemcpyAsync(b->filt_dev, b->filt.data(), b->filt.size() * sizeof(bpf::BatchFilter),
                              cudaMemcpyHostToDevice, b->stream) != cudaSuccess ||
              cudaMemcpyAsync(b->blk2f, blk2f.data(), blk2f.size() * sizeof(int), cudaMemcpyHostToDevice,
                              b->stream) != cudaSuccess ||
              cudaMemcpyAsync(b->order, order.data(), order.size() * sizeof(int), cudaMemcpyHostToDevice,
                              b->stream) != cudaSuccess ||
              cudaStreamSynchronize(b->stream) != cudaSuccess))
    rc = BPF_E_CUDA;
  if (!rc) rc = bpf::configure_batch_resample(b->max_n);
  if (!rc) rc = bpf::tune_batch_resample(b->filt_dev, b->order, b->nf, b->max_n, b->ld, b->stream, &b->rs_threads,
                                         b->rs_us);
  if (!rc) rc = batch_upload_params(b);
  if (!rc) rc = batch_enqueue_init(b);
  if (rc) {
    batch_free(b);
    delete b;
    return rc;
  }
  *out = b;
  return BPF_OK;
}

int bpf_batch_destroy(bpf_batch* b) {
  if (!b) return BPF_OK;
  cudaStreamSynchronize(b->stream);
  batch_free(b);
  delete b;
  return BPF_OK;
}

int bpf_batch_init(bpf_batch* b) {
  if (!b) return BPF_E_INVALID;
  return batch_enqueue_init(b);
}

int bpf_batch_set_theta(bpf_batch* b, const double* theta) {
  if (!b || !theta) return BPF_E_INVALID;
  bpf_model_desc m{};
  m.kind = b->model.kind;
  for (int f = 0; f < b->nf; ++f)
    if (batch_check_theta(&m, theta + (size_t)f * BPF_MAX_THETA)) return BPF_E_INVALID;
  std::copy(theta, theta + (size_t)b->nf * BPF_MAX_THETA, b->theta.begin());
  return batch_upload_params(b);
}

// events around enqueued work; the elapsed time is collected at the next
// synchronising read (bpf_batch_timing_read)
static int batch_timing_begin(bpf_batch* b) {
  if (b->timing) BPF_TRY(cudaEventRecord(b->ev[0], b->stream));
  return BPF_OK;
}

static int batch_timing_end(bpf_batch* b, int steps) {
  if (!b->timing) return BPF_OK;
  BPF_TRY(cudaEventRecord(b->ev[1], b->stream));
  BPF_TRY(cudaEventSynchronize(b->ev[1]));
  float ms = 0.0f;
  BPF_TRY(cudaEventElapsedTime(&ms, b->ev[0], b->ev[1]));
  b->timed_ms += ms;
  b->timed_steps += steps;
  return BPF_OK;
}

int bpf_batch_set_proposal(bpf_batch* b, bpf_proposal* p) {
  if (!b) return BPF_E_INVALID;
  if (p && b->model.kind == BPF_MODEL_PZ) {
    // the PZ proposal (one log-noise from three inputs) and its outputs
    const bpf::ProposalNet& net = *bpf::proposal_net(p);
    if (net.dim != 1 || net.din != 3 || net.hidden != bpf::kProposalHidden) return BPF_E_INVALID;
    if (!b->gO) {
      int rc = dalloc(&b->gO, (size_t)b->ld * sizeof(float2));
      if (rc) return rc;
    }
  } else if (p) {
    if (b->model.kind != BPF_MODEL_L96 || b->model.dim != 40 || b->model.precision != BPF_F32) return BPF_E_INVALID;
    const bpf::ProposalNet& net = *bpf::proposal_net(p);
    if (net.dim != b->model.dim || net.hidden != bpf::kProposalHidden) return BPF_E_INVALID;
    if (!b->tile2f) {
      std::vector<int> t2f((size_t)b->tiles);
      for (int f = 0; f < b->nf; ++f)
        for (int t = 0; t < b->filt[f].ntiles; ++t) t2f[(size_t)b->filt[f].tile0 + t] = f;
      int rc = dalloc(&b->tile2f, t2f.size() * sizeof(int));
      if (rc) return rc;
      BPF_TRY(cudaMemcpyAsync(b->tile2f, t2f.data(), t2f.size() * sizeof(int), cudaMemcpyHostToDevice, b->stream));
      BPF_TRY(cudaStreamSynchronize(b->stream));  // t2f is a temporary
    }
  }
  if (p != b->prop && b->graph) {
    // the captured steps launch the other step kernel
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  b->prop = p;
  return BPF_OK;
}

int bpf_batch_resample_threads(bpf_batch* b, int threads, int* current, double* tuned_us) {
  if (!b) return BPF_E_INVALID;
  if (threads != 0) {
    if (threads != 256 && threads != 512 && threads != 1024) return BPF_E_INVALID;
    if (threads != b->rs_threads && b->graph) {
      cudaGraphExecDestroy(b->graph);  // the captured steps launch the other count
      b->graph = nullptr;
    }
    b->rs_threads = threads;
  }
  if (current) *current = b->rs_threads;
  if (tuned_us)
    for (int c = 0; c < 3; ++c) tuned_us[c] = b->rs_us[c];
  return BPF_OK;
}

int bpf_batch_set_seeds(bpf_batch* b, const uint64_t* seeds) {
  if (!b || !seeds) return BPF_E_INVALID;
  for (int f = 0; f < b->nf; ++f) b->filt[f].seed = seeds[f];
  BPF_TRY(cudaMemcpyAsync(b->filt_dev, b->filt.data(), b->filt.size() * sizeof(bpf::BatchFilter),
                          cudaMemcpyHostToDevice, b->stream));
  BPF_TRY(cudaStreamSynchronize(b->stream));
  return BPF_OK;
}

int bpf_batch_step_device(bpf_batch* b, double t1, double t2, const void* y_device) {
  if (!b || !(t1 < t2)) return BPF_E_INVALID;
  int rc = batch_timing_begin(b);
  if (!rc) rc = batch_enqueue_step(b, t1, t2, y_device, nullptr, 0);
  if (!rc) rc = batch_timing_end(b, 1);
  return rc;
}

int bpf_batch_timing_enable(bpf_batch* b, int enable) {
  if (!b) return BPF_E_INVALID;
  if (enable)
    for (cudaEvent_t& e : b->ev)
      if (!e) BPF_TRY(cudaEventCreate(&e));
  b->timing = enable != 0;
  return BPF_OK;
}

int bpf_batch_timing_read(bpf_batch* b, int reset, double* ms, int* steps) {
  if (!b) return BPF_E_INVALID;
  if (ms) *ms = b->timed_ms;
  if (steps) *steps = b->timed_steps;
  if (reset) { b->timed_ms = 0.0; b->timed_steps = 0; }
  return BPF_OK;
}

int bpf_batch_stats(bpf_batch* b, double* log_likelihoods, double* ess, int* status) {
  if (!b) return BPF_E_INVALID;
  return batch_read(b, log_likelihoods, ess, status);
}

int bpf_batch_state_ptrs(bpf_batch* b, void** x, double** lw, int** as, int* ld, int* offsets) {
  if (!b) return BPF_E_INVALID;
  if (x) *x = b->x[b->cur];
  if (lw) *lw = b->lw;
  if (as) *as = b->as;
  if (ld) *ld = b->ld;
  if (offsets)
    for (int f = 0; f < b->nf; ++f) offsets[f] = b->filt[f].off;
  return BPF_OK;
}

int bpf_filter_batch(bpf_batch* b, int T, double t0, double dt, const void* y, double* log_likelihoods,
                     double* log_increments, double* ess, int* status) {
  if (!b || T <= 0 || !(dt > 0.0) || !y) return BPF_E_INVALID;
  const size_t step_b = (size_t)b->nf * b->nobs * b->esz;
  const size_t yb = (size_t)T * step_b;
  if (yb > b->y_cap) {
    if (b->y_dev) cudaFree(b->y_dev);
    b->y_dev = nullptr;
    b->y_cap = 0;
    int rc = dalloc(&b->y_dev, yb);
    if (rc) return rc;
    b->y_cap = yb;
  }
  const size_t hb = (size_t)3 * T * b->nf * sizeof(double);
  if (hb > b->hist_cap) {
    if (b->hist) cudaFree(b->hist);
    b->hist = nullptr;
    b->hist_cap = 0;
    int rc = dalloc(&b->hist, hb);
    if (rc) return rc;
    b->hist_cap = hb;
  }
  BPF_TRY(cudaMemcpyAsync(b->y_dev, y, yb, cudaMemcpyHostToDevice, b->stream));
  const bool reuse = b->graph && b->g_T == T && b->g_t0 == t0 && b->g_dt == dt && b->g_y == b->y_dev &&
                     b->g_hist == b->hist;
  if (!reuse) {
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
    // init + T steps, captured once: Filter::filter (share/src/bi/filter/Filter.hpp:58-70)
    BPF_TRY(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    int rc = batch_enqueue_init(b);
    for (int k = 1; !rc && k <= T; ++k)
      rc = batch_enqueue_step(b, t0 + (k - 1) * dt, t0 + k * dt, (const char*)b->y_dev + (size_t)(k - 1) * step_b,
                              b->hist, k - 1);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (e != cudaSuccess) { bpf_set_last_cuda_error(e); return BPF_E_CUDA; }
    e = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) { b->graph = nullptr; bpf_set_last_cuda_error(e); return BPF_E_CUDA; }
    b->g_T = T; b->g_t0 = t0; b->g_dt = dt; b->g_y = b->y_dev; b->g_hist = b->hist;
  }
  int rc = batch_timing_begin(b);
  if (rc) return rc;
  BPF_TRY(cudaGraphLaunch(b->graph, b->stream));
  rc = batch_timing_end(b, T);
  if (rc) return rc;
  // the host-side state the captured steps advanced
  b->cur = T & 1;
  b->step = T;
  if (log_increments || ess) {
    std::vector<double> h((size_t)3 * T * b->nf);
    BPF_TRY(cudaMemcpyAsync(h.data(), b->hist, hb, cudaMemcpyDeviceToHost, b->stream));
    BPF_TRY(cudaStreamSynchronize(b->stream));
    for (int k = 0; k < T; ++k)
      for (int f = 0; f < b->nf; ++f) {
        const double* r = h.data() + 3 * ((size_t)k * b->nf + f);
        if (log_increments) log_increments[(size_t)k * b->nf + f] = r[0];
        if (ess) ess[(size_t)k * b->nf + f] = r[1];
      }
  }
  // BootstrapPF::term (share/src/bi/filter/BootstrapPF.hpp:192-196):
  // logsumexp(lw) - log N is the last correct's lW, which each filter's
  // finalising block already formed over the same log-weights
  return batch_read(b, log_likelihoods, nullptr, status);
}

}  // extern "C"
