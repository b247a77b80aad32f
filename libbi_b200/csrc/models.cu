// Model transition + observation kernels of the single bootstrap particle
// filter (the per-particle bodies are in model_body.cuh).
//
// One thread advances one particle through one observation interval, fusing
// the ancestor gather (State::gather -> gather_rows,
// share/src/bi/state/State.hpp:907-909), the noise draw, the ODE, the
// deterministic update, the observation log-density and the block partial of
// the log-weight reduction (Resampler::reduce -> ess_reduce); the last block
// finalises the step statistics.  The state lives in registers for the whole
// interval; HBM sees one read and one write of the particle's state and
// log-weight.
#include "internal.cuh"
#include "reduce.cuh"
#include "model_body.cuh"

#include <cmath>

namespace bpf {

template <class T, int D>
__global__ void __launch_bounds__(kL96Block, l96_min_blocks(sizeof(T)))
k_l96_transition(const T* __restrict__ x_in, T* __restrict__ x_out, int ld, int n,
                 int* __restrict__ as, double* __restrict__ lw, const T* __restrict__ y,
                 double t1d, double t2d, uint64_t seed, int step, L96Params prm,
                 StepStats* st, LwPartial* partials, unsigned* counter, uint64_t mask) {
  // state staged here for the rolled noise/observation epilogue
  __shared__ T sx[D][kL96Block];
  pdl_wait();  // the resampler's ancestors and statistics
  const int p = blockIdx.x * kL96Block + threadIdx.x;
  const int resampled = st->resample;
  const bool ok = st->status == BPF_OK;
  LwPartial part = lw_empty();
  if (ok && p < n) {
    const int src = resampled ? as[p] : p;
    T x0[D];
#pragma unroll
    for (int i = 0; i < D; ++i) x0[i] = __ldg(x_in + (size_t)i * ld + src);
    l96_rk4<T, D>(x0, t1d, t2d, (T)prm.F, (T)prm.h);
#pragma unroll
    for (int i = 0; i < D; ++i) sx[i][threadIdx.x] = x0[i];
    // st->ll is read after the ODE (not held across it); the last block
    // rewrites it only after every block has arrived
    const double l = l96_noise_obs<T, D>(sx, x_out, (size_t)ld, p, y, seed, (uint32_t)p, step, prm,
                                         resampled ? st->ll : lw[p], mask);
    lw[p] = l;
    if (resampled) as[p] = src;
    lw_push(part, l);
  }
  pdl_trigger();
  transition_reduce_tail(part, partials, blockIdx.x, 0, gridDim.x, counter, n, st, ok, resampled, y != nullptr);
}

template <class T>
__global__ void __launch_bounds__(kPZBlock)
k_pz_transition(const T* __restrict__ x_in, T* __restrict__ x_out, int ld, int n,
                int* __restrict__ as, double* __restrict__ lw, const T* __restrict__ y,
                double t1d, double t2d, uint64_t seed, int step, PZParams prm,
                StepStats* st, LwPartial* partials, unsigned* counter, uint64_t mask) {
  pdl_wait();  // the resampler's ancestors and statistics
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  const int resampled = st->resample;
  const bool ok = st->status == BPF_OK;
  LwPartial part = lw_empty();
  if (p < n && ok) {
    const int src = resampled ? as[p] : p;
    T P = __ldg(x_in + src), Z = __ldg(x_in + (size_t)ld + src);
    const T alpha = pz_alpha<T>(seed, (uint32_t)p, step, prm);
    pz_advance<T>(P, Z, alpha, t1d, t2d, prm);
    double l = resampled ? st->ll : lw[p];
    if (y && (mask & 1ull)) l += pz_obs_term<T>(P, __ldg(y), prm);
    x_out[p] = P;
    x_out[(size_t)ld + p] = Z;
    lw[p] = l;
    if (resampled) as[p] = src;
    lw_push(part, l);
  }
  pdl_trigger();
  transition_reduce_tail(part, partials, blockIdx.x, 0, gridDim.x, counter, n, st, ok, resampled, y != nullptr);
}

// ---------------------------------------------------------------------------
// initial draws (Simulator::init -> Model::initialSamples)
// ---------------------------------------------------------------------------
template <class T>
__global__ void k_l96_init(T* x, int ld, int n, int D, double* lw, uint64_t seed, double mean, double sd) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  for (int b = 0; b < (D + 3) / 4; ++b) {
    bpf_u32x4 r = bpf_draw(seed, (uint32_t)p, 0u, (uint32_t)b, BPF_RNG_INIT);
    T z[4];
    box_muller(r.v[0], r.v[1], z[0], z[1]);
    box_muller(r.v[2], r.v[3], z[2], z[3]);
    for (int j = 0; j < 4; ++j) {
      int i = 4 * b + j;
      if (i < D) x[(size_t)i * ld + p] = Prec<T>::fma_((T)sd, z[j], (T)mean);
    }
  }
  lw[p] = 0.0;
}

template <class T>
__global__ void k_pz_init(T* x, int ld, int n, double* lw, uint64_t seed, PZParams prm) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  bpf_u32x4 r = bpf_draw(seed, (uint32_t)p, 0u, 0u, BPF_RNG_INIT);
  T z0, z1;
  box_muller(r.v[0], r.v[1], z0, z1);
  x[p] = Prec<T>::exp_(Prec<T>::fma_((T)prm.p0_sigma, z0, (T)prm.p0_mu));
  x[(size_t)ld + p] = Prec<T>::exp_(Prec<T>::fma_((T)prm.z0_sigma, z1, (T)prm.z0_mu));
  lw[p] = 0.0;
}

__global__ void k_stats_init(StepStats* st, int n, double ess_rel) {
  StepStats z{};
  z.mx = 0.0; z.s1 = 0.0; z.s2 = 0.0; z.ess = 0.0; z.lW = 0.0; z.ll = 0.0; z.inc = 0.0;
  z.resample = 0; z.resampled = 0; z.status = BPF_OK; z.step = 0; z.ess_rel = ess_rel; z.n = n;
  *st = z;
}

// the transitions are launched as programmatic dependents of the resampler
// before them (measured on B200 at N = 65536: 49.1 against 50.8 us per
// filter step), so that their blocks are scheduled while it finishes
#define L96_CASE(DD)                                                                                   \
  case DD:                                                                                             \
    BPF_TRY(launch_pdl(k_l96_transition<T, DD>, dim3(blocks), dim3(kL96Block), 0, st, (const T*)a.x_in,     \
                       (T*)a.x_out, a.ld, a.n, (int*)a.as, a.lw, (const T*)a.y, a.t1, a.t2, a.seed, a.step,   \
                       prm, a.stats, a.partials, a.counter, a.obs_mask));                               \
    break;

template <class T>
static int transition_t(const ModelArgs& m, const TransitionArgs& a, cudaStream_t st) {
  if (m.kind == BPF_MODEL_L96) {
    // one particle per thread: 64-thread blocks spread evenly over the SMs
    const int blocks = (a.n + kL96Block - 1) / kL96Block;
    if (blocks > a.max_partials) return BPF_E_INVALID;
    L96Params prm = l96_params<T>(m.theta, m.h);
    switch (m.dim) {
      L96_CASE(4)
      L96_CASE(8)
      L96_CASE(16)
      L96_CASE(32)
      L96_CASE(40)
      default:
        return BPF_E_INVALID;
    }
  } else if (m.kind == BPF_MODEL_PZ) {
    const int blocks = (a.n + kPZBlock - 1) / kPZBlock;
    if (blocks > a.max_partials) return BPF_E_INVALID;
    PZParams prm = pz_params<T>(m.theta, m.h, m.atoler, m.rtoler);
    BPF_TRY(launch_pdl(k_pz_transition<T>, dim3(blocks), dim3(kPZBlock), 0, st, (const T*)a.x_in, (T*)a.x_out,
                       a.ld, a.n, (int*)a.as, a.lw, (const T*)a.y, a.t1, a.t2, a.seed, a.step, prm, a.stats,
                       a.partials, a.counter, a.obs_mask));
  } else {
    return BPF_E_INVALID;
  }
  BPF_TRY(cudaGetLastError());
  return BPF_OK;
}

int launch_transition(const ModelArgs& m, const TransitionArgs& a, cudaStream_t st) {
  return m.precision == BPF_F64 ? transition_t<double>(m, a, st) : transition_t<float>(m, a, st);
}

template <class T>
static int init_t(const ModelArgs& m, void* x, int ld, int n, double* lw, uint64_t seed, cudaStream_t st) {
  const int blocks = (n + 127) / 128;
  if (m.kind == BPF_MODEL_L96) {
    k_l96_init<T><<<blocks, 128, 0, st>>>((T*)x, ld, n, m.dim, lw, seed, m.theta[3], m.theta[4]);
  } else {
    k_pz_init<T><<<blocks, 128, 0, st>>>((T*)x, ld, n, lw, seed, pz_params<T>(m.theta, m.h, m.atoler, m.rtoler));
  }
  BPF_TRY(cudaGetLastError());
  return BPF_OK;
}

int launch_stats_init(StepStats* stats, int n, double ess_rel, cudaStream_t st) {
  k_stats_init<<<1, 1, 0, st>>>(stats, n, ess_rel);
  BPF_TRY(cudaGetLastError());
  return BPF_OK;
}

int launch_init(const ModelArgs& m, void* x, int ld, int n, double* lw, uint64_t seed, StepStats* stats,
                double ess_rel, cudaStream_t st) {
  int rc = m.precision == BPF_F64 ? init_t<double>(m, x, ld, n, lw, seed, st)
                                  : init_t<float>(m, x, ld, n, lw, seed, st);
  if (rc) return rc;
  k_stats_init<<<1, 1, 0, st>>>(stats, n, ess_rel);
  BPF_TRY(cudaGetLastError());
  return BPF_OK;
}

}  // namespace bpf
