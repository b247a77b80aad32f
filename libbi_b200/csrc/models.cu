// Model transition + observation kernels of the bootstrap particle filter.
//
// One thread advances one particle through one observation interval, fusing
// what the reference runs as separate passes over the State:
//   ancestor gather  State::gather -> gather_rows (share/src/bi/state/State.hpp:907-909)
//   noise draw       StaticSampler::samples (share/src/bi/host/updater/StaticSamplerHost.hpp:44-65)
//   ODE              RK4IntegratorHost::update (share/src/bi/host/ode/RK4IntegratorHost.hpp:43-100)
//                    RK43IntegratorHost::update (share/src/bi/host/ode/RK43IntegratorHost.hpp:48-144)
//   x <- x + eta     DynamicUpdater (share/tt/cpp/block/eval_.hpp.tt:78-88)
//   log-density      SparseStaticLogDensity::logDensities
//                    (share/src/bi/host/updater/SparseStaticLogDensityHost.hpp:48-68,
//                     share/tt/cpp/action/gaussian.hpp.tt:48-73)
//   reduction        Resampler::reduce -> ess_reduce (block partials + last block)
// The state lives in registers for the whole interval; HBM sees one read and
// one write of the particle's state and log-weight.
//
// Floating-point expression order: where the reference writes a*b + c the
// kernels use fma(a, b, c), the form the reference's host code takes when
// compiled with FP contraction; the same order is restated in the oracle.
#include "internal.cuh"
#include "reduce.cuh"
#include "../../include/bpf_math.h"

#include <cmath>

namespace bpf {

// Arithmetic in the model precision T.  Products that feed sums are explicit
// fused multiply-adds and the elementary functions are the portable ones of
// bpf_math.h, so that a host build of the same expressions (the oracle)
// reproduces every bit.
template <class T> struct Prec;
template <> struct Prec<float> {
  __device__ static float fma_(float a, float b, float c) { return __fmaf_rn(a, b, c); }
  __device__ static float mul_(float a, float b) { return __fmul_rn(a, b); }
  __device__ static float add_(float a, float b) { return __fadd_rn(a, b); }
  __device__ static float log_(float x) { return bpf_logf(x); }
  __device__ static float exp_(float x) { return bpf_expf(x); }
};
template <> struct Prec<double> {
  __device__ static double fma_(double a, double b, double c) { return __fma_rn(a, b, c); }
  __device__ static double mul_(double a, double b) { return __dmul_rn(a, b); }
  __device__ static double add_(double a, double b) { return __dadd_rn(a, b); }
  __device__ static double log_(double x) { return bpf_log(x); }
  __device__ static double exp_(double x) { return bpf_exp(x); }
};

// Standard normal pair (bpf_normal_pair_f / _d of bpf_math.h): normals for
// component i come from Philox block i/4, words (i%4 & ~1, (i%4) | 1).
__device__ __forceinline__ void box_muller(uint32_t a, uint32_t b, float& z0, float& z1) {
  bpf_normal_pair_f(a, b, &z0, &z1);
}
__device__ __forceinline__ void box_muller(uint32_t a, uint32_t b, double& z0, double& z1) {
  bpf_normal_pair_d(a, b, &z0, &z1);
}

struct L96Params {
  double F, sigma_eta, sigma_y, h;
  double c_half_log_2pi;   // BI_HALF_LOG_TWO_PI in model precision
  double log_sigma_y;      // log(sigma_y) in model precision, host-computed
  double inv_sigma_y;      // 1/sigma_y when sigma_y is a power of two (exact), else 0
  double x0_mean, x0_std;
};

// ---------------------------------------------------------------------------
// Lorenz '96, RK4 (classic, fixed step, last step clipped to t2)
// ---------------------------------------------------------------------------
template <class T, int D>
__device__ __forceinline__ void l96_dfdt(const T (&x)[D], T (&k)[D], T F) {
#pragma unroll
  for (int i = 0; i < D; ++i) {
    // dx[i]/dt = (x[i+1] - x[i-2])*x[i-1] - x[i] + F
    T d = x[(i + 1) % D] - x[(i + D - 2) % D];
    k[i] = Prec<T>::fma_(d, x[(i + D - 1) % D], -x[i]) + F;
  }
}

// Blocks of 64 threads, at most 128 registers each: 8 blocks fit an SM, so
// N = 65536 particles (1024 blocks) run as a single wave on 148 SMs with 6 or
// 7 blocks on every SM.
constexpr int kL96Block = 64;

template <class T, int D>
__global__ void __launch_bounds__(kL96Block, (sizeof(T) == 4 && D <= 40 ? 8 : 4))
k_l96_transition(const T* __restrict__ x_in, T* __restrict__ x_out, int ld, int n,
                 int* __restrict__ as, double* __restrict__ lw, const T* __restrict__ y,
                 double t1d, double t2d, uint64_t seed, int step, L96Params prm,
                 StepStats* st, LwPartial* partials, unsigned* counter) {
  // state staged here for the rolled noise/observation epilogue
  __shared__ T sx[D][kL96Block];
  const int p = blockIdx.x * kL96Block + threadIdx.x;
  const int resampled = st->resample;
  const bool ok = st->status == BPF_OK;
  const T F = (T)prm.F, h0 = (T)prm.h;
  const double ll = st->ll;
  LwPartial part = lw_empty();
  if (ok && p < n) {
    const int src = resampled ? as[p] : p;
    T x0[D];
#pragma unroll
    for (int i = 0; i < D; ++i) x0[i] = __ldg(x_in + (size_t)i * ld + src);

    // RK4IntegratorHost::update (RK4IntegratorHost.hpp:63-97) with the stages
    // of RK4Stage (share/src/bi/ode/RK4Stage.hpp:128-178):
    // a21 = a32 = 1/2, a43 = 1 (exact scalings folded into h), b = 1/6,1/3,1/3,1/6
    const T b1 = (T)(1.0 / 6.0), b2 = (T)(1.0 / 3.0), b3 = (T)(1.0 / 3.0), b4 = (T)(1.0 / 6.0);
    const T t2 = (T)t2d;
    T t = (T)t1d, h = h0;
    while (t < t2) {
      if (Prec<T>::fma_((T)1.01, h, t) - t2 > (T)0) {
        h = t2 - t;
        if (h <= (T)0) { t = t2; break; }
      }
      const T hh = (T)0.5 * h;
      T xs[D], k[D], acc[D];
      l96_dfdt<T, D>(x0, k, F);
#pragma unroll
      for (int i = 0; i < D; ++i) { acc[i] = b1 * k[i]; xs[i] = Prec<T>::fma_(hh, k[i], x0[i]); }
      l96_dfdt<T, D>(xs, k, F);
#pragma unroll
      for (int i = 0; i < D; ++i) { acc[i] = Prec<T>::fma_(b2, k[i], acc[i]); xs[i] = Prec<T>::fma_(hh, k[i], x0[i]); }
      l96_dfdt<T, D>(xs, k, F);
#pragma unroll
      for (int i = 0; i < D; ++i) { acc[i] = Prec<T>::fma_(b3, k[i], acc[i]); xs[i] = Prec<T>::fma_(h, k[i], x0[i]); }
      l96_dfdt<T, D>(xs, k, F);
#pragma unroll
      for (int i = 0; i < D; ++i) { acc[i] = Prec<T>::fma_(b4, k[i], acc[i]); x0[i] = Prec<T>::fma_(h, acc[i], x0[i]); }
      t += h;
    }
#pragma unroll
    for (int i = 0; i < D; ++i) sx[i][threadIdx.x] = x0[i];

    // eta[i] ~ gaussian(0, sigma_eta); x[i] <- x[i] + eta[i]; then
    // lp += -0.5*((y - x)/sigma)^2 - BI_HALF_LOG_TWO_PI - log(sigma),
    // four components per Philox block, in component order
    const T se = (T)prm.sigma_eta;
    const T sy = (T)prm.sigma_y, isy = (T)prm.inv_sigma_y;
    const T c2 = (T)prm.c_half_log_2pi, ls = (T)prm.log_sigma_y;
    double l = resampled ? ll : lw[p];
#pragma unroll 1
    for (int b = 0; b < (D + 3) / 4; ++b) {
      bpf_u32x4 r = bpf_draw(seed, (uint32_t)p, (uint32_t)step, (uint32_t)b, BPF_RNG_NOISE);
      T z[4];
      box_muller(r.v[0], r.v[1], z[0], z[1]);
      box_muller(r.v[2], r.v[3], z[2], z[3]);
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int i = 4 * b + j;
        if (i < D) {
          const T xi = Prec<T>::add_(sx[i][threadIdx.x], Prec<T>::mul_(se, z[j]));
          x_out[(size_t)i * ld + p] = xi;
          if (y) {
            T dz = __ldg(y + i) - xi;
            dz = isy != (T)0 ? dz * isy : dz / sy;
            T term = Prec<T>::fma_((T)-0.5, dz * dz, -c2) - ls;
            l += (double)term;
          }
        }
      }
    }
    lw[p] = l;
    if (resampled) as[p] = src;
    lw_push(part, l);
  }
  part = block_combine(part);
  if (threadIdx.x == 0) partials[blockIdx.x] = part;
  __shared__ bool am_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) am_last = atomicAdd(counter, 1u) == gridDim.x - 1;
  __syncthreads();
  if (am_last) {
    __threadfence();
    if (ok) {
      finalize_partials(partials, gridDim.x, n, st, kFinalizeStep, y != nullptr);
      if (threadIdx.x == 0) st->resampled = resampled;
    }
    if (threadIdx.x == 0) *counter = 0;
  }
}

// ---------------------------------------------------------------------------
// PZ, RK4(3)5[2R+]C low-storage adaptive (Kennedy et al. 2000)
// ---------------------------------------------------------------------------
struct PZParams {
  double c, e, m, q, mu, sigma, sigma_y;
  double p0_mu, p0_sigma, z0_mu, z0_sigma;
  double h0, atoler, rtoler;
  double c_half_log_2pi, log_sigma_y, inv_sigma_y;
  // step-size control, share/src/bi/host/ode/IntegratorConstants.cpp:45-87
  double safe, facl, facr, beta, logsafe, expo;
  int nsteps;
};

template <class T>
__device__ __forceinline__ void pz_dfdt(T P, T Z, T alpha, T c, T e, T m, T q, T& dP, T& dZ) {
  // dP/dt = alpha*P - c*P*Z;  dZ/dt = e*c*P*Z - m*Z - q*Z*Z
  T cPZ = (c * P) * Z;
  dP = Prec<T>::fma_(alpha, P, -cPZ);
  T ecPZ = (e * c) * P * Z;
  dZ = Prec<T>::fma_(-q * Z, Z, Prec<T>::fma_(-m, Z, ecPZ));
}

template <class T>
__global__ void __launch_bounds__(128)
k_pz_transition(const T* __restrict__ x_in, T* __restrict__ x_out, int ld, int n,
                int* __restrict__ as, double* __restrict__ lw, const T* __restrict__ y,
                double t1d, double t2d, uint64_t seed, int step, PZParams prm,
                StepStats* st, LwPartial* partials, unsigned* counter) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  const int resampled = st->resample;
  const bool ok = st->status == BPF_OK;
  LwPartial part = lw_empty();
  if (p < n && ok) {
    const int src = resampled ? as[p] : p;
    T P = __ldg(x_in + src), Z = __ldg(x_in + (size_t)ld + src);

    // alpha ~ log_normal(mu, sigma): exp(gaussian(mu, sigma)) (gaussian.hpp.tt:37-43)
    bpf_u32x4 r = bpf_draw(seed, (uint32_t)p, (uint32_t)step, 0u, BPF_RNG_NOISE);
    T z0, z1;
    box_muller(r.v[0], r.v[1], z0, z1);
    const T alpha = Prec<T>::exp_(Prec<T>::fma_((T)prm.sigma, z0, (T)prm.mu));

    const T c = (T)prm.c, e = (T)prm.e, m = (T)prm.m, q = (T)prm.q;
    const T atol = (T)prm.atoler, rtol = (T)prm.rtoler;
    const T facl = (T)prm.facl, facr = (T)prm.facr, beta = (T)prm.beta;
    const T logsafe = (T)prm.logsafe, expo = (T)prm.expo;
    // RK43Stage coefficients (share/src/bi/ode/RK43Stage.hpp:172-227)
    const T a21 = (T)0.225022458725713, b1 = (T)0.0512293066403392, e1 = (T)-0.0859880154628801;
    // (the stage times c2..c5 are not needed: the PZ vector field is autonomous)
    const T a32 = (T)0.544043312951405, b2 = (T)0.380954825726402, e2c = (T)0.189074063397015;
    const T a43 = (T)0.144568243493995, b3 = (T)-0.373352596392383, e3 = (T)-0.144145875232852;
    const T a54 = (T)0.786664342198357, b4 = (T)0.592501285026362, e4 = (T)-0.0317933915175331;
    const T b5 = (T)0.34866717899928, e5 = (T)0.0728532188162504;

    const T t2 = (T)t2d;
    T t = (T)t1d, h = (T)prm.h0;
    T logfacold = Prec<T>::log_((T)1.0e-4);
    T oP = P, oZ = Z;     // old
    T r1P = P, r1Z = Z;   // r1 (stored state after stage 1, 3, 5)
    int nst = 0;
    // RK43IntegratorHost::update loop (RK43IntegratorHost.hpp:77-141)
    while (t < t2 && nst < prm.nsteps) {
      if (Prec<T>::fma_((T)1.01, h, t) - t2 > (T)0) {
        h = t2 - t;
        if (h <= (T)0) { t = t2; break; }
      }
      T r2P, r2Z, kP, kZ, errP, errZ, SP, SZ;
      // stage 1: r2 = f(S=r1)
      pz_dfdt<T>(r1P, r1Z, alpha, c, e, m, q, kP, kZ);
      errP = e1 * kP; errZ = e1 * kZ;
      r1P = Prec<T>::fma_(a21 * h, kP, r1P); r1Z = Prec<T>::fma_(a21 * h, kZ, r1Z);
      r2P = Prec<T>::fma_((b1 - a21) * h, kP, r1P); r2Z = Prec<T>::fma_((b1 - a21) * h, kZ, r1Z);
      SP = r1P; SZ = r1Z;
      // stage 2: r1 = f(S)
      pz_dfdt<T>(SP, SZ, alpha, c, e, m, q, kP, kZ);
      errP = Prec<T>::fma_(e2c, kP, errP); errZ = Prec<T>::fma_(e2c, kZ, errZ);
      r2P = Prec<T>::fma_(a32 * h, kP, r2P); r2Z = Prec<T>::fma_(a32 * h, kZ, r2Z);
      r1P = Prec<T>::fma_((b2 - a32) * h, kP, r2P); r1Z = Prec<T>::fma_((b2 - a32) * h, kZ, r2Z);
      SP = r2P; SZ = r2Z;
      // stage 3
      pz_dfdt<T>(SP, SZ, alpha, c, e, m, q, kP, kZ);
      errP = Prec<T>::fma_(e3, kP, errP); errZ = Prec<T>::fma_(e3, kZ, errZ);
      r1P = Prec<T>::fma_(a43 * h, kP, r1P); r1Z = Prec<T>::fma_(a43 * h, kZ, r1Z);
      r2P = Prec<T>::fma_((b3 - a43) * h, kP, r1P); r2Z = Prec<T>::fma_((b3 - a43) * h, kZ, r1Z);
      SP = r1P; SZ = r1Z;
      // stage 4
      pz_dfdt<T>(SP, SZ, alpha, c, e, m, q, kP, kZ);
      errP = Prec<T>::fma_(e4, kP, errP); errZ = Prec<T>::fma_(e4, kZ, errZ);
      r2P = Prec<T>::fma_(a54 * h, kP, r2P); r2Z = Prec<T>::fma_(a54 * h, kZ, r2Z);
      r1P = Prec<T>::fma_((b4 - a54) * h, kP, r2P); r1Z = Prec<T>::fma_((b4 - a54) * h, kZ, r2Z);
      SP = r2P; SZ = r2Z;
      // stage 5
      pz_dfdt<T>(SP, SZ, alpha, c, e, m, q, kP, kZ);
      errP = Prec<T>::fma_(e5, kP, errP); errZ = Prec<T>::fma_(e5, kZ, errZ);
      r1P = Prec<T>::fma_(b5 * h, kP, r1P); r1Z = Prec<T>::fma_(b5 * h, kZ, r1Z);

      // error norm, RK43IntegratorHost.hpp:106-111
      T eP = (errP * h) / Prec<T>::fma_(rtol, fmax(fabs(oP), fabs(r1P)), atol);
      T eZ = (errZ * h) / Prec<T>::fma_(rtol, fmax(fabs(oZ), fabs(r1Z)), atol);
      T e2 = Prec<T>::fma_(eZ, eZ, eP * eP) / (T)2;

      if (e2 <= (T)1) {
        t += h;
        if (t < t2) { oP = r1P; oZ = r1Z; }
      } else {
        r1P = oP; r1Z = oZ;
      }
      if (t < t2) {
        T logfac11 = Prec<T>::mul_(expo, Prec<T>::log_(e2));
        if (e2 > (T)1) {
          h = Prec<T>::mul_(h, fmax(facl, Prec<T>::exp_(logsafe - logfac11)));
        } else {
          T fac = Prec<T>::exp_(Prec<T>::fma_(beta, logfacold, logsafe) - logfac11);
          fac = fmin(facr, fmax(facl, fac));
          h = Prec<T>::mul_(h, fac);
          logfacold = Prec<T>::mul_((T)0.5, Prec<T>::log_(fmax(e2, (T)1.0e-8)));
        }
      }
      ++nst;
    }
    P = r1P; Z = r1Z;

    double l = resampled ? st->ll : lw[p];
    if (y) {
      // y ~ gaussian(log(P), sigma_y)
      T dz = __ldg(y) - Prec<T>::log_(P);
      const T isy = (T)prm.inv_sigma_y;
      dz = isy != (T)0 ? dz * isy : dz / (T)prm.sigma_y;
      T term = Prec<T>::fma_((T)-0.5, dz * dz, -(T)prm.c_half_log_2pi) - (T)prm.log_sigma_y;
      l += (double)term;
    }
    x_out[p] = P;
    x_out[(size_t)ld + p] = Z;
    lw[p] = l;
    if (resampled) as[p] = src;
    lw_push(part, l);
  }
  part = block_combine(part);
  if (threadIdx.x == 0) partials[blockIdx.x] = part;
  __shared__ bool am_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) am_last = atomicAdd(counter, 1u) == gridDim.x - 1;
  __syncthreads();
  if (am_last) {
    __threadfence();
    if (ok) {
      finalize_partials(partials, gridDim.x, n, st, kFinalizeStep, y != nullptr);
      if (threadIdx.x == 0) st->resampled = resampled;
    }
    if (threadIdx.x == 0) *counter = 0;
  }
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

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
static bool is_pow2(double v) {
  if (!(v > 0.0)) return false;
  int e;
  double m = frexp(v, &e);
  return m == 0.5;
}

template <class T>
static L96Params l96_params(const ModelArgs& m) {
  L96Params p;
  p.F = m.theta[0];
  p.sigma_eta = m.theta[1];
  p.sigma_y = m.theta[2];
  p.x0_mean = m.theta[3];
  p.x0_std = m.theta[4];
  p.h = m.h;
  p.c_half_log_2pi = (double)(T)0.91893853320467274178032973640562;
  p.log_sigma_y = (double)(T)std::log((T)m.theta[2]);
  p.inv_sigma_y = is_pow2(m.theta[2]) ? 1.0 / m.theta[2] : 0.0;
  return p;
}

template <class T>
static PZParams pz_params(const ModelArgs& m) {
  PZParams p;
  p.c = m.theta[0]; p.e = m.theta[1]; p.m = m.theta[2]; p.q = m.theta[3];
  p.mu = m.theta[4]; p.sigma = m.theta[5]; p.sigma_y = m.theta[6];
  p.p0_mu = m.theta[7]; p.p0_sigma = m.theta[8]; p.z0_mu = m.theta[9]; p.z0_sigma = m.theta[10];
  p.h0 = m.h; p.atoler = m.atoler; p.rtoler = m.rtoler;
  p.c_half_log_2pi = (double)(T)0.91893853320467274178032973640562;
  p.log_sigma_y = (double)(T)std::log((T)m.theta[6]);
  p.inv_sigma_y = is_pow2(m.theta[6]) ? 1.0 / m.theta[6] : 0.0;
  // h_ode_init defaults (share/src/bi/host/ode/IntegratorConstants.cpp:77-87)
  p.safe = 0.9; p.facl = 0.2; p.facr = 10.0; p.beta = 0.04; p.nsteps = 1000;
  // h_ode_set_safe / h_ode_set_beta (IntegratorConstants.cpp:45-60), in T
  p.logsafe = (double)(T)std::log((T)0.9);
  p.expo = (double)((T)0.5 * (T)std::fma(-(T)0.04, (T)0.75, (T)0.2));
  return p;
}

#define L96_CASE(DD)                                                                                   \
  case DD:                                                                                             \
    k_l96_transition<T, DD><<<blocks, kL96Block, 0, st>>>((const T*)a.x_in, (T*)a.x_out, a.ld, a.n,          \
        (int*)a.as, a.lw, (const T*)a.y, a.t1, a.t2, a.seed, a.step, prm, a.stats, a.partials, a.counter); \
    break;

template <class T>
static int transition_t(const ModelArgs& m, const TransitionArgs& a, cudaStream_t st) {
  if (m.kind == BPF_MODEL_L96) {
    // one particle per thread: 64-thread blocks spread evenly over the SMs
    const int blocks = (a.n + kL96Block - 1) / kL96Block;
    if (blocks > a.max_partials) return BPF_E_INVALID;
    L96Params prm = l96_params<T>(m);
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
    const int blocks = (a.n + 127) / 128;
    if (blocks > a.max_partials) return BPF_E_INVALID;
    PZParams prm = pz_params<T>(m);
    k_pz_transition<T><<<blocks, 128, 0, st>>>((const T*)a.x_in, (T*)a.x_out, a.ld, a.n, (int*)a.as, a.lw,
                                               (const T*)a.y, a.t1, a.t2, a.seed, a.step, prm, a.stats,
                                               a.partials, a.counter);
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
    k_pz_init<T><<<blocks, 128, 0, st>>>((T*)x, ld, n, lw, seed, pz_params<T>(m));
  }
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
