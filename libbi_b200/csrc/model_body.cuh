// Per-particle bodies of the two models, shared by the single-filter kernels
// (models.cu) and the batched kernels (batch.cu).
//
// One thread advances one particle through one observation interval, fusing
// what the reference runs as separate passes over the State:
//   noise draw       StaticSampler::samples (share/src/bi/host/updater/StaticSamplerHost.hpp:44-65)
//   ODE              RK4IntegratorHost::update (share/src/bi/host/ode/RK4IntegratorHost.hpp:43-100)
//                    RK43IntegratorHost::update (share/src/bi/host/ode/RK43IntegratorHost.hpp:48-144)
//   x <- x + eta     DynamicUpdater (share/tt/cpp/block/eval_.hpp.tt:78-88)
//   log-density      SparseStaticLogDensity::logDensities
//                    (share/src/bi/host/updater/SparseStaticLogDensityHost.hpp:48-68,
//                     share/tt/cpp/action/gaussian.hpp.tt:48-73)
//
// Floating-point expression order: where the reference writes a*b + c the
// bodies use fma(a, b, c), the form the reference's host code takes when
// compiled with FP contraction; the same order is restated in the oracle.
#pragma once
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

// Blocks of 128 threads, at most 128 registers each (FP32): 4 blocks fit an
// SM, so N = 65536 particles (512 blocks) run as a single wave on 148 SMs
// with 3 or 4 blocks on every SM.  Against 64-thread blocks this halves the
// block partials the last block combines (measured on B200 at N = 65536:
// 34.5 against 36.3 us per transition).
constexpr int kL96Block = 128;
// resident blocks per SM the L96 kernels are compiled for (launch bounds)
constexpr int l96_min_blocks(int esz) { return esz == 4 ? 512 / kL96Block : 256 / kL96Block; }
// PZ: one particle per thread, 128-thread blocks
constexpr int kPZBlock = 128;

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

// RK4IntegratorHost::update (RK4IntegratorHost.hpp:63-97) with the stages of
// RK4Stage (share/src/bi/ode/RK4Stage.hpp:128-178): a21 = a32 = 1/2, a43 = 1
// (exact scalings folded into h), b = 1/6, 1/3, 1/3, 1/6.
template <class T, int D>
__device__ __forceinline__ void l96_rk4(T (&x0)[D], double t1d, double t2d, T F, T h0) {
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
}

// eta[i] ~ gaussian(0, sigma_eta); x[i] <- x[i] + eta[i]; then
// lp += -0.5*((y - x)/sigma)^2 - BI_HALF_LOG_TWO_PI - log(sigma), four
// components per Philox block, in component order.  The integrated state is
// staged in sx[.][threadIdx.x]; the new state goes to x_out[i*ld + p_out];
// prng is the particle's index in its filter's random stream; bit i of mask
// says whether component i is observed (the observation Mask of
// SparseStaticLogDensity, share/src/bi/state/Mask.hpp).  Returns l plus the
// observation terms.
template <class T, int D, bool MASKED>
__device__ __forceinline__ double l96_noise_obs_impl(const T (&sx)[D][kL96Block], T* __restrict__ x_out, size_t ld,
                                                     int p_out, const T* __restrict__ y, uint64_t seed, uint32_t prng,
                                                     int step, const L96Params& prm, double l, uint64_t mask) {
  const T se = (T)prm.sigma_eta;
  const T sy = (T)prm.sigma_y, isy = (T)prm.inv_sigma_y;
  const T c2 = (T)prm.c_half_log_2pi, ls = (T)prm.log_sigma_y;
#pragma unroll 1
  for (int b = 0; b < (D + 3) / 4; ++b) {
    bpf_u32x4 r = bpf_draw(seed, prng, (uint32_t)step, (uint32_t)b, BPF_RNG_NOISE);
    T z[4];
    box_muller(r.v[0], r.v[1], z[0], z[1]);
    box_muller(r.v[2], r.v[3], z[2], z[3]);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int i = 4 * b + j;
      if (i < D) {
        const T xi = Prec<T>::add_(sx[i][threadIdx.x], Prec<T>::mul_(se, z[j]));
        x_out[(size_t)i * ld + p_out] = xi;
        if (y && (!MASKED || ((mask >> i) & 1ull))) {
          T dz = __ldg(y + i) - xi;
          dz = isy != (T)0 ? dz * isy : dz / sy;
          T term = Prec<T>::fma_((T)-0.5, dz * dz, -c2) - ls;
          l += (double)term;
        }
      }
    }
  }
  return l;
}

// Every component observed (the usual case): the loop without the per
// component test of the mask.
template <class T, int D>
__device__ __forceinline__ double l96_noise_obs(const T (&sx)[D][kL96Block], T* __restrict__ x_out, size_t ld,
                                                int p_out, const T* __restrict__ y, uint64_t seed, uint32_t prng,
                                                int step, const L96Params& prm, double l,
                                                uint64_t mask = ~0ull) {
  constexpr uint64_t all = D >= 64 ? ~0ull : (1ull << D) - 1ull;
  if ((mask & all) == all)
    return l96_noise_obs_impl<T, D, false>(sx, x_out, ld, p_out, y, seed, prng, step, prm, l, mask);
  return l96_noise_obs_impl<T, D, true>(sx, x_out, ld, p_out, y, seed, prng, step, prm, l, mask);
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

// alpha ~ log_normal(mu, sigma): exp(gaussian(mu, sigma)) (gaussian.hpp.tt:37-43)
template <class T>
__device__ __forceinline__ T pz_alpha(uint64_t seed, uint32_t prng, int step, const PZParams& prm) {
  bpf_u32x4 r = bpf_draw(seed, prng, (uint32_t)step, 0u, BPF_RNG_NOISE);
  T z0, z1;
  box_muller(r.v[0], r.v[1], z0, z1);
  return Prec<T>::exp_(Prec<T>::fma_((T)prm.sigma, z0, (T)prm.mu));
}

// RK43IntegratorHost::update loop (RK43IntegratorHost.hpp:77-141) for one
// particle; (P, Z) in, the state after the last accepted step out.
template <class T>
__device__ __forceinline__ void pz_advance(T& P, T& Z, T alpha, double t1d, double t2d, const PZParams& prm) {
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
}

// y ~ gaussian(log(P), sigma_y): the log-density term
template <class T>
__device__ __forceinline__ double pz_obs_term(T P, T yv, const PZParams& prm) {
  T dz = yv - Prec<T>::log_(P);
  const T isy = (T)prm.inv_sigma_y;
  dz = isy != (T)0 ? dz * isy : dz / (T)prm.sigma_y;
  T term = Prec<T>::fma_((T)-0.5, dz * dz, -(T)prm.c_half_log_2pi) - (T)prm.log_sigma_y;
  return (double)term;
}

// ---------------------------------------------------------------------------
// host-side parameter blocks
// ---------------------------------------------------------------------------
inline bool params_is_pow2(double v) {
  if (!(v > 0.0)) return false;
  int e;
  double m = std::frexp(v, &e);
  return m == 0.5;
}

template <class T>
inline L96Params l96_params(const double* theta, double h) {
  L96Params p;
  p.F = theta[0];
  p.sigma_eta = theta[1];
  p.sigma_y = theta[2];
  p.x0_mean = theta[3];
  p.x0_std = theta[4];
  p.h = h;
  p.c_half_log_2pi = (double)(T)0.91893853320467274178032973640562;
  p.log_sigma_y = (double)(T)std::log((T)theta[2]);
  p.inv_sigma_y = params_is_pow2(theta[2]) ? 1.0 / theta[2] : 0.0;
  return p;
}

template <class T>
inline PZParams pz_params(const double* theta, double h, double atoler, double rtoler) {
  PZParams p;
  p.c = theta[0]; p.e = theta[1]; p.m = theta[2]; p.q = theta[3];
  p.mu = theta[4]; p.sigma = theta[5]; p.sigma_y = theta[6];
  p.p0_mu = theta[7]; p.p0_sigma = theta[8]; p.z0_mu = theta[9]; p.z0_sigma = theta[10];
  p.h0 = h; p.atoler = atoler; p.rtoler = rtoler;
  p.c_half_log_2pi = (double)(T)0.91893853320467274178032973640562;
  p.log_sigma_y = (double)(T)std::log((T)theta[6]);
  p.inv_sigma_y = params_is_pow2(theta[6]) ? 1.0 / theta[6] : 0.0;
  // h_ode_init defaults (share/src/bi/host/ode/IntegratorConstants.cpp:77-87)
  p.safe = 0.9; p.facl = 0.2; p.facr = 10.0; p.beta = 0.04; p.nsteps = 1000;
  // h_ode_set_safe / h_ode_set_beta (IntegratorConstants.cpp:45-60), in T
  p.logsafe = (double)(T)std::log((T)0.9);
  p.expo = (double)((T)0.5 * (T)std::fma(-(T)0.04, (T)0.75, (T)0.2));
  return p;
}

}  // namespace bpf
