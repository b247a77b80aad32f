/*
 * ORACLE — test infrastructure only.  Never linked into the product; used by
 * tests/, by the smoke check and by the bench's CPU-baseline leg.
 *
 * A CPU restatement, in plain C, of LibBi's bootstrap particle filter step as
 * the reference's host code computes it (paths relative to the LibBi tree):
 *   ess_reduce / logsumexp_reduce   share/src/bi/primitive/vector_primitive.hpp:933-974
 *   ScanResampler::precompute       share/src/bi/resampler/ScanResampler.hpp:35-40
 *   systematic offspring            share/src/bi/resampler/SystematicResampler.hpp:47-50,111-130
 *   offspring -> ancestors[Permute] share/src/bi/host/resampler/ResamplerHost.hpp:110-168
 *   ResamplerHost::permute          share/src/bi/host/resampler/ResamplerHost.hpp:171-190
 *   multinomial (Bentley & Saxe)    share/src/bi/host/resampler/MultinomialResamplerHost.hpp:29-65
 *   Metropolis                      share/src/bi/host/resampler/MetropolisResamplerHost.hpp:32-62
 *   gather_rows                     share/src/bi/host/primitive/matrix_primitive.hpp:66-75
 *   RK4                             share/src/bi/host/ode/RK4IntegratorHost.hpp:43-100, ode/RK4Stage.hpp:128-178
 *   RK4(3)                          share/src/bi/host/ode/RK43IntegratorHost.hpp:48-144, ode/RK43Stage.hpp:172-227
 *   ODE constants                   share/src/bi/host/ode/IntegratorConstants.cpp:45-87
 *   gaussian sample / log-density   share/tt/cpp/action/gaussian.hpp.tt:32-73
 *   BootstrapPF::step/correct/term  share/src/bi/filter/BootstrapPF.hpp:158-196
 *   Resampler::resample trigger     share/src/bi/resampler/Resampler.hpp:167-182
 *   Filter::filter                  share/src/bi/filter/Filter.hpp:58-70
 * Random draws are replayed from the documented counter-based stream
 * (include/bpf_philox.h, include/bpf_math.h), the tape-replay stand-in for
 * the reference's per-thread generators.  Expressions a*b + c are written as
 * fma(a, b, c), the reference's form under FP contraction; build with
 * -ffp-contract=off so that nothing else is contracted.
 *
 * Parity pinning: the resampler restatement is checked bit for bit against
 * the reference's own resampler code compiled from its sources
 * (oracle/ref/ref_resampler.cpp -> oracle/_ref/libbiref.so) on golden
 * vectors committed under tests/golden/.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/libbi_b200.h"
#include "../include/bpf_philox.h"
#include "../include/bpf_math.h"

#define HALF_LOG_TWO_PI 0.91893853320467274178032973640562

/* ------------------------------------------------------------ reductions */

/* nan_less max (share/src/bi/primitive/functor.hpp:43-53) */
static double nan_max_reduce(const double* x, int n) {
  double m = x[0];
  for (int i = 1; i < n; ++i) {
    if (isnan(m)) { if (!isnan(x[i])) m = x[i]; }
    else if (!isnan(x[i]) && m < x[i]) m = x[i];
  }
  return m;
}

static double nanexp(double x) { return isnan(x) ? 0.0 : exp(x); }

double orc_ess_reduce(const double* lw, int n, double* lW) {
  double mx = nan_max_reduce(lw, n), s1 = 0.0, s2 = 0.0;
  for (int i = 0; i < n; ++i) {
    double z = nanexp(lw[i] - mx);
    s1 += z;
    s2 += z * z;
  }
  if (lW) *lW = mx + log(s1) - log((double)n);
  return s1 * s1 / s2;
}

double orc_logsumexp(const double* lw, int n) {
  double mx = nan_max_reduce(lw, n), s = 0.0;
  for (int i = 0; i < n; ++i) s += nanexp(lw[i] - mx);
  return mx + log(s);
}

/* ------------------------------------------------------------ resamplers */

/* inclusive sequential FP64 scan of nanexp(lw - max); returns W = Ws[n-1] */
static double scan_weights(const double* lw, int n, double* Ws) {
  double mx = nan_max_reduce(lw, n), acc = 0.0;
  for (int i = 0; i < n; ++i) {
    acc = acc + nanexp(lw[i] - mx);
    Ws[i] = acc;
  }
  return Ws[n - 1];
}

/* The CUDA path's cumulative weights: each weight rounded once to a multiple
 * of 2^-63, exact 128-bit prefix sums, each rounded once to FP64. */
void orc_cumsum_exact(const double* lw, int n, double* Ws) {
  double mx = nan_max_reduce(lw, n);
  unsigned __int128 acc = 0;
  for (int i = 0; i < n; ++i) {
    double w = nanexp(lw[i] - mx);
    acc += (unsigned __int128)(uint64_t)nearbyint(w * 9223372036854775808.0);
    uint64_t hi = (uint64_t)(acc >> 64), lo = (uint64_t)acc;
    Ws[i] = (double)hi * 2.0 + (double)lo * 1.0842021724855044e-19;
  }
}

/* ResamplerHost::cumulativeOffspringToAncestors */
static void cum_to_ancestors(const int* Os, int n, int* as) {
  for (int i = 0; i < n; ++i) {
    int O1 = i > 0 ? Os[i - 1] : 0;
    for (int j = O1; j < Os[i]; ++j) as[j] = i;
  }
}

/* ResamplerHost::cumulativeOffspringToAncestorsPermute: survivors stay in
 * place, further copies (by ancestor) fill the childless slots in order. */
static void cum_to_ancestors_permute(const int* Os, int n, int* as) {
  int k = 0;
  for (int i = 0; i < n; ++i) {
    int O1 = i > 0 ? Os[i - 1] : 0;
    int o = Os[i] - O1;
    if (o > 0) { as[i] = i; --o; }
    if (k == 0 && o > 0) {
      if (Os[0] > 0) ++k;
      else { as[k++] = i; --o; }
    }
    for (int j = 0; j < o; ++j) {
      while (Os[k] - Os[k - 1] > 0) ++k;
      as[k++] = i;
    }
  }
}

/* ResamplerHost::permute (swap-based, depends on input order) */
void orc_ref_permute(int* as, int n) {
  for (int i = 0; i < n; ++i) {
    int k = as[i];
    if (k < n && k != i && as[k] != k) {
      int j = as[k];
      as[k] = k;
      as[i] = j;
      --i;
    }
  }
}

/* The permutation the CUDA path applies to any ancestor vector: offspring
 * counts -> cumulative counts -> cum_to_ancestors_permute. */
void orc_permute_rule(const int* as_in, int n, int* as_out) {
  int* Os = (int*)calloc((size_t)n, sizeof(int));
  for (int i = 0; i < n; ++i) Os[as_in[i]] += 1;
  for (int i = 1; i < n; ++i) Os[i] += Os[i - 1];
  cum_to_ancestors_permute(Os, n, as_out);
  free(Os);
}

/* Systematic: returns 0, or 1 (degenerate) when W <= 0. */
int orc_systematic(const double* lw, int n, double a, int permute, double* Ws_out, int* Os_out, int* as) {
  double* Ws = (double*)malloc(sizeof(double) * (size_t)n);
  int* Os = (int*)malloc(sizeof(int) * (size_t)n);
  double W = scan_weights(lw, n, Ws);
  if (!(W > 0.0)) { free(Ws); free(Os); return 1; }
  const double nd = (double)n;
  for (int i = 0; i < n; ++i) {
    double r = Ws[i] / W * nd + a;   /* three rounded operations, no contraction */
    int o = (int)r;
    Os[i] = o < n ? o : n;
  }
  if (permute) cum_to_ancestors_permute(Os, n, as);
  else cum_to_ancestors(Os, n, as);
  if (Ws_out) memcpy(Ws_out, Ws, sizeof(double) * (size_t)n);
  if (Os_out) memcpy(Os_out, Os, sizeof(int) * (size_t)n);
  free(Ws);
  free(Os);
  return 0;
}

/* Multinomial, sorted draws (one host thread): u[t] is the t-th uniform
 * consumed.  permute: 0 none, 1 the CUDA path's rule, 2 ResamplerHost::permute. */
int orc_multinomial(const double* lw, int n, const double* u, int permute, int* as) {
  double* Ws = (double*)malloc(sizeof(double) * (size_t)n);
  double W = scan_weights(lw, n, Ws);
  if (!(W > 0.0)) { free(Ws); return 1; }
  const double lW = log(W);
  int j = n;
  double lMax = 0.0;
  int t = 0;
  for (int i = n; i > 0; --i) {
    lMax += log(u[t++]) / i;
    double lu = lW + lMax;
    while (j > 0 && lu < log(Ws[j - 1])) --j;
    as[i - 1] = j < n ? j : n - 1;
  }
  free(Ws);
  if (permute == 1) {
    int* tmp = (int*)malloc(sizeof(int) * (size_t)n);
    orc_permute_rule(as, n, tmp);
    memcpy(as, tmp, sizeof(int) * (size_t)n);
    free(tmp);
  } else if (permute == 2) {
    orc_ref_permute(as, n);
  }
  return 0;
}

/* Metropolis: u holds (index draw, accept draw) per step, particle-major. */
int orc_metropolis(const double* lw, int n, int B, const double* u, int permute, int* as) {
  const double nd = (double)n;
  for (int p = 0; p < n; ++p) {
    int p1 = p;
    double lw1 = lw[p];
    for (int k = 0; k < B; ++k) {
      size_t idx = 2 * ((size_t)p * B + k);
      int p2 = (int)(u[idx] * nd);
      if (p2 > n - 1) p2 = n - 1;
      double lw2 = lw[p2];
      if (log(u[idx + 1]) < lw2 - lw1) { p1 = p2; lw1 = lw2; }
    }
    as[p] = p1;
  }
  if (permute == 1) {
    int* tmp = (int*)malloc(sizeof(int) * (size_t)n);
    orc_permute_rule(as, n, tmp);
    memcpy(as, tmp, sizeof(int) * (size_t)n);
    free(tmp);
  } else if (permute == 2) {
    orc_ref_permute(as, n);
  }
  return 0;
}

/* gather_rows out of place on SoA buffers (esz 4 or 8) */
void orc_gather(const int* as, const void* X, void* Y, int n, int d, int ld, int esz) {
  for (int j = 0; j < d; ++j)
    for (int i = 0; i < n; ++i)
      memcpy((char*)Y + ((size_t)j * ld + i) * esz, (const char*)X + ((size_t)j * ld + as[i]) * esz, esz);
}

/* ------------------------------------------------------- draws of a step */

/* uniforms the CUDA path draws for a resample at schedule index step */
void orc_resample_uniforms(int kind, int n, int B, uint64_t seed, int step, double* u) {
  if (kind == BPF_RESAMPLER_SYSTEMATIC) {
    bpf_u32x4 r = bpf_draw(seed, 0u, (uint32_t)step, 0u, BPF_RNG_SYSTEMATIC);
    u[0] = bpf_u01d(r.v[0], r.v[1]);
  } else if (kind == BPF_RESAMPLER_MULTINOMIAL) {
    for (int t = 0; t < n; ++t) {
      bpf_u32x4 r = bpf_draw(seed, (uint32_t)t, (uint32_t)step, 0u, BPF_RNG_MULTINOMIAL);
      u[t] = bpf_u01d(r.v[0], r.v[1]);
    }
  } else {
    for (int p = 0; p < n; ++p)
      for (int k = 0; k < B; ++k) {
        bpf_u32x4 r = bpf_draw(seed, (uint32_t)p, (uint32_t)step, (uint32_t)k, BPF_RNG_METROPOLIS);
        u[2 * ((size_t)p * B + k)] = bpf_u01d(r.v[0], r.v[1]);
        u[2 * ((size_t)p * B + k) + 1] = bpf_u01d(r.v[2], r.v[3]);
      }
  }
}

/* ----------------------------------------------------------------- models */

static int is_pow2(double v) {
  int e;
  return v > 0.0 && frexp(v, &e) == 0.5;
}

/* L96 transition of one particle in float: x (d values) in/out; returns the
 * observation log-density added to base (FP64) when y != NULL. */
static double l96_particle_f(const bpf_model_desc* m, float* x, const float* y, double t1d, double t2d,
                             uint64_t seed, int step, uint32_t p, double base, uint64_t mask) {
  const int D = m->dim;
  const float F = (float)m->theta[0], h0 = (float)m->h;
  const float b1 = (float)(1.0 / 6.0), b2 = (float)(1.0 / 3.0), b3 = (float)(1.0 / 3.0), b4 = (float)(1.0 / 6.0);
  float xs[64], k[64], acc[64];
  const float t2 = (float)t2d;
  float t = (float)t1d, h = h0;
#define L96F(X, K)                                                        \
  for (int i = 0; i < D; ++i) {                                           \
    float dd = X[(i + 1) % D] - X[(i + D - 2) % D];                        \
    K[i] = fmaf(dd, X[(i + D - 1) % D], -X[i]) + F;                        \
  }
  while (t < t2) {
    if (fmaf(1.01f, h, t) - t2 > 0.0f) {
      h = t2 - t;
      if (h <= 0.0f) { t = t2; break; }
    }
    const float hh = 0.5f * h;
    L96F(x, k)
    for (int i = 0; i < D; ++i) { acc[i] = b1 * k[i]; xs[i] = fmaf(hh, k[i], x[i]); }
    L96F(xs, k)
    for (int i = 0; i < D; ++i) { acc[i] = fmaf(b2, k[i], acc[i]); xs[i] = fmaf(hh, k[i], x[i]); }
    L96F(xs, k)
    for (int i = 0; i < D; ++i) { acc[i] = fmaf(b3, k[i], acc[i]); xs[i] = fmaf(h, k[i], x[i]); }
    L96F(xs, k)
    for (int i = 0; i < D; ++i) { acc[i] = fmaf(b4, k[i], acc[i]); x[i] = fmaf(h, acc[i], x[i]); }
    t += h;
  }
#undef L96F
  const float se = (float)m->theta[1], sy = (float)m->theta[2];
  const float isy = is_pow2(m->theta[2]) ? (float)(1.0 / m->theta[2]) : 0.0f;
  const float c2 = (float)HALF_LOG_TWO_PI, ls = logf((float)m->theta[2]);
  double l = base;
  for (int b = 0; b < (D + 3) / 4; ++b) {
    bpf_u32x4 r = bpf_draw(seed, p, (uint32_t)step, (uint32_t)b, BPF_RNG_NOISE);
    float z[4];
    bpf_normal_pair_f(r.v[0], r.v[1], &z[0], &z[1]);
    bpf_normal_pair_f(r.v[2], r.v[3], &z[2], &z[3]);
    for (int j = 0; j < 4; ++j) {
      int i = 4 * b + j;
      if (i < D) {
        x[i] = x[i] + se * z[j];
        if (y && ((mask >> i) & 1u)) {
          float dz = y[i] - x[i];
          dz = isy != 0.0f ? dz * isy : dz / sy;
          float term = fmaf(-0.5f, dz * dz, -c2) - ls;
          l += (double)term;
        }
      }
    }
  }
  return l;
}

static double l96_particle_d(const bpf_model_desc* m, double* x, const double* y, double t1d, double t2d,
                             uint64_t seed, int step, uint32_t p, double base, uint64_t mask) {
  const int D = m->dim;
  const double F = m->theta[0], h0 = m->h;
  const double b1 = 1.0 / 6.0, b2 = 1.0 / 3.0, b3 = 1.0 / 3.0, b4 = 1.0 / 6.0;
  double xs[64], k[64], acc[64];
  double t = t1d, h = h0;
  const double t2 = t2d;
#define L96D(X, K)                                                        \
  for (int i = 0; i < D; ++i) {                                           \
    double dd = X[(i + 1) % D] - X[(i + D - 2) % D];                       \
    K[i] = fma(dd, X[(i + D - 1) % D], -X[i]) + F;                         \
  }
  while (t < t2) {
    if (fma(1.01, h, t) - t2 > 0.0) {
      h = t2 - t;
      if (h <= 0.0) { t = t2; break; }
    }
    const double hh = 0.5 * h;
    L96D(x, k)
    for (int i = 0; i < D; ++i) { acc[i] = b1 * k[i]; xs[i] = fma(hh, k[i], x[i]); }
    L96D(xs, k)
    for (int i = 0; i < D; ++i) { acc[i] = fma(b2, k[i], acc[i]); xs[i] = fma(hh, k[i], x[i]); }
    L96D(xs, k)
    for (int i = 0; i < D; ++i) { acc[i] = fma(b3, k[i], acc[i]); xs[i] = fma(h, k[i], x[i]); }
    L96D(xs, k)
    for (int i = 0; i < D; ++i) { acc[i] = fma(b4, k[i], acc[i]); x[i] = fma(h, acc[i], x[i]); }
    t += h;
  }
#undef L96D
  const double se = m->theta[1], sy = m->theta[2];
  const double isy = is_pow2(sy) ? 1.0 / sy : 0.0;
  const double c2 = HALF_LOG_TWO_PI, ls = log(sy);
  double l = base;
  for (int b = 0; b < (D + 3) / 4; ++b) {
    bpf_u32x4 r = bpf_draw(seed, p, (uint32_t)step, (uint32_t)b, BPF_RNG_NOISE);
    double z[4];
    bpf_normal_pair_d(r.v[0], r.v[1], &z[0], &z[1]);
    bpf_normal_pair_d(r.v[2], r.v[3], &z[2], &z[3]);
    for (int j = 0; j < 4; ++j) {
      int i = 4 * b + j;
      if (i < D) {
        x[i] = x[i] + se * z[j];
        if (y && ((mask >> i) & 1u)) {
          double dz = y[i] - x[i];
          dz = isy != 0.0 ? dz * isy : dz / sy;
          double term = fma(-0.5, dz * dz, -c2) - ls;
          l += term;
        }
      }
    }
  }
  return l;
}

/* PZ transition of one particle in FP64 (RK4(3) adaptive) */
/* the RK4(3) day of one particle with a given alpha, then the observation
 * term */
static double pz_particle_alpha(const bpf_model_desc* m, double* x, const double* y, double t1d, double t2d,
                                double alpha, double base, uint64_t mask) {
  const double c = m->theta[0], e = m->theta[1], mm = m->theta[2], q = m->theta[3];
  const double sy = m->theta[6];
  const double atol = m->atoler, rtol = m->rtoler;
  const double facl = 0.2, facr = 10.0, beta = 0.04;
  const double logsafe = log(0.9), expo = 0.5 * fma(-0.04, 0.75, 0.2);
  const double a21 = 0.225022458725713, b1 = 0.0512293066403392, e1 = -0.0859880154628801;
  const double a32 = 0.544043312951405, b2 = 0.380954825726402, e2c = 0.189074063397015;
  const double a43 = 0.144568243493995, b3 = -0.373352596392383, e3 = -0.144145875232852;
  const double a54 = 0.786664342198357, b4 = 0.592501285026362, e4 = -0.0317933915175331;
  const double b5 = 0.34866717899928, e5 = 0.0728532188162504;
  double t = t1d, h = m->h;
  const double t2 = t2d;
  double logfacold = bpf_log(1.0e-4);
  double oP = x[0], oZ = x[1], r1P = x[0], r1Z = x[1];
  int nst = 0;
#define PZF(P_, Z_, dP, dZ)                                   \
  do {                                                        \
    double cPZ = (c * (P_)) * (Z_);                           \
    dP = fma(alpha, (P_), -cPZ);                              \
    double ecPZ = (e * c) * (P_) * (Z_);                      \
    dZ = fma(-q * (Z_), (Z_), fma(-mm, (Z_), ecPZ));          \
  } while (0)
  while (t < t2 && nst < 1000) {
    if (fma(1.01, h, t) - t2 > 0.0) {
      h = t2 - t;
      if (h <= 0.0) { t = t2; break; }
    }
    double r2P, r2Z, kP, kZ, errP, errZ, SP, SZ;
    PZF(r1P, r1Z, kP, kZ);
    errP = e1 * kP; errZ = e1 * kZ;
    r1P = fma(a21 * h, kP, r1P); r1Z = fma(a21 * h, kZ, r1Z);
    r2P = fma((b1 - a21) * h, kP, r1P); r2Z = fma((b1 - a21) * h, kZ, r1Z);
    SP = r1P; SZ = r1Z;
    PZF(SP, SZ, kP, kZ);
    errP = fma(e2c, kP, errP); errZ = fma(e2c, kZ, errZ);
    r2P = fma(a32 * h, kP, r2P); r2Z = fma(a32 * h, kZ, r2Z);
    r1P = fma((b2 - a32) * h, kP, r2P); r1Z = fma((b2 - a32) * h, kZ, r2Z);
    SP = r2P; SZ = r2Z;
    PZF(SP, SZ, kP, kZ);
    errP = fma(e3, kP, errP); errZ = fma(e3, kZ, errZ);
    r1P = fma(a43 * h, kP, r1P); r1Z = fma(a43 * h, kZ, r1Z);
    r2P = fma((b3 - a43) * h, kP, r1P); r2Z = fma((b3 - a43) * h, kZ, r1Z);
    SP = r1P; SZ = r1Z;
    PZF(SP, SZ, kP, kZ);
    errP = fma(e4, kP, errP); errZ = fma(e4, kZ, errZ);
    r2P = fma(a54 * h, kP, r2P); r2Z = fma(a54 * h, kZ, r2Z);
    r1P = fma((b4 - a54) * h, kP, r2P); r1Z = fma((b4 - a54) * h, kZ, r2Z);
    SP = r2P; SZ = r2Z;
    PZF(SP, SZ, kP, kZ);
    errP = fma(e5, kP, errP); errZ = fma(e5, kZ, errZ);
    r1P = fma(b5 * h, kP, r1P); r1Z = fma(b5 * h, kZ, r1Z);
    double eP = (errP * h) / fma(rtol, fmax(fabs(oP), fabs(r1P)), atol);
    double eZ = (errZ * h) / fma(rtol, fmax(fabs(oZ), fabs(r1Z)), atol);
    double e2 = fma(eZ, eZ, eP * eP) / 2.0;
    if (e2 <= 1.0) {
      t += h;
      if (t < t2) { oP = r1P; oZ = r1Z; }
    } else {
      r1P = oP; r1Z = oZ;
    }
    if (t < t2) {
      double logfac11 = expo * bpf_log(e2);
      if (e2 > 1.0) {
        h = h * fmax(facl, bpf_exp(logsafe - logfac11));
      } else {
        double fac = bpf_exp(fma(beta, logfacold, logsafe) - logfac11);
        fac = fmin(facr, fmax(facl, fac));
        h = h * fac;
        logfacold = 0.5 * bpf_log(fmax(e2, 1.0e-8));
      }
    }
    ++nst;
  }
#undef PZF
  x[0] = r1P;
  x[1] = r1Z;
  double l = base;
  if (y && (mask & 1u)) {
    double dz = y[0] - bpf_log(x[0]);
    dz = is_pow2(sy) ? dz * (1.0 / sy) : dz / sy;
    double term = fma(-0.5, dz * dz, -HALF_LOG_TWO_PI) - log(sy);
    l += term;
  }
  return l;
}

static double pz_particle_d(const bpf_model_desc* m, double* x, const double* y, double t1d, double t2d,
                            uint64_t seed, int step, uint32_t p, double base, uint64_t mask) {
  const double mu = m->theta[4], sigma = m->theta[5];
  bpf_u32x4 r = bpf_draw(seed, p, (uint32_t)step, 0u, BPF_RNG_NOISE);
  double z0, z1;
  bpf_normal_pair_d(r.v[0], r.v[1], &z0, &z1);
  return pz_particle_alpha(m, x, y, t1d, t2d, bpf_exp(fma(sigma, z0, mu)), base, mask);
}

/* The guided step of the PZ model (libbi_b200/csrc/guided_pz.cu) for n
 * particles given the proposal's outputs delta[p], s[p] (s already clamped):
 * log alpha = mu + delta + exp(s) z, z the particle's transition normal;
 * the ODE with alpha = exp(log alpha); lw[p] = base + the observation term
 * - ((log alpha - mu)/sigma)^2 / 2 - log sigma + z^2 / 2 + s.  x_in/x_out:
 * SoA (2 x ld); the gather through as when resampled, base ll then. */
void orc_pz_guided_step(const bpf_model_desc* m, const double* x_in, double* x_out, int ld, int n, const int* as,
                        int resampled, double* lw, double y, double t1, double t2, uint64_t seed, int step,
                        double ll, const double* delta, const double* s) {
  const double mu = m->theta[4], sigma = m->theta[5];
  for (int p = 0; p < n; ++p) {
    const int src = resampled ? as[p] : p;
    double x[2] = {x_in[src], x_in[(size_t)ld + src]};
    bpf_u32x4 r = bpf_draw(seed, (uint32_t)p, (uint32_t)step, 0u, BPF_RNG_NOISE);
    double z0, z1;
    bpf_normal_pair_d(r.v[0], r.v[1], &z0, &z1);
    const double la = fma(bpf_exp(s[p]), z0, mu + delta[p]);
    double l = pz_particle_alpha(m, x, &y, t1, t2, bpf_exp(la), resampled ? ll : lw[p], ~(uint64_t)0);
    const double u = (la - mu) / sigma;
    l += fma(-0.5, u * u, -bpf_log(sigma)) + fma(0.5, z0 * z0, s[p]);
    lw[p] = l;
    x_out[p] = x[0];
    x_out[(size_t)ld + p] = x[1];
  }
}

/* ------------------------------------------- models in the generated form
 *
 * Two models written as LibBi's code generator renders them and compiled by
 * nvcc against include/bpf_model.cuh with -fmad=false (tests/cpp/): every
 * expression of the model source in its source order, no contraction, the
 * integrators' own arithmetic as in the built-in kernels.  The oracle kinds
 * below restate them for the oracle's filter loop:
 *   ORC_MODEL_TEST_AR1  the reference's Test.bi (AR(1)) plus an observation,
 *                       tests/cpp/model_test_ar1.cuh: theta = {theta, sigma2}
 *   ORC_MODEL_L96_GEN   Lorenz '96 in the generated form,
 *                       tests/cpp/model_l96_generated.cuh:
 *                       theta = {F, sigma_eta, sigma_y, x0 mean, x0 std}
 * Normal i of a particle's step is the i-th of the stream the built-in models
 * use (block i/4, Box-Muller pairs), rng.gaussian(mu, sigma) = mu + sigma*z
 * with the product rounded first. */
#define ORC_MODEL_TEST_AR1 101
#define ORC_MODEL_L96_GEN 102

static void gen_normals_f(uint64_t seed, uint32_t p, int step, uint32_t tag, int n, float* z) {
  for (int b = 0; b < (n + 3) / 4; ++b) {
    bpf_u32x4 r = bpf_draw(seed, p, (uint32_t)step, (uint32_t)b, tag);
    float f[4];
    bpf_normal_pair_f(r.v[0], r.v[1], &f[0], &f[1]);
    bpf_normal_pair_f(r.v[2], r.v[3], &f[2], &f[3]);
    for (int j = 0; j < 4 && 4 * b + j < n; ++j) z[4 * b + j] = f[j];
  }
}

static void gen_normals_d(uint64_t seed, uint32_t p, int step, uint32_t tag, int n, double* z) {
  for (int b = 0; b < (n + 3) / 4; ++b) {
    bpf_u32x4 r = bpf_draw(seed, p, (uint32_t)step, (uint32_t)b, tag);
    double f[4];
    bpf_normal_pair_d(r.v[0], r.v[1], &f[0], &f[1]);
    bpf_normal_pair_d(r.v[2], r.v[3], &f[2], &f[3]);
    for (int j = 0; j < 4 && 4 * b + j < n; ++j) z[4 * b + j] = f[j];
  }
}

/* y ~ gaussian(mu, sigma): -0.5*pow((y - mu)/sigma, 2) - BI_HALF_LOG_TWO_PI - log(sigma)
 * (share/tt/cpp/action/gaussian.hpp.tt:58-69) in source order */
static float gen_gauss_term_f(float y, float mu, float sigma) {
  float a = (y - mu) / sigma;
  float c = a * a;
  float d = -0.5f * c;
  float e = d - (float)HALF_LOG_TWO_PI;
  return e - bpf_logf(sigma);
}

static double gen_gauss_term_d(double y, double mu, double sigma) {
  double a = (y - mu) / sigma;
  double c = a * a;
  double d = -0.5 * c;
  double e = d - HALF_LOG_TWO_PI;
  return e - bpf_log(sigma);
}

/* AR(1): w ~ gaussian(0, sqrt(sigma2)); x <- theta*x + w; y ~ gaussian(x, 0.5) */
static double ar1_particle(const bpf_model_desc* m, void* xv, const void* y, uint64_t seed, int step, uint32_t p,
                           double base, uint64_t mask) {
  double l = base;
  if (m->precision == BPF_F32) {
    float* x = (float*)xv;
    float z;
    gen_normals_f(seed, p, step, BPF_RNG_NOISE, 1, &z);
    const float theta = (float)m->theta[0], sigma2 = (float)m->theta[1];
    const float sigma = sqrtf(sigma2);
    const float w = 0.0f + sigma * z;
    x[0] = theta * x[0] + w;
    if (y && (mask & 1u)) l += (double)gen_gauss_term_f(((const float*)y)[0], x[0], 0.5f);
  } else {
    double* x = (double*)xv;
    double z;
    gen_normals_d(seed, p, step, BPF_RNG_NOISE, 1, &z);
    const double theta = m->theta[0], sigma2 = m->theta[1];
    const double sigma = sqrt(sigma2);
    const double w = 0.0 + sigma * z;
    x[0] = theta * x[0] + w;
    if (y && (mask & 1u)) l += gen_gauss_term_d(((const double*)y)[0], x[0], 0.5);
  }
  return l;
}

/* Lorenz '96 in the generated form: noise block, RK4 over the dfdt action
 * (x[n+1] - x[n-2])*x[n-1] - x[n] + F in source order, x <- x + eta,
 * observation terms gaussian(x, sigma_y) */
#define L96GEN_DFDT(REAL, X, K)                                                               \
  for (int i = 0; i < D; ++i) {                                                               \
    REAL a = X[(i + 1) % D] - X[(i + D - 2) % D];                                             \
    REAL b = a * X[(i + D - 1) % D];                                                          \
    REAL c = b - X[i];                                                                        \
    K[i] = c + F;                                                                             \
  }
#define L96GEN_RK4(REAL, FMA, X)                                                              \
  {                                                                                           \
    const REAL b1 = (REAL)(1.0 / 6.0), b2 = (REAL)(1.0 / 3.0), b3 = (REAL)(1.0 / 3.0),        \
               b4 = (REAL)(1.0 / 6.0);                                                        \
    REAL xs[64], k[64], acc[64];                                                              \
    const REAL t2 = (REAL)t2d;                                                                \
    REAL t = (REAL)t1d, h = (REAL)m->h;                                                       \
    while (t < t2) {                                                                          \
      if (FMA((REAL)1.01, h, t) - t2 > (REAL)0) {                                             \
        h = t2 - t;                                                                           \
        if (h <= (REAL)0) { t = t2; break; }                                                  \
      }                                                                                       \
      const REAL hh = (REAL)0.5 * h;                                                          \
      L96GEN_DFDT(REAL, X, k)                                                                 \
      for (int i = 0; i < D; ++i) { acc[i] = b1 * k[i]; xs[i] = FMA(hh, k[i], X[i]); }        \
      L96GEN_DFDT(REAL, xs, k)                                                                \
      for (int i = 0; i < D; ++i) { acc[i] = FMA(b2, k[i], acc[i]); xs[i] = FMA(hh, k[i], X[i]); } \
      L96GEN_DFDT(REAL, xs, k)                                                                \
      for (int i = 0; i < D; ++i) { acc[i] = FMA(b3, k[i], acc[i]); xs[i] = FMA(h, k[i], X[i]); } \
      L96GEN_DFDT(REAL, xs, k)                                                                \
      for (int i = 0; i < D; ++i) { acc[i] = FMA(b4, k[i], acc[i]); X[i] = FMA(h, acc[i], X[i]); } \
      t += h;                                                                                 \
    }                                                                                         \
  }

static double l96gen_particle(const bpf_model_desc* m, void* xv, const void* y, double t1d, double t2d,
                              uint64_t seed, int step, uint32_t p, double base, uint64_t mask) {
  const int D = m->dim;
  double l = base;
  if (m->precision == BPF_F32) {
    float* x = (float*)xv;
    const float F = (float)m->theta[0], se = (float)m->theta[1], sy = (float)m->theta[2];
    float eta[64];
    gen_normals_f(seed, p, step, BPF_RNG_NOISE, D, eta);
    for (int i = 0; i < D; ++i) eta[i] = 0.0f + se * eta[i];
    L96GEN_RK4(float, fmaf, x)
    for (int i = 0; i < D; ++i) x[i] = x[i] + eta[i];
    if (y)
      for (int i = 0; i < D; ++i)
        if ((mask >> i) & 1u) l += (double)gen_gauss_term_f(((const float*)y)[i], x[i], sy);
  } else {
    double* x = (double*)xv;
    const double F = m->theta[0], se = m->theta[1], sy = m->theta[2];
    double eta[64];
    gen_normals_d(seed, p, step, BPF_RNG_NOISE, D, eta);
    for (int i = 0; i < D; ++i) eta[i] = 0.0 + se * eta[i];
    L96GEN_RK4(double, fma, x)
    for (int i = 0; i < D; ++i) x[i] = x[i] + eta[i];
    if (y)
      for (int i = 0; i < D; ++i)
        if ((mask >> i) & 1u) l += gen_gauss_term_d(((const double*)y)[i], x[i], sy);
  }
  return l;
}
#undef L96GEN_RK4
#undef L96GEN_DFDT

static int is_gen_kind(int kind) { return kind == ORC_MODEL_TEST_AR1 || kind == ORC_MODEL_L96_GEN; }

/* initial draw of a generated-form model: AR(1) x ~ gaussian();
 * Lorenz '96 x[i] ~ gaussian(x0 mean, x0 std) */
static void gen_init_particle(const bpf_model_desc* m, void* x, int ld, uint32_t p, uint64_t seed) {
  const int D = m->dim;
  const double mu = m->kind == ORC_MODEL_TEST_AR1 ? 0.0 : m->theta[3];
  const double sd = m->kind == ORC_MODEL_TEST_AR1 ? 1.0 : m->theta[4];
  if (m->precision == BPF_F32) {
    float z[64];
    gen_normals_f(seed, p, 0, BPF_RNG_INIT, D, z);
    for (int i = 0; i < D; ++i) ((float*)x)[(size_t)i * ld + p] = (float)mu + (float)sd * z[i];
  } else {
    double z[64];
    gen_normals_d(seed, p, 0, BPF_RNG_INIT, D, z);
    for (int i = 0; i < D; ++i) ((double*)x)[(size_t)i * ld + p] = mu + sd * z[i];
  }
}

/* initial draw of particle p (Model::initialSamples) */
static void init_particle(const bpf_model_desc* m, void* x, int ld, uint32_t p, uint64_t seed) {
  if (is_gen_kind(m->kind)) {
    gen_init_particle(m, x, ld, p, seed);
  } else if (m->kind == BPF_MODEL_L96) {
    for (int b = 0; b < (m->dim + 3) / 4; ++b) {
      bpf_u32x4 r = bpf_draw(seed, p, 0u, (uint32_t)b, BPF_RNG_INIT);
      if (m->precision == BPF_F32) {
        float z[4];
        bpf_normal_pair_f(r.v[0], r.v[1], &z[0], &z[1]);
        bpf_normal_pair_f(r.v[2], r.v[3], &z[2], &z[3]);
        for (int j = 0; j < 4; ++j)
          if (4 * b + j < m->dim)
            ((float*)x)[(size_t)(4 * b + j) * ld + p] = fmaf((float)m->theta[4], z[j], (float)m->theta[3]);
      } else {
        double z[4];
        bpf_normal_pair_d(r.v[0], r.v[1], &z[0], &z[1]);
        bpf_normal_pair_d(r.v[2], r.v[3], &z[2], &z[3]);
        for (int j = 0; j < 4; ++j)
          if (4 * b + j < m->dim)
            ((double*)x)[(size_t)(4 * b + j) * ld + p] = fma(m->theta[4], z[j], m->theta[3]);
      }
    }
  } else {
    bpf_u32x4 r = bpf_draw(seed, p, 0u, 0u, BPF_RNG_INIT);
    double z0, z1;
    bpf_normal_pair_d(r.v[0], r.v[1], &z0, &z1);
    ((double*)x)[p] = bpf_exp(fma(m->theta[8], z0, m->theta[7]));
    ((double*)x)[(size_t)ld + p] = bpf_exp(fma(m->theta[10], z1, m->theta[9]));
  }
}

void orc_init(const bpf_model_desc* m, void* x, int ld, int n, double* lw, uint64_t seed) {
  for (int p = 0; p < n; ++p) {
    init_particle(m, x, ld, (uint32_t)p, seed);
    lw[p] = 0.0;
  }
}

/* One fused transition over all particles (gather from as when resampled).
 * x_in/x_out: SoA, ld; lw updated in place; base_ll used when resampled. */
/* orc_transition with observation mask (bit i: component i observed) */
void orc_transition_mask(const bpf_model_desc* m, const void* x_in, void* x_out, int ld, int n, int* as,
                         int resampled, double* lw, const void* y, double t1, double t2, uint64_t seed, int step,
                         double ll, uint64_t mask) {
  const int D = m->dim;
#pragma omp parallel for schedule(static)
  for (int p = 0; p < n; ++p) {
    const int src = resampled ? as[p] : p;
    const double base = resampled ? ll : lw[p];
    if (is_gen_kind(m->kind)) {
      double xp[64];
      const size_t esz = m->precision == BPF_F32 ? 4 : 8;
      for (int i = 0; i < D; ++i) memcpy((char*)xp + i * esz, (const char*)x_in + ((size_t)i * ld + src) * esz, esz);
      lw[p] = m->kind == ORC_MODEL_TEST_AR1
                  ? ar1_particle(m, xp, y, seed, step, (uint32_t)p, base, mask)
                  : l96gen_particle(m, xp, y, t1, t2, seed, step, (uint32_t)p, base, mask);
      for (int i = 0; i < D; ++i) memcpy((char*)x_out + ((size_t)i * ld + p) * esz, (char*)xp + i * esz, esz);
    } else if (m->precision == BPF_F32) {
      float xp[64];
      for (int i = 0; i < D; ++i) xp[i] = ((const float*)x_in)[(size_t)i * ld + src];
      lw[p] = l96_particle_f(m, xp, (const float*)y, t1, t2, seed, step, (uint32_t)p, base, mask);
      for (int i = 0; i < D; ++i) ((float*)x_out)[(size_t)i * ld + p] = xp[i];
    } else {
      double xp[64];
      for (int i = 0; i < D; ++i) xp[i] = ((const double*)x_in)[(size_t)i * ld + src];
      if (m->kind == BPF_MODEL_L96)
        lw[p] = l96_particle_d(m, xp, (const double*)y, t1, t2, seed, step, (uint32_t)p, base, mask);
      else
        lw[p] = pz_particle_d(m, xp, (const double*)y, t1, t2, seed, step, (uint32_t)p, base, mask);
      for (int i = 0; i < D; ++i) ((double*)x_out)[(size_t)i * ld + p] = xp[i];
    }
  }
}

/* One fused transition over all particles (gather from as when resampled).
 * x_in/x_out: SoA, ld; lw updated in place; base_ll used when resampled. */
void orc_transition(const bpf_model_desc* m, const void* x_in, void* x_out, int ld, int n, int* as, int resampled,
                    double* lw, const void* y, double t1, double t2, uint64_t seed, int step, double ll) {
  orc_transition_mask(m, x_in, x_out, ld, n, as, resampled, lw, y, t1, t2, seed, step, ll, ~(uint64_t)0);
}

/* ---------------------------------------------------------------- filter */

/* Filter<BootstrapPF>::filter with the CUDA path's draws.  Outputs (may be
 * NULL): inc[T], ess[T], resampled[T], *ll (BootstrapPF::term), and the final
 * state x_final (SoA, ld = n rounded up to 32) and lw_final[n].
 * Returns 0 or BPF_E_DEGENERATE. */
int orc_filter(const bpf_model_desc* m, const bpf_config* cfg, int T, double t0, double dt, const void* y,
               double* inc, double* ess_out, int* resampled_out, double* ll_out, void* x_final, double* lw_final) {
  const int n = cfg->nparticles, D = m->dim;
  const int nobs = m->kind == BPF_MODEL_L96 || m->kind == ORC_MODEL_L96_GEN ? D : 1;
  const int ld = ((n + 31) / 32) * 32;
  const size_t esz = m->precision == BPF_F64 ? 8 : 4;
  void* xa = calloc((size_t)ld * D, esz);
  void* xb = calloc((size_t)ld * D, esz);
  double* lw = (double*)malloc(sizeof(double) * (size_t)n);
  int* as = (int*)malloc(sizeof(int) * (size_t)n);
  size_t nu = cfg->resampler == BPF_RESAMPLER_METROPOLIS ? (size_t)2 * n * (cfg->metropolis_steps > 0 ? cfg->metropolis_steps : 1)
                                                          : (size_t)n;
  double* u = (double*)malloc(sizeof(double) * nu);
  orc_init(m, xa, ld, n, lw, cfg->seed);
  double ll = 0.0, ess = 0.0;
  int resample_next = 0, rc = 0;
  for (int k = 1; k <= T; ++k) {
    int resampled = 0;
    if (resample_next) {
      orc_resample_uniforms(cfg->resampler, n, cfg->metropolis_steps, cfg->seed, k, u);
      if (cfg->resampler == BPF_RESAMPLER_SYSTEMATIC) rc = orc_systematic(lw, n, u[0], 1, NULL, NULL, as);
      else if (cfg->resampler == BPF_RESAMPLER_MULTINOMIAL) rc = orc_multinomial(lw, n, u, 1, as);
      else rc = orc_metropolis(lw, n, cfg->metropolis_steps, u, 1, as);
      if (rc) { rc = BPF_E_DEGENERATE; break; }
      resampled = 1;
    }
    const char* yk = (const char*)y + (size_t)(k - 1) * nobs * esz;
    orc_transition(m, xa, xb, ld, n, as, resampled, lw, yk, t0 + (k - 1) * dt, t0 + k * dt, cfg->seed, k, ll);
    void* tmp = xa; xa = xb; xb = tmp;
    double lW;
    ess = orc_ess_reduce(lw, n, &lW);
    if (inc) inc[k - 1] = lW - ll;
    ll = lW;
    if (ess_out) ess_out[k - 1] = ess;
    if (resampled_out) resampled_out[k - 1] = resampled;
    resample_next = ess < cfg->ess_rel * (double)n;
  }
  if (!rc) {
    if (ll_out) *ll_out = orc_logsumexp(lw, n) - log((double)n);
    if (x_final) memcpy(x_final, xa, (size_t)ld * D * esz);
    if (lw_final) memcpy(lw_final, lw, sizeof(double) * (size_t)n);
  }
  free(xa); free(xb); free(lw); free(as); free(u);
  return rc;
}

/* synthetic observations: one model run from the initial draw of particle 0
 * under the data seed, observed every dt with the model's observation noise
 * (tag BPF_RNG_DATA).  y: T*nobs values in the model precision (nobs = dim
 * for L96, 1 for PZ).  Optionally returns the true states (T*dim). */
void orc_simulate(const bpf_model_desc* m, uint64_t seed, int T, double t0, double dt, void* y, void* xtrue) {
  const int D = m->dim;
  const size_t esz = m->precision == BPF_F64 ? 8 : 4;
  char xbuf[64 * 8];
  init_particle(m, xbuf, 1, 0u, seed);
  for (int k = 1; k <= T; ++k) {
    /* the filter's transition with its own noise, no observation */
    if (m->precision == BPF_F32) {
      l96_particle_f(m, (float*)xbuf, NULL, t0 + (k - 1) * dt, t0 + k * dt, seed, k, 0u, 0.0, 0u);
    } else if (m->kind == BPF_MODEL_L96) {
      l96_particle_d(m, (double*)xbuf, NULL, t0 + (k - 1) * dt, t0 + k * dt, seed, k, 0u, 0.0, 0u);
    } else {
      pz_particle_d(m, (double*)xbuf, NULL, t0 + (k - 1) * dt, t0 + k * dt, seed, k, 0u, 0.0, 0u);
    }
    if (xtrue) memcpy((char*)xtrue + (size_t)(k - 1) * D * esz, xbuf, (size_t)D * esz);
    /* observation noise */
    const int nobs = m->kind == BPF_MODEL_L96 ? D : 1;
    for (int b = 0; b < (nobs + 3) / 4; ++b) {
      bpf_u32x4 r = bpf_draw(seed, 1u, (uint32_t)k, (uint32_t)b, BPF_RNG_DATA);
      double z[4];
      bpf_normal_pair_d(r.v[0], r.v[1], &z[0], &z[1]);
      bpf_normal_pair_d(r.v[2], r.v[3], &z[2], &z[3]);
      for (int j = 0; j < 4; ++j) {
        int i = 4 * b + j;
        if (i >= nobs) continue;
        if (m->kind == BPF_MODEL_L96) {
          double mean = m->precision == BPF_F32 ? (double)((float*)xbuf)[i] : ((double*)xbuf)[i];
          double v = mean + m->theta[2] * z[j];
          if (m->precision == BPF_F32) ((float*)y)[(size_t)(k - 1) * D + i] = (float)v;
          else ((double*)y)[(size_t)(k - 1) * D + i] = v;
        } else {
          double v = log(((double*)xbuf)[0]) + m->theta[6] * z[j];
          ((double*)y)[(size_t)(k - 1) * 1 + i] = v;
        }
      }
    }
  }
}

/* ------------------------------------------------ test access to helpers */

/* fn: 0 bpf_exp, 1 bpf_log, 2 sin(pi x), 3 cos(pi x), 4 bpf_expf, 5 bpf_logf,
 *     6 sinpif, 7 cospif (float functions take and return float values) */
void orc_math_eval(int fn, const double* x, double* y, int n) {
  for (int i = 0; i < n; ++i) {
    double s, c;
    float sf, cf;
    switch (fn) {
      case 0: y[i] = bpf_exp(x[i]); break;
      case 1: y[i] = bpf_log(x[i]); break;
      case 2: bpf_sincospi(x[i], &s, &c); y[i] = s; break;
      case 3: bpf_sincospi(x[i], &s, &c); y[i] = c; break;
      case 4: y[i] = bpf_expf((float)x[i]); break;
      case 5: y[i] = bpf_logf((float)x[i]); break;
      case 6: bpf_sincospif((float)x[i], &sf, &cf); y[i] = sf; break;
      default: bpf_sincospif((float)x[i], &sf, &cf); y[i] = cf; break;
    }
  }
}

void orc_philox(const uint32_t* c, const uint32_t* k, uint32_t* out) {
  bpf_u32x4 r = bpf_philox4x32_10(c[0], c[1], c[2], c[3], k[0], k[1]);
  memcpy(out, r.v, sizeof(r.v));
}

/* n standard normals of the noise stream for particle p at step (4 per block) */
void orc_noise_normals(uint64_t seed, uint32_t p, int step, int n, int prec, double* z) {
  for (int b = 0; b < (n + 3) / 4; ++b) {
    bpf_u32x4 r = bpf_draw(seed, p, (uint32_t)step, (uint32_t)b, BPF_RNG_NOISE);
    if (prec == BPF_F32) {
      float f[4];
      bpf_normal_pair_f(r.v[0], r.v[1], &f[0], &f[1]);
      bpf_normal_pair_f(r.v[2], r.v[3], &f[2], &f[3]);
      for (int j = 0; j < 4 && 4 * b + j < n; ++j) z[4 * b + j] = f[j];
    } else {
      double d[4];
      bpf_normal_pair_d(r.v[0], r.v[1], &d[0], &d[1]);
      bpf_normal_pair_d(r.v[2], r.v[3], &d[2], &d[3]);
      for (int j = 0; j < 4 && 4 * b + j < n; ++j) z[4 * b + j] = d[j];
    }
  }
}

/* PMMH draws of chain c at filter run r (the scheme documented in
 * libbi_b200/csrc/pmmh.cu): the proposal normal of parameter j from block
 * j/2, word pair j%2 (Box-Muller, double); the acceptance uniform from block
 * 64; tag BPF_RNG_PMMH. */
void orc_pmmh_draws(uint64_t seed, int c, int r, int nparams, double* z, double* u) {
  for (int j = 0; j < nparams; ++j) {
    bpf_u32x4 w = bpf_draw(seed, (uint32_t)c, (uint32_t)r, (uint32_t)(j / 2), BPF_RNG_PMMH);
    double z0, z1;
    bpf_normal_pair_d(w.v[0], w.v[1], &z0, &z1);
    z[j] = (j & 1) ? z1 : z0;
  }
  bpf_u32x4 w = bpf_draw(seed, (uint32_t)c, (uint32_t)r, 64u, BPF_RNG_PMMH);
  *u = bpf_u01d(w.v[0], w.v[1]);
}
