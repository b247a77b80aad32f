/*
 * Portable elementary functions for the particle filter's random stream and
 * model arithmetic.
 *
 * These are written so that the CUDA kernels and a host (C99) build of the
 * same code produce bit-identical results: every product that feeds a sum is
 * an explicit fused multiply-add, all other operations are single IEEE-754
 * operations (+, -, *, /, sqrt, rint), and exponent handling is done on the
 * bit patterns.  Host builds must not contract expressions on their own
 * (-ffp-contract=off).  The methods are textbook ones:
 *   exp(x)      Cody-Waite reduction x = k ln2 + r (ln2 split in a short
 *               "hi" part, exact in k*hi, and a "lo" remainder), Taylor
 *               series of e^r on |r| <= ln2/2, scaling by 2^k;
 *   log(x)      x = 2^e m with m in [sqrt(1/2), sqrt(2)),
 *               log m = 2 atanh(s), s = (m-1)/(m+1), atanh by its series;
 *   sincospi(x) reduction x = r + q/2 with q = rint(2x), |r| <= 1/4, Taylor
 *               series of sin(pi r) and cos(pi r) with coefficients
 *               (+-)pi^k/k!, and the quarter-turn identities.
 * Series are truncated where the next term is below half an ulp; observed
 * errors are within 2 ulp of the correctly rounded value (checked by the
 * test suite against the C library on the host and CUDA on the device).
 */
#ifndef BPF_MATH_H
#define BPF_MATH_H

#include <stdint.h>
#include <string.h>
#include <math.h>

#include "bpf_philox.h"

#define BPF_MATH_FMA(a, b, c) fma((a), (b), (c))
#define BPF_MATH_FMAF(a, b, c) fmaf((a), (b), (c))
/* a product that must be rounded on its own before it feeds a sum */
#if defined(__CUDA_ARCH__)
#define BPF_MATH_MUL(a, b) __dmul_rn((a), (b))
#define BPF_MATH_MULF(a, b) __fmul_rn((a), (b))
#else
#define BPF_MATH_MUL(a, b) ((a) * (b))
#define BPF_MATH_MULF(a, b) ((a) * (b))
#endif

BPF_HD uint64_t bpf_dbits(double x) { uint64_t u; memcpy(&u, &x, 8); return u; }
BPF_HD double bpf_bitsd(uint64_t u) { double x; memcpy(&x, &u, 8); return x; }
BPF_HD uint32_t bpf_fbits(float x) { uint32_t u; memcpy(&u, &x, 4); return u; }
BPF_HD float bpf_bitsf(uint32_t u) { float x; memcpy(&x, &u, 4); return x; }

/* Exact conversions without integer<->float instructions, for the integer
 * ranges used below: 2^23 + k (float) and 2^52 + k (double) hold k in their
 * low mantissa bits, so adding 1.5*2^23 (1.5*2^52) rounds a value to the
 * nearest integer (ties to even) and exposes its low bits. */
BPF_HD float bpf_small_int_to_float(int k) {      /* |k| < 2^21 */
  return bpf_bitsf(0x4B000000u | (uint32_t)(k + (1 << 22))) - 12582912.0f;
}
BPF_HD double bpf_small_int_to_double(int k) {    /* |k| < 2^30 */
  return bpf_bitsd(0x4330000000000000ull | (uint64_t)(uint32_t)(k + (1 << 30))) - 4503600701112320.0;
}

/* ---------------------------------------------------------------- double */

BPF_HD double bpf_exp(double x) {
  const double inv_ln2 = 1.4426950408889634;
  const double ln2_hi = 0.6931471803691238;     /* 32 significant bits */
  const double ln2_lo = 1.9082149292705877e-10; /* ln2 - ln2_hi */
  if (x != x) return x;
  if (x > 709.782712893384) return INFINITY;
  if (x < -745.1332191019412) return 0.0;
  /* k = rint(x / ln2) by the 1.5*2^52 rounding constant; its low bits are k */
  const double t = BPF_MATH_MUL(x, inv_ln2) + 6755399441055744.0;
  const double k = t - 6755399441055744.0;
  const int ki = (int)(uint32_t)bpf_dbits(t);
  double r = BPF_MATH_FMA(-k, ln2_hi, x);
  r = BPF_MATH_FMA(-k, ln2_lo, r);
  /* e^r = sum r^j / j!, j <= 13 */
  double p = 1.0 / 6227020800.0;                 /* 1/13! */
  p = BPF_MATH_FMA(p, r, 1.0 / 479001600.0);     /* 1/12! */
  p = BPF_MATH_FMA(p, r, 1.0 / 39916800.0);
  p = BPF_MATH_FMA(p, r, 1.0 / 3628800.0);
  p = BPF_MATH_FMA(p, r, 1.0 / 362880.0);
  p = BPF_MATH_FMA(p, r, 1.0 / 40320.0);
  p = BPF_MATH_FMA(p, r, 1.0 / 5040.0);
  p = BPF_MATH_FMA(p, r, 1.0 / 720.0);
  p = BPF_MATH_FMA(p, r, 1.0 / 120.0);
  p = BPF_MATH_FMA(p, r, 1.0 / 24.0);
  p = BPF_MATH_FMA(p, r, 1.0 / 6.0);
  p = BPF_MATH_FMA(p, r, 0.5);
  p = BPF_MATH_FMA(p, r, 1.0);
  p = BPF_MATH_FMA(p, r, 1.0);
  if (ki >= -1022) {
    if (ki > 1023) return p * bpf_bitsd((uint64_t)(1023 + 1023) << 52) * 2.0;
    return p * bpf_bitsd((uint64_t)(ki + 1023) << 52);
  }
  /* subnormal result: scale in two steps */
  return (p * bpf_bitsd((uint64_t)(ki + 1000 + 1023) << 52)) * bpf_bitsd((uint64_t)(-1000 + 1023) << 52);
}

/* log of a positive, finite, normal x times 2^e0: the body of bpf_log
 * without its special cases */
BPF_HD double bpf_log_normal(double x, int e0) {
  const double ln2_hi = 0.6931471803691238;
  const double ln2_lo = 1.9082149292705877e-10;
  const uint64_t u = bpf_dbits(x);
  int e = e0 + (int)(u >> 52) - 1023;
  double m = bpf_bitsd((u & 0x000FFFFFFFFFFFFFull) | 0x3FF0000000000000ull); /* [1,2) */
  if (m > 1.4142135623730951) { m = m * 0.5; e += 1; }
  double s = (m - 1.0) / (m + 1.0);
  double s2 = s * s;
  /* 2 atanh(s) = 2s (1 + s^2/3 + s^4/5 + ... + s^20/21) */
  double p = 1.0 / 21.0;
  p = BPF_MATH_FMA(p, s2, 1.0 / 19.0);
  p = BPF_MATH_FMA(p, s2, 1.0 / 17.0);
  p = BPF_MATH_FMA(p, s2, 1.0 / 15.0);
  p = BPF_MATH_FMA(p, s2, 1.0 / 13.0);
  p = BPF_MATH_FMA(p, s2, 1.0 / 11.0);
  p = BPF_MATH_FMA(p, s2, 1.0 / 9.0);
  p = BPF_MATH_FMA(p, s2, 1.0 / 7.0);
  p = BPF_MATH_FMA(p, s2, 1.0 / 5.0);
  p = BPF_MATH_FMA(p, s2, 1.0 / 3.0);
  p = p * s2;
  double t = 2.0 * s;
  double lm = BPF_MATH_FMA(t, p, t);
  const double ed = bpf_small_int_to_double(e);
  return BPF_MATH_FMA(ed, ln2_hi, BPF_MATH_FMA(ed, ln2_lo, lm));
}

BPF_HD double bpf_log(double x) {
  if (x != x) return x;
  if (x < 0.0) return NAN;
  if (x == 0.0) return -INFINITY;
  if (x == INFINITY) return x;
  if ((bpf_dbits(x) >> 52) == 0) return bpf_log_normal(x * 18014398509481984.0, -54); /* subnormal: x 2^54 */
  return bpf_log_normal(x, 0);
}

/* sin(pi x), cos(pi x) from q = rint(2x) and its quadrant qi */
BPF_HD void bpf_sincospi_q(double x, double q, int qi, double* sp, double* cp) {
  double r = BPF_MATH_FMA(-0.5, q, x);
  double r2 = r * r;
  double s = -2.2948428997269873e-08;            /* -pi^19/19! */
  s = BPF_MATH_FMA(s, r2, 7.952054001475513e-07);
  s = BPF_MATH_FMA(s, r2, -2.1915353447830217e-05);
  s = BPF_MATH_FMA(s, r2, 0.00046630280576761255);
  s = BPF_MATH_FMA(s, r2, -0.0073704309457143504);
  s = BPF_MATH_FMA(s, r2, 0.08214588661112823);
  s = BPF_MATH_FMA(s, r2, -0.5992645293207921);
  s = BPF_MATH_FMA(s, r2, 2.5501640398773455);
  s = BPF_MATH_FMA(s, r2, -5.16771278004997);
  s = BPF_MATH_FMA(s, r2, 3.141592653589793);
  s = s * r;
  double c = -1.3878952462213771e-07;            /* -pi^18/18! */
  c = BPF_MATH_FMA(c, r2, 4.303069587032947e-06);
  c = BPF_MATH_FMA(c, r2, -0.0001046381049248457);
  c = BPF_MATH_FMA(c, r2, 0.0019295743094039231);
  c = BPF_MATH_FMA(c, r2, -0.02580689139001406);
  c = BPF_MATH_FMA(c, r2, 0.2353306303588932);
  c = BPF_MATH_FMA(c, r2, -1.3352627688545895);
  c = BPF_MATH_FMA(c, r2, 4.0587121264167685);
  c = BPF_MATH_FMA(c, r2, -4.934802200544679);
  c = BPF_MATH_FMA(c, r2, 1.0);
  switch (qi) {
    case 0: *sp = s; *cp = c; break;
    case 1: *sp = c; *cp = -s; break;
    case 2: *sp = -s; *cp = -c; break;
    default: *sp = -c; *cp = s; break;
  }
}


/* bpf_sincospi for |x| < 1e15: q = rint(2x) by the rounding constant, the
 * quadrant in its low bits */
BPF_HD void bpf_sincospi_small(double x, double* sp, double* cp) {
  const double t = 2.0 * x + 6755399441055744.0;
  bpf_sincospi_q(x, t - 6755399441055744.0, (int)(bpf_dbits(t) & 3u), sp, cp);
}

/* sin(pi x) and cos(pi x) */
BPF_HD void bpf_sincospi(double x, double* sp, double* cp) {
  if (fabs(x) < 1.0e15) {
    bpf_sincospi_small(x, sp, cp);
    return;
  }
  const double q = rint(2.0 * x);
  bpf_sincospi_q(x, q, ((int)fmod(q, 4.0) + 4) & 3, sp, cp);
}

/* ----------------------------------------------------------------- float */

BPF_HD float bpf_expf(float x) {
  const float inv_ln2 = 1.44269502f;
  const float ln2_hi = 0.693145751953125f;    /* 16 significant bits */
  const float ln2_lo = 1.428606765330187e-06f;
  if (x != x) return x;
  if (x > 88.72283f) return INFINITY;
  if (x < -103.97208f) return 0.0f;
  const float t = BPF_MATH_MULF(x, inv_ln2) + 12582912.0f;
  const float k = t - 12582912.0f;
  const int ki = (int)(bpf_fbits(t) & 0x7FFFFFu) - 0x400000;
  float r = BPF_MATH_FMAF(-k, ln2_hi, x);
  r = BPF_MATH_FMAF(-k, ln2_lo, r);
  float p = 1.0f / 5040.0f;
  p = BPF_MATH_FMAF(p, r, 1.0f / 720.0f);
  p = BPF_MATH_FMAF(p, r, 1.0f / 120.0f);
  p = BPF_MATH_FMAF(p, r, 1.0f / 24.0f);
  p = BPF_MATH_FMAF(p, r, 1.0f / 6.0f);
  p = BPF_MATH_FMAF(p, r, 0.5f);
  p = BPF_MATH_FMAF(p, r, 1.0f);
  p = BPF_MATH_FMAF(p, r, 1.0f);
  if (ki >= -126) {
    if (ki > 127) return p * bpf_bitsf((uint32_t)(127 + 127) << 23) * 2.0f;
    return p * bpf_bitsf((uint32_t)(ki + 127) << 23);
  }
  return (p * bpf_bitsf((uint32_t)(ki + 64 + 127) << 23)) * bpf_bitsf((uint32_t)(-64 + 127) << 23);
}

/* log of a positive, finite, normal x times 2^e0: the body of bpf_logf
 * without its special cases */
BPF_HD float bpf_logf_normal(float x, int e0) {
  const float ln2_hi = 0.693145751953125f;
  const float ln2_lo = 1.428606765330187e-06f;
  const uint32_t u = bpf_fbits(x);
  int e = e0 + (int)(u >> 23) - 127;
  float m = bpf_bitsf((u & 0x007FFFFFu) | 0x3F800000u);
  if (m > 1.41421354f) { m = m * 0.5f; e += 1; }
  float s = (m - 1.0f) / (m + 1.0f);
  float s2 = s * s;
  float p = 1.0f / 9.0f;
  p = BPF_MATH_FMAF(p, s2, 1.0f / 7.0f);
  p = BPF_MATH_FMAF(p, s2, 1.0f / 5.0f);
  p = BPF_MATH_FMAF(p, s2, 1.0f / 3.0f);
  p = p * s2;
  float t = 2.0f * s;
  float lm = BPF_MATH_FMAF(t, p, t);
  const float ef = bpf_small_int_to_float(e);
  return BPF_MATH_FMAF(ef, ln2_hi, BPF_MATH_FMAF(ef, ln2_lo, lm));
}

BPF_HD float bpf_logf(float x) {
  if (x != x) return x;
  if (x < 0.0f) return NAN;
  if (x == 0.0f) return -INFINITY;
  if (x == INFINITY) return x;
  if ((bpf_fbits(x) >> 23) == 0) return bpf_logf_normal(x * 16777216.0f, -24); /* subnormal: x 2^24 */
  return bpf_logf_normal(x, 0);
}

/* sin(pi x), cos(pi x) from q = rint(2x) and its quadrant qi */
BPF_HD void bpf_sincospif_q(float x, float q, int qi, float* sp, float* cp) {
  float r = BPF_MATH_FMAF(-0.5f, q, x);
  float r2 = r * r;
  float s = 0.08214588463306427f;                /* pi^9/9! */
  s = BPF_MATH_FMAF(s, r2, -0.5992645025253296f);
  s = BPF_MATH_FMAF(s, r2, 2.550163984298706f);
  s = BPF_MATH_FMAF(s, r2, -5.167712688446045f);
  s = BPF_MATH_FMAF(s, r2, 3.1415927410125732f);
  s = s * r;
  float c = -0.025806890800595284f;              /* -pi^10/10! */
  c = BPF_MATH_FMAF(c, r2, 0.23533062636852264f);
  c = BPF_MATH_FMAF(c, r2, -1.3352627754211426f);
  c = BPF_MATH_FMAF(c, r2, 4.058712005615234f);
  c = BPF_MATH_FMAF(c, r2, -4.934802055358887f);
  c = BPF_MATH_FMAF(c, r2, 1.0f);
  switch (qi) {
    case 0: *sp = s; *cp = c; break;
    case 1: *sp = c; *cp = -s; break;
    case 2: *sp = -s; *cp = -c; break;
    default: *sp = -c; *cp = s; break;
  }
}

/* bpf_sincospif for |x| < 2^20: q = rint(2x) by the rounding constant, the
 * quadrant in its low bits */
BPF_HD void bpf_sincospif_small(float x, float* sp, float* cp) {
  const float t = 2.0f * x + 12582912.0f;
  bpf_sincospif_q(x, t - 12582912.0f, (int)(bpf_fbits(t) & 3u), sp, cp);
}

BPF_HD void bpf_sincospif(float x, float* sp, float* cp) {
  if (fabsf(x) < 1048576.0f) {
    bpf_sincospif_small(x, sp, cp);
    return;
  }
  const float q = rintf(2.0f * x);
  bpf_sincospif_q(x, q, ((int)fmodf(q, 4.0f) + 4) & 3, sp, cp);
}

/* --------------------------------------------------- standard normals */

/* Box-Muller pair from two 32-bit words: u_a, u_b are the 23-bit uniforms of
 * bpf_u01f; z0 = sqrt(-2 log u_a) cos(2 pi u_b), z1 = ... sin(2 pi u_b). */
BPF_HD void bpf_normal_pair_f(uint32_t a, uint32_t b, float* z0, float* z1) {
  /* u_a, u_b lie in [2^-24, 1 - 2^-24]: u_a is positive, finite and normal
   * and |2 u_b| < 2^20, so the special cases of bpf_logf and
   * bpf_sincospif cannot arise and their cores give the same values */
  float ua = bpf_u01f(a), ub = bpf_u01f(b);
  float r = sqrtf(-2.0f * bpf_logf_normal(ua, 0));
  float s, c;
  bpf_sincospif_small(2.0f * ub, &s, &c);
  *z0 = r * c;
  *z1 = r * s;
}

BPF_HD void bpf_normal_pair_d(uint32_t a, uint32_t b, double* z0, double* z1) {
  /* as in bpf_normal_pair_f: the guards of bpf_log and bpf_sincospi
   * cannot arise for these uniforms */
  double ua = (double)bpf_u01f(a), ub = (double)bpf_u01f(b);
  double r = sqrt(-2.0 * bpf_log_normal(ua, 0));
  double s, c;
  bpf_sincospi_small(2.0 * ub, &s, &c);
  *z0 = r * c;
  *z1 = r * s;
}

#endif
