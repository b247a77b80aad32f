/*
 * Counter-based random numbers for the bootstrap particle filter.
 *
 * Philox4x32-10 (Salmon, Moraes, Dror & Shaw, "Parallel random numbers: as
 * easy as 1, 2, 3", SC'11), written from the published description.  Every
 * draw of the filter is addressed by a 128-bit counter
 *   (c0, c1, c2, c3) = (particle or slot, step, block within the draw, stream tag)
 * under the 64-bit key (seed low word, seed high word), so any draw can be
 * reproduced on the host from its coordinates alone, in any order and by any
 * number of threads.  This replaces the reference's per-thread mt19937 on the
 * host and per-thread cuRAND XORWOW state on the device
 * (share/src/bi/host/random/RngHost.hpp:27-214,
 *  share/src/bi/cuda/random/RngGPU.cuh:19-206), whose streams depend on the
 * thread count.
 *
 * The header is plain C99 plus CUDA qualifiers so that host code and device
 * code compute bit-identical words.
 */
#ifndef BPF_PHILOX_H
#define BPF_PHILOX_H

#include <stdint.h>

#if defined(__CUDACC__)
#define BPF_HD __host__ __device__ __forceinline__
#else
#define BPF_HD static inline
#endif

/* stream tags (c3) */
enum {
  BPF_RNG_NOISE = 0,        /* process noise of the transition */
  BPF_RNG_INIT = 1,         /* initial particle draw */
  BPF_RNG_SYSTEMATIC = 2,   /* the one offset a of a systematic resample */
  BPF_RNG_MULTINOMIAL = 3,  /* the n uniforms of a multinomial resample */
  BPF_RNG_METROPOLIS = 4,   /* the 2*B uniforms per particle of a Metropolis resample */
  BPF_RNG_DATA = 5,         /* synthetic data generation */
  BPF_RNG_PMMH = 6,         /* PMMH proposals, acceptance draws and initial parameters */
  BPF_RNG_PATH = 7          /* the particle a sampled path ends in */
};

typedef struct { uint32_t v[4]; } bpf_u32x4;

BPF_HD void bpf_mulhilo32(uint32_t a, uint32_t b, uint32_t* hi, uint32_t* lo) {
  uint64_t p = (uint64_t)a * (uint64_t)b;
  *hi = (uint32_t)(p >> 32);
  *lo = (uint32_t)p;
}

/* Philox4x32 with 10 rounds.  Round multipliers and Weyl key increments are
 * the values published for Philox4x32 in the SC'11 paper. */
BPF_HD bpf_u32x4 bpf_philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                   uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
  int r;
  for (r = 0; r < 10; ++r) {
    uint32_t hi0, lo0, hi1, lo1;
    bpf_mulhilo32(M0, c0, &hi0, &lo0);
    bpf_mulhilo32(M1, c2, &hi1, &lo1);
    uint32_t n0 = hi1 ^ c1 ^ k0;
    uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    k0 += W0; k1 += W1;
  }
  bpf_u32x4 out;
  out.v[0] = c0; out.v[1] = c1; out.v[2] = c2; out.v[3] = c3;
  return out;
}

BPF_HD bpf_u32x4 bpf_draw(uint64_t seed, uint32_t p, uint32_t step, uint32_t blk, uint32_t tag) {
  return bpf_philox4x32_10(p, step, blk, tag, (uint32_t)seed, (uint32_t)(seed >> 32));
}

/* 32 random bits -> float uniform on (0,1): (2m+1)*2^-24 with m the top 23
 * bits; exactly representable, never 0 or 1.  Formed from the bit pattern
 * 1 + m*2^-23 (two exact additions, no integer-to-float conversion). */
BPF_HD float bpf_u01f(uint32_t x) {
  union { uint32_t u; float f; } b;
  b.u = 0x3F800000u | (x >> 9);
  return (b.f - 1.0f) + 5.9604644775390625e-08f; /* 2^-24 */
}

/* 64 random bits -> double uniform on (0,1): (2m+1)*2^-53 with m the top 52
 * bits of (hi:lo); exactly representable, never 0 or 1. */
BPF_HD double bpf_u01d(uint32_t hi, uint32_t lo) {
  uint64_t m = (((uint64_t)hi << 32) | (uint64_t)lo) >> 12;
  return (double)(2u*m + 1u) * 1.1102230246251565e-16; /* 2^-53 */
}

#endif
