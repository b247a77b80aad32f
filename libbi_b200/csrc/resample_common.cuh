// Device helpers shared by the single-filter resamplers (resample.cu) and the
// batched ones (batch.cu): the systematic offspring expression, the
// multinomial draws and block-wide scans of any block size.
#pragma once
#include "internal.cuh"

namespace bpf {

// ---------------------------------------------------------------------------
// Os_i = min(n, int(Ws_i / W * n + a)): resample_cumulative_offspring,
// share/src/bi/resampler/SystematicResampler.hpp:47-50, evaluated as three
// rounded FP64 operations in that order and truncated.  The quotient Ws/W is
// formed as q0 = Ws*y, r = fma(-q0, W, Ws), q = fma(r, y, q0) with y the
// correctly rounded 1/W, which equals the IEEE quotient (Markstein).
__device__ __forceinline__ double quotient(double Ws, double W, double y) {
  const double q0 = __dmul_rn(Ws, y);
  return __fma_rn(__fma_rn(-q0, W, Ws), y, q0);
}

__device__ __forceinline__ int systematic_Os(double Ws, double W, double y, double nd, double a, int n) {
  double r = __dadd_rn(__dmul_rn(quotient(Ws, W, y), nd), a);
  int o = __double2int_rz(r);
  return o < n ? o : n;
}

// uniform for the multinomial draw consumed at position t (t = 0 first)
__device__ __forceinline__ double multinomial_uniform(const double* u, int t, uint64_t seed, int step) {
  if (u) return u[t];
  bpf_u32x4 r = bpf_draw(seed, (uint32_t)t, (uint32_t)step, 0u, BPF_RNG_MULTINOMIAL);
  return bpf_u01d(r.v[0], r.v[1]);
}

// Bentley & Saxe spacing of output slot s: the reference accumulates
// lMax += log(u)/i for i = n, n-1, ..., 1 and writes slot i-1
// (share/src/bi/host/resampler/MultinomialResamplerHost.hpp:239-249);
// slot s = i-1 consumes draw t = n-1-s.  Returns -log(u)/i >= 0.
__device__ __forceinline__ double multinomial_spacing(const double* u, int s, int n, uint64_t seed, int step) {
  double uu = multinomial_uniform(u, n - 1 - s, seed, step);
  return -__ddiv_rn(log(uu), (double)(s + 1));
}

template <int NT>
__device__ __forceinline__ u128 block_exclusive_scan_u128_nt(u128 v, u128* total) {
  __shared__ u128 wt[NT / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  u128 inc = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    u128 o = shfl_up_u128(inc, d);
    if (lane >= d) inc = u128_add(inc, o);
  }
  if (lane == 31) wt[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    u128 t = lane < NT / 32 ? wt[lane] : u128_zero();
#pragma unroll
    for (int d = 1; d < NT / 32; d <<= 1) {
      u128 o = shfl_up_u128(t, d);
      if (lane >= d) t = u128_add(t, o);
    }
    if (lane < NT / 32) wt[lane] = t;
  }
  __syncthreads();
  u128 r = u128_add(warp > 0 ? wt[warp - 1] : u128_zero(), u128_sub(inc, v));
  *total = wt[NT / 32 - 1];
  __syncthreads();
  return r;
}

template <int NT>
__device__ __forceinline__ int block_exclusive_scan_int_nt(int v, int* total) {
  __shared__ int wt[NT / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int inc = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    int o = __shfl_up_sync(0xffffffffu, inc, d);
    if (lane >= d) inc += o;
  }
  if (lane == 31) wt[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    int t = lane < NT / 32 ? wt[lane] : 0;
#pragma unroll
    for (int d = 1; d < NT / 32; d <<= 1) {
      int o = __shfl_up_sync(0xffffffffu, t, d);
      if (lane >= d) t += o;
    }
    if (lane < NT / 32) wt[lane] = t;
  }
  __syncthreads();
  int r = (warp > 0 ? wt[warp - 1] : 0) + inc - v;
  *total = wt[NT / 32 - 1];
  __syncthreads();
  return r;
}

// Metropolis ancestor of particle p after B steps, following
// MetropolisResamplerHost::ancestors
// (share/src/bi/host/resampler/MetropolisResamplerHost.hpp:290-321); draw k
// uses (u_int, u_acc) = u[2(p*B+k)], u[2(p*B+k)+1] when u is given, else the
// counter-based stream.
__device__ __forceinline__ int metropolis_ancestor(const double* __restrict__ lw, int n, int B, const double* u,
                                                   uint64_t seed, int step, int p) {
  const double nd = (double)n;
  int p1 = p;
  double lw1 = lw[p];
  for (int k = 0; k < B; ++k) {
    double ui, ua;
    if (u) {
      size_t idx = 2 * ((size_t)p * B + k);
      ui = u[idx];
      ua = u[idx + 1];
    } else {
      bpf_u32x4 r = bpf_draw(seed, (uint32_t)p, (uint32_t)step, (uint32_t)k, BPF_RNG_METROPOLIS);
      ui = bpf_u01d(r.v[0], r.v[1]);
      ua = bpf_u01d(r.v[2], r.v[3]);
    }
    int p2 = __double2int_rz(__dmul_rn(ui, nd));
    p2 = p2 < n - 1 ? p2 : n - 1;  // uniformInt(0, n-1); also bounds caller-supplied uniforms
    p2 = p2 > 0 ? p2 : 0;
    double lw2 = __ldg(lw + p2);
    if (log(ua) < __dsub_rn(lw2, lw1)) {
      p1 = p2;
      lw1 = lw2;
    }
  }
  return p1;
}

}  // namespace bpf
