// Hand-overs between the blocks of one launch through published words.
// Used where every block of a launch is resident (cooperative launches):
// the one-launch systematic resampler (resample.cu) and the fused filter
// step (step_fused.cu).
#pragma once
#include "internal.cuh"

namespace bpf {

// ---------------------------------------------------------------------------
// Block results published as tagged words.  A word holds the launch's epoch
// in its high half and 32 bits of payload in its low half, written by one
// store, so a reader that finds the epoch has the payload with it.  The
// readers of one transition poll all G blocks' words at once (every load of
// a round in flight together) until each carries the epoch: no atomics, no
// barrier, and the data arrives with the wait.  The epoch is a scratch word
// every block reads at its start; block 0 advances it once it has seen every
// block's first publication (so every block has read it), and the next
// launch on the scratch publishes under the next value.
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long tagged(unsigned epoch, unsigned payload) {
  return ((unsigned long long)epoch << 32) | payload;
}

__device__ __forceinline__ void st_relaxed_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ void st_release_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ unsigned ld_relaxed_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Warp 0 polls words p[i * stride + k] (i < G, k < W) until every one
// carries the epoch, W words of each of up to 128 entries in flight per
// round; fn(i, words) then consumes entry i's payloads.  Bounded by the
// barrier limit: returns false (warp-uniform) when it gave up.  Ends with an
// acquire fence, so that what the publishers released before their words is
// visible to this warp afterwards.
template <int W, class F>
__device__ __forceinline__ bool warp_poll_tagged(const unsigned long long* p, int stride, int G, unsigned epoch,
                                                 long long lim, F fn) {
  const int lane = threadIdx.x & 31;
  if (lim < 0) return false;  // the diagnostic limit: every poll gives up
  const long long t0 = clock64();
  for (int base = 0; base < G; base += 128) {
    unsigned long long w[4][W];
    while (true) {
      bool mine = true;
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int i = base + 32 * u + lane;
#pragma unroll
        for (int k = 0; k < W; ++k) w[u][k] = i < G ? ld_relaxed_u64(p + (size_t)i * stride + k) : tagged(epoch, 0u);
      }
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int k = 0; k < W; ++k) mine &= (unsigned)(w[u][k] >> 32) == epoch;
      if (__all_sync(0xffffffffu, mine)) break;
      const int give_up = lane == 0 && clock64() - t0 > lim;
      if (__shfl_sync(0xffffffffu, give_up, 0)) return false;
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int i = base + 32 * u + lane;
      if (i < G) {
        unsigned pl[W];
#pragma unroll
        for (int k = 0; k < W; ++k) pl[k] = (unsigned)w[u][k];
        fn(i, pl);
      }
    }
  }
  __threadfence();
  return true;
}

// All NT threads of the block poll words p[i * stride + k] (i < G <= 8 NT,
// k < W), entries tid, tid + NT, ... of each round in flight together, until
// every one carries the epoch; fn(i, payloads) then consumes entry i (in
// the thread that loaded it).  Bounded by `lim` cycles (a negative limit:
// give up at once); returns false (block-uniform) when it gave up.  Ends
// with an acquire fence.
template <int NT, int W, class F>
__device__ __forceinline__ bool block_poll_tagged(const unsigned long long* p, int stride, int G, unsigned epoch,
                                                  long long lim, F fn) {
  constexpr int kMaxPer = 8;
  if (lim < 0) return false;  // the diagnostic limit: every poll gives up
  const long long t0 = clock64();
  unsigned long long w[kMaxPer][W];
  while (true) {
    bool mine = true;
#pragma unroll
    for (int u = 0; u < kMaxPer; ++u) {
      const int i = (int)threadIdx.x + u * NT;
#pragma unroll
      for (int k = 0; k < W; ++k) w[u][k] = i < G ? ld_relaxed_u64(p + (size_t)i * stride + k) : tagged(epoch, 0u);
    }
#pragma unroll
    for (int u = 0; u < kMaxPer; ++u)
#pragma unroll
      for (int k = 0; k < W; ++k) mine &= (unsigned)(w[u][k] >> 32) == epoch;
    if (__syncthreads_and(mine)) break;
    if (__syncthreads_or(clock64() - t0 > lim)) return false;
  }
  __threadfence();
#pragma unroll
  for (int u = 0; u < kMaxPer; ++u) {
    const int i = (int)threadIdx.x + u * NT;
    if (i < G) {
      unsigned pl[W];
#pragma unroll
      for (int k = 0; k < W; ++k) pl[k] = (unsigned)w[u][k];
      fn(i, pl);
    }
  }
  return true;
}

}  // namespace bpf
