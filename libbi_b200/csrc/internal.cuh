// Internal declarations shared by the libbi_b200 CUDA sources.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include "../../include/libbi_b200.h"
#include "../../include/bpf_philox.h"
#include "../../include/bpf_device.cuh"

#define BPF_TRY(call)                                          \
  do {                                                         \
    cudaError_t e_ = (call);                                   \
    if (e_ != cudaSuccess) { bpf_set_last_cuda_error(e_); return BPF_E_CUDA; } \
  } while (0)

void bpf_set_last_cuda_error(cudaError_t e);

namespace bpf {

// Resampler tile: 256 threads x 2 items (512 log-weights), so that the
// N = 65536 workload spreads over 128 blocks.
constexpr int kBlock = 256;
constexpr int kItems = 2;
constexpr int kTile = kBlock * kItems;

inline int ntiles(int n) { return (n + kTile - 1) / kTile; }

// ---------------------------------------------------------------------------
// Exact 128-bit fixed-point sums.
//
// Normalised weights w = exp(lw - max) lie in [0, 1].  Each is rounded once
// to a multiple of 2^-63 (q = rint(w * 2^63), at most 2^63) and all prefix
// sums are formed exactly in 128-bit integers.  Integer addition is
// associative, so every tile order, look-back path and thread count gives the
// same sums: the prefix sum is deterministic and at least as accurate as a
// sequential FP64 sum.  A sum is rounded to FP64 once, by u128_to_weight().
// ---------------------------------------------------------------------------
struct u128 {
  unsigned long long lo, hi;
};

__host__ __device__ __forceinline__ u128 u128_zero() { u128 r; r.lo = 0; r.hi = 0; return r; }

// on the device through the carry flag (add.cc / addc), one carry chain
// instead of a compare and a select per operation
__host__ __device__ __forceinline__ u128 u128_add(u128 a, u128 b) {
  u128 r;
#ifdef __CUDA_ARCH__
  asm("add.cc.u64 %0, %2, %4;\n\taddc.u64 %1, %3, %5;"
      : "=l"(r.lo), "=l"(r.hi)
      : "l"(a.lo), "l"(a.hi), "l"(b.lo), "l"(b.hi));
#else
  r.lo = a.lo + b.lo;
  r.hi = a.hi + b.hi + (r.lo < a.lo ? 1ull : 0ull);
#endif
  return r;
}

__host__ __device__ __forceinline__ u128 u128_sub(u128 a, u128 b) {
  u128 r;
#ifdef __CUDA_ARCH__
  asm("sub.cc.u64 %0, %2, %4;\n\tsubc.u64 %1, %3, %5;"
      : "=l"(r.lo), "=l"(r.hi)
      : "l"(a.lo), "l"(a.hi), "l"(b.lo), "l"(b.hi));
#else
  r.lo = a.lo - b.lo;
  r.hi = a.hi - b.hi - (a.lo < b.lo ? 1ull : 0ull);
#endif
  return r;
}

// weight in [0,1] -> fixed point q = rint(w * 2^63)
__device__ __forceinline__ unsigned long long weight_to_fixed(double w) {
  return __double2ull_rn(__dmul_rn(w, 9223372036854775808.0));
}

// fixed-point weight sum -> FP64 value of the sum (unscaled): hi*2 + lo*2^-63
__device__ __forceinline__ double u128_to_weight(u128 q) {
  return __dadd_rn(__dmul_rn((double)q.hi, 2.0),
                   __dmul_rn(__ull2double_rn(q.lo), 1.0842021724855044e-19 /* 2^-63 */));
}

// non-negative double -> fixed point with 64 fraction bits: (floor(v), frac(v)*2^64 truncated)
__device__ __forceinline__ u128 spacing_to_fixed(double v) {
  double f = floor(v);
  u128 r;
  r.hi = (unsigned long long)f;
  r.lo = __double2ull_rz(__dmul_rn(__dsub_rn(v, f), 18446744073709551616.0));
  return r;
}

// fixed point with 64 fraction bits -> double: hi + lo*2^-64
__device__ __forceinline__ double fixed_to_spacing(u128 q) {
  return __dadd_rn((double)q.hi, __dmul_rn(__ull2double_rn(q.lo), 5.421010862427522e-20 /* 2^-64 */));
}

__device__ __forceinline__ u128 shfl_up_u128(u128 v, int d) {
  u128 r;
  r.lo = __shfl_up_sync(0xffffffffu, v.lo, d);
  r.hi = __shfl_up_sync(0xffffffffu, v.hi, d);
  return r;
}

__device__ __forceinline__ u128 shfl_u128(u128 v, int src) {
  u128 r;
  r.lo = __shfl_sync(0xffffffffu, v.lo, src);
  r.hi = __shfl_sync(0xffffffffu, v.hi, src);
  return r;
}

// Block-wide exclusive scan of one u128 per thread (blockDim.x == kBlock).
// Returns the exclusive prefix; *total receives the block sum.
__device__ __forceinline__ u128 block_exclusive_scan_u128(u128 v, u128* total) {
  __shared__ u128 warp_tot[kBlock / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  u128 inc = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    u128 o = shfl_up_u128(inc, d);
    if (lane >= d) inc = u128_add(inc, o);
  }
  if (lane == 31) warp_tot[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    u128 t = lane < kBlock / 32 ? warp_tot[lane] : u128_zero();
#pragma unroll
    for (int d = 1; d < kBlock / 32; d <<= 1) {
      u128 o = shfl_up_u128(t, d);
      if (lane >= d) t = u128_add(t, o);
    }
    if (lane < kBlock / 32) warp_tot[lane] = t;  // inclusive warp prefixes
  }
  __syncthreads();
  u128 warp_excl = warp > 0 ? warp_tot[warp - 1] : u128_zero();
  *total = warp_tot[kBlock / 32 - 1];
  u128 excl = u128_sub(inc, v);
  __syncthreads();
  return u128_add(warp_excl, excl);
}

// Block-wide exclusive scan of one int per thread.
__device__ __forceinline__ int block_exclusive_scan_int(int v, int* total) {
  __shared__ int wt[kBlock / 32];
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
    int t = lane < kBlock / 32 ? wt[lane] : 0;
#pragma unroll
    for (int d = 1; d < kBlock / 32; d <<= 1) {
      int o = __shfl_up_sync(0xffffffffu, t, d);
      if (lane >= d) t += o;
    }
    if (lane < kBlock / 32) wt[lane] = t;
  }
  __syncthreads();
  int r = (warp > 0 ? wt[warp - 1] : 0) + inc - v;
  *total = wt[kBlock / 32 - 1];
  __syncthreads();
  return r;
}

// nanexp: share/src/bi/math/function.hpp:158-164 (NaN gives zero)
__device__ __forceinline__ double nanexp(double x) { return isnan(x) ? 0.0 : exp(x); }

// nan_less max: share/src/bi/primitive/functor.hpp:43-53 (NaN orders first)
__device__ __forceinline__ double nan_max(double a, double b) {
  if (isnan(a)) return b;
  if (isnan(b)) return a;
  return a < b ? b : a;
}

// LwPartial and StepStats: include/bpf_device.cuh

// Scratch of the resampler pipeline for up to max_n particles.
struct ResampleScratch {
  int max_n = 0;
  int max_tiles = 0;
  u128* tile_sum = nullptr;     // per-tile weight sums
  u128* tile_prefix = nullptr;  // exclusive prefixes (+1 entry: total)
  u128* vtile_sum = nullptr;    // per-tile spacing sums (multinomial)
  u128* vtile_prefix = nullptr;
  int* zcount = nullptr;        // per-tile childless counts
  int* zprefix = nullptr;       // exclusive prefixes (+1 entry: total)
  int* icount = nullptr;        // per-tile integer sums (offspring counts)
  int* iprefix = nullptr;
  int* Os = nullptr;            // cumulative offspring
  int* E = nullptr;             // cumulative extra copies
  int* slot = nullptr;          // childless slot of each rank
  int* etile = nullptr;         // every 2^k-th value of E (coarse search index)
  int* o = nullptr;             // offspring counts (Metropolis)
  double* Ws = nullptr;         // FP64 cumulative weights (multinomial search)
  double* lu = nullptr;         // log sorted uniforms (multinomial)
  unsigned* counters = nullptr; // last-block tickets; word kEpochWord: the one-launch kernel's epoch
  // block results the one-launch systematic kernel and the fused step
  // publish (tagged words, kPubWords per block, pub_entries blocks at most;
  // every tag 0xFFFFFFFF when allocated)
  unsigned long long* pub = nullptr;
  int pub_entries = 0;
  StepStats* stats = nullptr;   // reduction results
  LwPartial* partials = nullptr;
  int max_partials = 0;
};

// the one-launch systematic kernel's epoch (a counters word) and the
// published words per tile: three for the weight total, one for the
// childless count, one for "phase 3 written"
constexpr int kEpochWord = 10;
constexpr int kPubWords = 5;
// blocks that may publish for n particles: tiles of at least 128 particles
inline int pub_entries_for(int n) { return n / 128 + 2; }
int scratch_alloc(ResampleScratch& s, int max_n);
// counters[0 .. kEpochWord) to zero and the epoch advanced (after a timeout,
// and before a filter starts over)
int reset_scratch_words(ResampleScratch& s, cudaStream_t st);
void scratch_free(ResampleScratch& s);

// Reduction of lw[0..n) into s.stats (mx, s1, s2, ess, lW); stats->ll/inc untouched.
int launch_lw_reduce(const double* lw, int n, ResampleScratch& s, cudaStream_t st);
int launch_logsumexp(const double* lw, int n, ResampleScratch& s, cudaStream_t st);

// Resampler pipelines.  uniforms: device pointer or null (then drawn from
// Philox with (seed, step)).  gate: device int or null; when non-null the
// kernels do nothing unless *gate != 0.  mx from s.stats->mx when
// use_stats_max, else computed first.
struct ResampleArgs {
  int kind;
  int n;
  int B;
  const double* lw;
  const double* uniforms;
  uint64_t seed;
  int step;
  int permute;
  int* as;
  int* Os_out;
  const int* gate;
  bool max_known;  // s.stats->mx already holds max(lw)
  int shape = -1;  // tile shape of the one-launch systematic kernel (-1: autotuned or default)
};
int launch_resample(const ResampleArgs& a, ResampleScratch& s, cudaStream_t st);
// time every tile shape of the one-launch systematic resampler for n
// particles and keep the fastest for n's size class on this device
int autotune_systematic(int n, cudaStream_t st, int* best, double* us);
// the kept shape for n's size class, -1 when none was tuned, -2 when no
// shape holds n particles in one wave
int autotuned_shape(int n);

// Pruned ancestry store of the path output (ancestry.cu)
struct AncestryPool {
  int n = 0, dim = 0, esz = 0;
  int cap = 0;                       // nodes
  void* x = nullptr;                 // states: element i of node v at x[i * cap + v]
  int* par = nullptr;                // parent node (-1: first generation)
  int* ref = nullptr;                // recorded children
  int* stack = nullptr;              // free nodes, stack[0 .. *top)
  int* top = nullptr;                // device counter
  int* leaf[2] = {nullptr, nullptr};  // node of each particle of the current generation
  int cur = 0;
  int* host_top = nullptr;           // pinned copy of *top
};
// (re)start the record with the state x as the first generation
int ancestry_reset(AncestryPool& a, int n, int dim, int esz, const void* x, int ld, cudaStream_t st);
// the next generation: state x, ancestors as (read when st->resampled);
// synchronises st once
int ancestry_append(AncestryPool& a, const void* x, int ld, const int* as, const StepStats* st, cudaStream_t s);
// the len states of the line ending in particle *p_dev into path_dev (len x dim)
int ancestry_trace(const AncestryPool& a, int len, const int* p_dev, void* path_dev, cudaStream_t st);
// nodes in use and pool capacity (synchronises st)
int ancestry_nodes(AncestryPool& a, cudaStream_t st, int* nodes, int* capacity);
void ancestry_free(AncestryPool& a);

// limit of the grid-barrier waits of the cooperative resamplers on the
// current device, in SM clock cycles (negative: give up at once)
int set_barrier_limit(long long cycles);
// the current device's wait limit (what set_barrier_limit last set there)
long long barrier_limit();

int launch_gather(const int* as, const void* X, void* Y, int n, int d, int ld, int esz,
                  const int* gate, cudaStream_t st);

// Raise a kernel's dynamic shared-memory limit once per device (the
// attribute is per device; a process may drive several GPUs).  `done` is
// the caller's static bitmask of configured devices.
template <class K>
inline cudaError_t set_dyn_smem_once(K kernel, int bytes, unsigned& done) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const unsigned bit = 1u << (dev & 31);
  if (done & bit) return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess) done |= bit;
  return e;
}

// Models
struct ModelArgs {
  int kind, dim, precision, integrator;
  double h, atoler, rtoler;
  double theta[BPF_MAX_THETA];
};

struct TransitionArgs {
  const void* x_in;   // state before the step (model precision, SoA)
  void* x_out;        // state after the step
  int ld, n;
  const int* as;      // ancestors, read when *resampled_flag
  double* lw;         // FP64 log-weights, updated in place
  const void* y;      // device observation (dim values) or null
  double t1, t2;
  uint64_t seed;
  int step;
  StepStats* stats;   // reads resample flag / ll; finalised by the last block
  LwPartial* partials;
  int max_partials;   // capacity of partials (one per block)
  unsigned* counter;
  uint64_t obs_mask = ~0ull;  // bit i: component i observed (when y is given)
};
int launch_transition(const ModelArgs& m, const TransitionArgs& a, cudaStream_t st);
// The Lorenz-96 step in one cooperative launch with the permuted systematic
// resampling as its prologue (step_fused.cu); BPF_E_INVALID when the model
// is not the built-in Lorenz-96 or the blocks cannot all be resident
struct FusedStepArgs {
  TransitionArgs t;
  int* E;                    // n: extra-copy counts (scratch)
  int* ecoarse;              // n/16 + 1: every 16th of them (scratch)
  unsigned long long* pub;   // kPubWords per block (scratch)
  int max_pub;               // blocks the published words have room for
  unsigned* epoch_word;      // the scratch's epoch
};
int launch_fused_step(const ModelArgs& m, const FusedStepArgs& a, cudaStream_t st);
// 1 when the fused step can run n particles of model m on the current device
int fused_step_available(const ModelArgs& m, int n);
// the step statistics of a freshly initialised filter
int launch_stats_init(StepStats* stats, int n, double ess_rel, cudaStream_t st);
int launch_init(const ModelArgs& m, void* x, int ld, int n, double* lw, uint64_t seed,
                StepStats* stats, double ess_rel, cudaStream_t st);

}  // namespace bpf
