// The Lorenz-96 filter step in one launch: the permuted systematic
// resampling as the kernel's prologue, over the same blocks that then run
// the fused transition.
//
// The two-launch step (the one-launch resampler, then the transition as its
// programmatic dependent) pays a launch and the resampler's own tail between
// the two; here the transition's blocks (one particle per thread, 128 per
// block, every block resident: a cooperative launch) resample first, each
// block for its own 128 particles, and go straight on with the ancestor
// each thread found:
//   1. fixed-point weight of the thread's particle, the block's total
//      published as tagged words; every block polls all blocks' totals
//      (prefix below it and the total W) — hand-over 1
//   2. cumulative offspring Os (the reference's systematic expression), the
//      block's childless count published and polled — hand-over 2
//   3. E_i = Os_{i-1} - i + Z_i and its every 16th value written to global
//      memory, "E written" published and polled — hand-over 3
//   4. a survivor keeps itself; a childless slot of rank Z searches the
//      coarse index (copied to shared memory) and a 16-wide window of E for
//      the ancestor whose extra copies cover Z
// then the transition of k_l96_transition with that ancestor.  The integers
// are those of the one-launch resampler (exact fixed-point sums, the same
// quotient and the same closed-form permutation), so the ancestors are the
// same bit for bit, whatever the tiling.  The hand-overs are those of
// k_systematic_coop1 (handover.cuh), here polled by every thread of a block.
#include "internal.cuh"
#include "reduce.cuh"
#include "model_body.cuh"
#include "resample_common.cuh"
#include "handover.cuh"

#include <mutex>

namespace bpf {
namespace {

constexpr int kFusedCoarseShift = 4;  // the coarse index holds every 16th E
// block_poll_tagged reads at most 8 entries per thread: the grid's blocks
constexpr int kFusedMaxBlocks = 8 * kL96Block;

// this thread's ancestor for the step, by permuted systematic resampling
// over the launch's blocks (every block calls it; false: a wait gave up or
// the weights were degenerate, recorded in the status)
template <int NT>
__device__ __noinline__ bool fused_systematic_ancestor(const double* __restrict__ lw, int n, StepStats* st,
                                                          uint64_t seed, int step, int* __restrict__ E,
                                                          int* __restrict__ ecoarse, unsigned long long* pub,
                                                          unsigned* epoch_word, long long lim, int* s_coarse,
                                                          int* src) {
  __shared__ u128 s_u[2];
  __shared__ int s_i[2];
  __shared__ int s_os[NT];
  const int G = gridDim.x, b = blockIdx.x, tid = threadIdx.x;
  const int p = b * NT + tid;
  const bool live = p < n;
  *src = p;
  const unsigned epoch = ld_relaxed_u32(epoch_word);  // before this block publishes anything
  const double mx = st->mx;
  const bpf_u32x4 r = bpf_draw(seed, 0u, (uint32_t)step, 0u, BPF_RNG_SYSTEMATIC);
  const double a = bpf_u01d(r.v[0], r.v[1]);

  // 1. the particle's fixed-point weight and the block total
  u128 qq;
  qq.lo = live ? weight_to_fixed(nanexp(__dsub_rn(__ldg(lw + p), mx))) : 0ull;
  qq.hi = 0;
  u128 btot;
  const u128 texcl = block_exclusive_scan_u128_nt<NT>(qq, &btot);
  unsigned long long* mine = pub + (size_t)b * kPubWords;
  if (tid == 0) {
    st_relaxed_u64(mine + 0, tagged(epoch, (unsigned)btot.lo));
    st_relaxed_u64(mine + 1, tagged(epoch, (unsigned)(btot.lo >> 32)));
    st_relaxed_u64(mine + 2, tagged(epoch, (unsigned)btot.hi));
  }
  u128 lo = u128_zero(), tot = u128_zero();
  if (!block_poll_tagged<NT, 3>(pub, kPubWords, G, epoch, lim, [&](int i, const unsigned* pl) {
        u128 v;
        v.lo = (unsigned long long)pl[0] | ((unsigned long long)pl[1] << 32);
        v.hi = pl[2];
        tot = u128_add(tot, v);
        if (i < b) lo = u128_add(lo, v);
      })) {
    if (tid == 0) st->status = BPF_E_TIMEOUT;
    return false;
  }
  {
    u128 below, all;
    block_exclusive_scan_u128_nt<NT>(lo, &below);
    block_exclusive_scan_u128_nt<NT>(tot, &all);
    if (tid == 0) {
      s_u[0] = below;
      s_u[1] = all;
      // every block has published under this epoch, so every block has read
      // it: the next launch on the scratch may use the next one
      if (b == 0) *epoch_word = epoch + 1u;
    }
    __syncthreads();
  }
  const u128 prefix = s_u[0];
  const double W = u128_to_weight(s_u[1]);
  // SystematicResampler::cumulativeOffspring throws
  // ParticleFilterDegeneratedException unless W > 0
  // (share/src/bi/resampler/SystematicResampler.hpp:118-129); every block
  // sees the same W
  if (!(W > 0.0)) {
    if (b == 0 && tid == 0) st->status = BPF_E_DEGENERATE;
    return false;
  }
  const double nd = (double)n, yW = __ddiv_rn(1.0, W);

  // 2. cumulative offspring and the childless count
  const int os = systematic_Os(u128_to_weight(u128_add(u128_add(prefix, texcl), qq)), W, yW, nd, a, n);
  s_os[tid] = os;
  __syncthreads();
  const int before = tid > 0 ? s_os[tid - 1] : (b == 0 ? 0 : systematic_Os(u128_to_weight(prefix), W, yW, nd, a, n));
  const int zero = live && os == before ? 1 : 0;
  int ztot;
  const int zexcl = block_exclusive_scan_int_nt<NT>(zero, &ztot);
  if (tid == 0) st_relaxed_u64(mine + 3, tagged(epoch, (unsigned)ztot));
  int zlo = 0, zall = 0;
  if (!block_poll_tagged<NT, 1>(pub + 3, kPubWords, G, epoch, lim, [&](int i, const unsigned* pl) {
        zall += (int)pl[0];
        if (i < b) zlo += (int)pl[0];
      })) {
    if (tid == 0) st->status = BPF_E_TIMEOUT;
    return false;
  }
  {
    int below, all;
    block_exclusive_scan_int_nt<NT>(zlo, &below);
    block_exclusive_scan_int_nt<NT>(zall, &all);
    if (tid == 0) s_i[0] = below;
    __syncthreads();
  }
  const int Z = s_i[0] + zexcl;  // childless slots before p

  // 3. E: extra copies of the particles before p
  if (live) {
    const int e = before - p + Z;
    E[p] = e;
    if ((p & ((1 << kFusedCoarseShift) - 1)) == 0) ecoarse[p >> kFusedCoarseShift] = e;
  }
  __syncthreads();
  if (tid == 0) st_release_u64(mine + 4, tagged(epoch, 1u));
  if (!block_poll_tagged<NT, 1>(pub + 4, kPubWords, G, epoch, lim, [](int, const unsigned*) {})) {
    if (tid == 0) st->status = BPF_E_TIMEOUT;
    return false;
  }

  // 4. the childless slots' ancestors
  const int nc = ((n - 1) >> kFusedCoarseShift) + 1;
  {
    const int nc4 = nc >> 2;
    const int4* srcv = reinterpret_cast<const int4*>(ecoarse);
    int4* dst = reinterpret_cast<int4*>(s_coarse);
    for (int i = tid; i < nc4; i += NT) dst[i] = __ldcg(srcv + i);
    for (int i = 4 * nc4 + tid; i < nc; i += NT) s_coarse[i] = __ldcg(ecoarse + i);
  }
  __syncthreads();
  if (live && zero) {
    int clo = 0, chi = nc;
    while (clo < chi) {
      const int mid = (clo + chi) >> 1;
      if (s_coarse[mid] <= Z) clo = mid + 1; else chi = mid;
    }
    int lo_i = (clo - 1) << kFusedCoarseShift;  // s_coarse[0] = E_0 = 0 <= Z
    int hi_i = min(n, lo_i + (1 << kFusedCoarseShift));
    if (hi_i - lo_i == 16) {
      // lo_i is a multiple of 16: the window is 64-byte aligned
      const int4* w = reinterpret_cast<const int4*>(E + lo_i);
      int cnt = 0;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int4 e = __ldcg(w + j);
        cnt += (e.x <= Z) + (e.y <= Z) + (e.z <= Z) + (e.w <= Z);
      }
      lo_i += cnt;  // E is nondecreasing: the first index with E > Z
    } else {
      while (lo_i < hi_i) {
        const int mid = (lo_i + hi_i) >> 1;
        if (__ldcg(E + mid) <= Z) lo_i = mid + 1; else hi_i = mid;
      }
    }
    *src = min(max(lo_i - 1, 0), n - 1);
  }
  return true;
}

// The whole step.  Without resampling due (the gate of the step statistics)
// it is k_l96_transition; with it, the prologue above first.
template <class T, int D>
__global__ void __launch_bounds__(kL96Block, l96_min_blocks(sizeof(T)))
k_l96_step(const T* __restrict__ x_in, T* __restrict__ x_out, int ld, int n, int* __restrict__ as,
           double* __restrict__ lw, const T* __restrict__ y, double t1d, double t2d, uint64_t seed, int step,
           L96Params prm, StepStats* st, LwPartial* partials, unsigned* counter, uint64_t mask, int* E,
           int* ecoarse, unsigned long long* pub, unsigned* epoch_word, long long lim) {
  __shared__ T sx[D][kL96Block];
  extern __shared__ __align__(16) int s_coarse[];
  pdl_wait();  // the previous step's statistics, log-weights and state
  const int p = blockIdx.x * kL96Block + threadIdx.x;
  const int resampled = st->resample;  // uniform: written by the previous step's last block
  bool ok = st->status == BPF_OK;
  int src = p;
  if (ok && resampled)
    ok = fused_systematic_ancestor<kL96Block>(lw, n, st, seed, step, E, ecoarse, pub, epoch_word, lim, s_coarse,
                                              &src);
  LwPartial part = lw_empty();
  if (ok && p < n) {
    T x0[D];
#pragma unroll
    for (int i = 0; i < D; ++i) x0[i] = __ldg(x_in + (size_t)i * ld + src);
    l96_rk4<T, D>(x0, t1d, t2d, (T)prm.F, (T)prm.h);
#pragma unroll
    for (int i = 0; i < D; ++i) sx[i][threadIdx.x] = x0[i];
    // the weights were read by every block before the first hand-over
    // completed, so the in-place update cannot race with them
    const double l = l96_noise_obs<T, D>(sx, x_out, (size_t)ld, p, y, seed, (uint32_t)p, step, prm,
                                         resampled ? st->ll : lw[p], mask);
    lw[p] = l;
    if (resampled) as[p] = src;
    lw_push(part, l);
  }
  pdl_trigger();
  transition_reduce_tail(part, partials, blockIdx.x, 0, gridDim.x, counter, n, st, ok, resampled, y != nullptr);
}

size_t coarse_bytes(int n) { return (size_t)((((n - 1) >> kFusedCoarseShift) + 1 + 3) & ~3) * sizeof(int); }

// resident blocks per SM of each instantiation at its shared memory, per
// device (the launch is cooperative: every block must be resident)
template <class T, int D>
int fused_fits(int n, int blocks, size_t smem) {
  static std::mutex mu;
  static int cached[64] = {0};
  static size_t cached_smem[64] = {0};
  static int sms[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 0;
  std::lock_guard<std::mutex> lk(mu);
  if (!sms[dev] && cudaDeviceGetAttribute(&sms[dev], cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  if (cached_smem[dev] < smem || !cached[dev]) {
    if (cudaFuncSetAttribute(k_l96_step<T, D>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&cached[dev], k_l96_step<T, D>, kL96Block, smem) !=
            cudaSuccess) {
      cudaGetLastError();
      cached[dev] = 0;
      return 0;
    }
    cached_smem[dev] = smem;
  }
  (void)n;
  return blocks <= cached[dev] * sms[dev];
}

template <class T, int D>
int launch_step_t(const FusedStepArgs& a, const L96Params& prm, cudaStream_t st) {
  const int blocks = (a.t.n + kL96Block - 1) / kL96Block;
  if (blocks > a.t.max_partials || blocks > a.max_pub || blocks > kFusedMaxBlocks) return BPF_E_INVALID;
  const size_t smem = coarse_bytes(a.t.n);
  if (!fused_fits<T, D>(a.t.n, blocks, smem)) return BPF_E_INVALID;
  const T* x_in = (const T*)a.t.x_in;
  T* x_out = (T*)a.t.x_out;
  int ld = a.t.ld, n = a.t.n;
  int* as = (int*)a.t.as;
  double* lw = a.t.lw;
  const T* y = (const T*)a.t.y;
  double t1 = a.t.t1, t2 = a.t.t2;
  uint64_t seed = a.t.seed;
  int step = a.t.step;
  L96Params pr = prm;
  StepStats* stats = a.t.stats;
  LwPartial* partials = a.t.partials;
  unsigned* counter = a.t.counter;
  uint64_t mask = a.t.obs_mask;
  int* E = a.E;
  int* ec = a.ecoarse;
  unsigned long long* pub = a.pub;
  unsigned* ew = a.epoch_word;
  long long lim = barrier_limit();
  void* args[] = {(void*)&x_in, (void*)&x_out, (void*)&ld, (void*)&n, (void*)&as, (void*)&lw, (void*)&y,
                  (void*)&t1, (void*)&t2, (void*)&seed, (void*)&step, (void*)&pr, (void*)&stats,
                  (void*)&partials, (void*)&counter, (void*)&mask, (void*)&E, (void*)&ec, (void*)&pub,
                  (void*)&ew, (void*)&lim};
  // cooperative (the blocks poll each other's words) and a programmatic
  // dependent of the kernel before it (the previous step)
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute at[2];
  at[0].id = cudaLaunchAttributeCooperative;
  at[0].val.cooperative = 1;
  at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[1].val.programmaticStreamSerializationAllowed = 1;
  cfg.gridDim = dim3((unsigned)blocks);
  cfg.blockDim = dim3((unsigned)kL96Block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cfg.attrs = at;
  cfg.numAttrs = 2;
  BPF_TRY(cudaLaunchKernelExC(&cfg, (const void*)k_l96_step<T, D>, args));
  return BPF_OK;
}

template <class T>
int launch_step_prec(const ModelArgs& m, const FusedStepArgs& a, cudaStream_t st) {
  const L96Params prm = l96_params<T>(m.theta, m.h);
  switch (m.dim) {
    case 4: return launch_step_t<T, 4>(a, prm, st);
    case 8: return launch_step_t<T, 8>(a, prm, st);
    case 16: return launch_step_t<T, 16>(a, prm, st);
    case 32: return launch_step_t<T, 32>(a, prm, st);
    case 40: return launch_step_t<T, 40>(a, prm, st);
    default: return BPF_E_INVALID;
  }
}

}  // namespace

int fused_step_available(const ModelArgs& m, int n) {
  if (m.kind != BPF_MODEL_L96 || n <= 0) return 0;
  const int blocks = (n + kL96Block - 1) / kL96Block;
  if (blocks > kFusedMaxBlocks) return 0;
  const size_t smem = coarse_bytes(n);
  const bool f64 = m.precision == BPF_F64;
  switch (m.dim) {
    case 4: return f64 ? fused_fits<double, 4>(n, blocks, smem) : fused_fits<float, 4>(n, blocks, smem);
    case 8: return f64 ? fused_fits<double, 8>(n, blocks, smem) : fused_fits<float, 8>(n, blocks, smem);
    case 16: return f64 ? fused_fits<double, 16>(n, blocks, smem) : fused_fits<float, 16>(n, blocks, smem);
    case 32: return f64 ? fused_fits<double, 32>(n, blocks, smem) : fused_fits<float, 32>(n, blocks, smem);
    case 40: return f64 ? fused_fits<double, 40>(n, blocks, smem) : fused_fits<float, 40>(n, blocks, smem);
    default: return 0;
  }
}

int launch_fused_step(const ModelArgs& m, const FusedStepArgs& a, cudaStream_t st) {
  if (m.kind != BPF_MODEL_L96 || !a.E || !a.ecoarse || !a.pub || !a.epoch_word) return BPF_E_INVALID;
  return m.precision == BPF_F64 ? launch_step_prec<double>(m, a, st) : launch_step_prec<float>(m, a, st);
}

}  // namespace bpf
