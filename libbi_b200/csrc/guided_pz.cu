// The guided step of the plankton (PZ) model for every filter of a batch:
// the learned proposal over each particle's log-noise.
//
// PZ's transition draws log alpha ~ N(mu, sigma) (alpha ~ log_normal,
// share/tt/cpp/action/gaussian.hpp.tt:37-43) and integrates the ODE over the
// day with that alpha (RK4(3), share/src/bi/host/ode/RK43IntegratorHost.hpp:
// 48-144).  The guided step draws instead
//   log alpha ~ q = N(mu + delta, exp(2 s)),  (delta, s) = MLP([log P, log Z, y - log P]),
// the network trained on the model's own simulated transitions (proposal.cu,
// bpf_proposal_set_states), integrates the ODE with exp(log alpha), and
// weights each particle by p(y | x') p(log alpha) / q(log alpha):
//   lw += log N(y; log P', sigma_y) - (log alpha - mu)^2 / (2 sigma^2) - log sigma + z^2 / 2 + s,
// z the standard normal of the particle's draw, so the likelihood estimate
// stays unbiased.  Two launches per step:
//   k_pz_net      the network of every particle in one kernel: a persistent
//                 CTA per SM loads the three weight images once (bulk
//                 copies, 44.5 KB, the biases of layers 1 and 2 folded in
//                 as extra K columns) and runs all three layers as tcgen05
//                 MMA chains into tensor memory, in four thread groups that
//                 take turns on the tensor core; only 8 bytes per particle
//                 leave the kernel, nothing of the hidden layers touches HBM
//                 and no weight is read by a load instruction;
//   k_batch_pz_guided  the batched PZ transition with the proposal's draw
//                 and the weight correction, ending in the same per-filter
//                 reduction tail.
// The ODE kernel keeps its own occupancy (FP64 RK4(3), 128 threads, no
// shared memory).  No counterpart in the reference, whose bootstrap filter
// proposes from the transition.
#include "internal.cuh"
#include "model_body.cuh"
#include "batch.cuh"
#include "mlp.cuh"
#include "proposal.cuh"
#include "guided_tc.cuh"

namespace bpf {
namespace {

// Shared memory of k_pz_net: the three weight images, then per group its
// block's layer-1 input rows (128 x 16) and its activation tile (128 x 144:
// the hidden values in columns 0..127, constant-1 columns for the folded
// biases in 128..130).
constexpr uint32_t kNetW1B = kProposalHidden * kPZNetK1 * 2;  // 4 KB
constexpr uint32_t kNetW2B = kProposalHidden * kPZNetK2 * 2;  // 36 KB
constexpr uint32_t kNetW3B = kPZNetN3 * kPZNetK2 * 2;         // 4.5 KB
constexpr uint32_t kNetUB = 128 * kPZNetK1 * 2;               // 4 KB
constexpr uint32_t kNetAB = 128 * kPZNetK2 * 2;               // 36 KB
constexpr uint32_t kNetTileB = kNetUB + kNetAB;
constexpr int kNetGroups = 4;  // independent groups of 128 threads (one block each) per CTA
constexpr int kNetThreads = kGTile * kNetGroups;
constexpr int kNetSmem = (int)(kNetW1B + kNetW2B + kNetW3B + kNetGroups * kNetTileB) + 1024;  // + alignment slack

struct PZNetArgs {
  const double* x_in;
  int ld;
  const int* as;
  const double* y;  // nf observations
  const BatchFilter* filt;
  const int* blk2f;
  StepStats* stats;
  int blocks;
  const unsigned char* packed;  // the PZ images (ProposalNet::packed)
  int pk_w1, pk_w2, pk_w3;
  const float *b3, *shift, *scale;
  float2* O;  // (delta, raw s) per column
  int* err;
};

// barrier of one group (named barrier `id`, 128 threads) returning the AND
// of p over the group
__device__ __forceinline__ bool group_and(int id, bool p) {
  int r;
  asm volatile(
      "{\n\t"
      ".reg .pred p, q;\n\t"
      "setp.ne.s32 p, %1, 0;\n\t"
      "bar.red.and.pred q, %2, %3, p;\n\t"
      "selp.s32 %0, 1, 0, q;\n\t"
      "}\n"
      : "=r"(r)
      : "r"((int)p), "r"(id), "n"(kGTile)
      : "memory");
  return r != 0;
}

// the group's leader (when `wait`) waits for an mbarrier phase (the weight
// copy or an MMA chain); the group agrees on the outcome.  The proxy fence
// first makes every thread's shared-memory writes visible to the tensor
// core, the tcgen05 fences order the accumulator loads around the barrier.
__device__ __forceinline__ bool group_wait(int id, uint64_t* mb, uint32_t parity, bool ok, bool wait) {
  tc::fence_before_sync();
  tc::fence_proxy_async();
  bool mine = ok;
  if (wait && ok) mine = tc::mbar_wait(mb, parity, kGWaitCycles);
  const bool r = group_and(id, mine);
  tc::fence_after_sync();
  return r;
}

// one MMA chain D = A * W^T over K (a multiple of 16; the operands in the
// canonical K-major layout), committed to mb
template <int K, int N>
__device__ __forceinline__ void issue_chain(uint32_t tmem, const unsigned char* A, const unsigned char* W,
                                            uint64_t* mb) {
  constexpr uint32_t idesc = tc::idesc_bf16(128, N);
#pragma unroll
  for (int ks = 0; ks < K / 16; ++ks) {
    const uint64_t ad = tc::smem_desc(tc::smem_u32(A) + ks * 256, 128, K * 16);
    const uint64_t bd = tc::smem_desc(tc::smem_u32(W) + ks * 256, 128, K * 16);
    tc::mma_bf16(tmem, ad, bd, idesc, ks > 0 ? 1u : 0u);
  }
  tc::mma_commit(mb);
}

// this thread's accumulator row (128 columns) + ReLU as BF16 into row r of
// its activation tile (the bias came in through the constant-1 columns)
__device__ __forceinline__ void relu_row(uint32_t trow, unsigned char* sA, int r) {
#pragma unroll 1
  for (int n0 = 0; n0 < kProposalHidden; n0 += 32) {
    float v[32];
    tc::tmem_ld32(trow + (uint32_t)n0, v);
#pragma unroll
    for (int j = 0; j < 32; ++j) v[j] = fmaxf(v[j], 0.0f);
#pragma unroll
    for (int c = 0; c < 4; ++c)
      *reinterpret_cast<uint4*>(sA + tc::kmajor_off(r, n0 + 8 * c, kPZNetK2)) = pack8(v + 8 * c);
  }
}

// The network of every particle of the batch (after its ancestor gather),
// all three layers on the tensor cores.  A CTA (one per SM, persistent)
// holds the weight images once and four independent groups of 128 threads;
// thread r of group g owns particle r of the group's block (TMEM lane r,
// columns 128 g ..).  Per block a group writes its input rows [u, 1, 1, 1]
// (BF16), then runs
//   layer 1  128 x 128 x 16   (b1 folded in), ReLU -> activation tile
//   layer 2  128 x 128 x 144  (b2 folded in), ReLU -> activation tile
//   layer 3  128 x 16 x 144   (W3 padded to 16 rows), + b3 in FP32,
// each an MMA chain its leader issues and waits for; while one group waits
// for the tensor core the others compute.  The inputs of the group's next
// block are fetched in stages across these waits: its ancestor index while
// layer 1 runs, its state while layer 2 runs, its features while layer 3
// runs.
__global__ void __launch_bounds__(kNetThreads, 1) k_pz_net(PZNetArgs a) {
  constexpr int H = kProposalHidden;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  unsigned char* sW1 = smem;
  unsigned char* sW2 = sW1 + kNetW1B;
  unsigned char* sW3 = sW2 + kNetW2B;
  __shared__ uint64_t wbar, mbar[kNetGroups];
  __shared__ uint32_t s_taddr;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int g = tid / kGTile, r = tid % kGTile;
  const bool leader = r == 0;
  unsigned char* sU = sW3 + kNetW3B + (size_t)g * kNetTileB;  // the group's input rows
  unsigned char* sA = sU + kNetUB;                             // and activation tile
  if (warp == 0) tc::tmem_alloc(&s_taddr, 512);
  if (tid == 0) {
    tc::mbar_init(&wbar, 1);
    for (int q = 0; q < kNetGroups; ++q) tc::mbar_init(&mbar[q], 1);
  }
  // the constant-1 columns of this thread's activation row (128..130 ones,
  // 131..143 zeros), never overwritten
  {
    const float one[8] = {1.0f, 1.0f, 1.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    *reinterpret_cast<uint4*>(sA + tc::kmajor_off(r, H, kPZNetK2)) = pack8(one);
    *reinterpret_cast<uint4*>(sA + tc::kmajor_off(r, H + 8, kPZNetK2)) = make_uint4(0u, 0u, 0u, 0u);
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t taddr = s_taddr;
  const uint32_t tg = taddr + (uint32_t)(128 * g);  // the group's accumulator
  const uint32_t trow = tg + ((uint32_t)((warp & 3) * 32) << 16);
  if (tid == 0) {
    tc::mbar_expect_tx(&wbar, kNetW1B + kNetW2B + kNetW3B);
    tc::bulk_g2s(sW1, a.packed + a.pk_w1, kNetW1B, &wbar);
    tc::bulk_g2s(sW2, a.packed + a.pk_w2, kNetW2B, &wbar);
    tc::bulk_g2s(sW3, a.packed + a.pk_w3, kNetW3B, &wbar);
  }
  const float sh0 = __ldg(a.shift), sh1 = __ldg(a.shift + 1), sh2 = __ldg(a.shift + 2);
  const float sc0 = __ldg(a.scale), sc1 = __ldg(a.scale + 1), sc2 = __ldg(a.scale + 2);
  const float b30 = __ldg(a.b3), b31 = __ldg(a.b3 + 1);
  const int bar = 1 + g;
  const int stride = gridDim.x * kNetGroups;
  // stage 1 of a block's inputs: its filter, column and ancestor index
  int nf_ = 0, ncol = 0, nsrc = 0, noff = 0;
  bool nlive = false;
  auto stage1 = [&](int blk) {
    nlive = false;
    if (blk < a.blocks) {
      nf_ = __ldg(a.blk2f + blk);
      const int n = a.filt[nf_].n;
      noff = a.filt[nf_].off;
      const int p = (blk - a.filt[nf_].block0) * kGTile + r;
      nlive = p < n;
      ncol = noff + p;
      if (nlive) nsrc = a.stats[nf_].resample ? min(max(__ldg(a.as + ncol), 0), n - 1) : p;
    }
  };
  // stage 2: its state; stage 3: its features
  double nP = 1.0, nZ = 1.0;
  auto stage2 = [&]() {
    if (nlive) {
      nP = __ldg(a.x_in + noff + nsrc);
      nZ = __ldg(a.x_in + (size_t)a.ld + noff + nsrc);
    }
  };
  float nu[3] = {0.0f, 0.0f, 0.0f};
  auto stage3 = [&]() {
    if (nlive) {
      const double lp = bpf_log(nP);
      nu[0] = ((float)lp - sh0) * sc0;
      nu[1] = ((float)bpf_log(nZ) - sh1) * sc1;
      nu[2] = ((float)(__ldg(a.y + nf_) - lp) - sh2) * sc2;
    }
  };
  int it = blockIdx.x * kNetGroups + g;
  stage1(it);
  stage2();
  stage3();
  bool ok = true, wready = false;
  uint32_t phase = 0;
  for (; it < a.blocks; it += stride) {
    const int f = nf_, col = ncol;
    const bool live = nlive;
    {
      const float u[8] = {nu[0], nu[1], nu[2], 1.0f, 1.0f, 1.0f, 0.0f, 0.0f};
      *reinterpret_cast<uint4*>(sU + tc::kmajor_off(r, 0, kPZNetK1)) = pack8(u);
      *reinterpret_cast<uint4*>(sU + tc::kmajor_off(r, 8, kPZNetK1)) = make_uint4(0u, 0u, 0u, 0u);
    }
    // layer 1 (the first time, after the weight images have landed)
    ok = group_wait(bar, &wbar, 0u, ok, leader && !wready);
    wready = true;
    if (ok && leader) issue_chain<kPZNetK1, H>(tg, sU, sW1, &mbar[g]);
    stage1(it + stride);
    ok = group_wait(bar, &mbar[g], phase, ok, leader);
    phase ^= 1u;
    if (ok) relu_row(trow, sA, r);
    // layer 2
    ok = group_wait(bar, &mbar[g], phase, ok, false);  // no wait: the fences and the barrier only
    if (ok && leader) issue_chain<kPZNetK2, H>(tg, sA, sW2, &mbar[g]);
    stage2();
    ok = group_wait(bar, &mbar[g], phase, ok, leader);
    phase ^= 1u;
    if (ok) relu_row(trow, sA, r);
    // layer 3
    ok = group_wait(bar, &mbar[g], phase, ok, false);
    if (ok && leader) issue_chain<kPZNetK2, kPZNetN3>(tg, sA, sW3, &mbar[g]);
    stage3();
    ok = group_wait(bar, &mbar[g], phase, ok, leader);
    phase ^= 1u;
    if (!ok) {
      // a wait gave up: this block's filter stops (and so does the filter
      // of every later block of this group)
      if (live && r == 0) a.stats[f].status = BPF_E_TIMEOUT;
      continue;
    }
    uint32_t v0, v1;
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%2];" : "=r"(v0), "=r"(v1) : "r"(trow));
    asm volatile("tcgen05.wait::ld.sync.aligned;" : "+r"(v0), "+r"(v1) : : "memory");
    if (live) a.O[col] = make_float2(__uint_as_float(v0) + b30, __uint_as_float(v1) + b31);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(taddr, 512);
  if (!ok && tid == 0) atomicExch(a.err, 1);
}

// the step: proposal draw, ODE, observation and weight correction, per
// filter reduction tail (the batched PZ transition's layout)
__global__ void __launch_bounds__(kPZBlock)
k_batch_pz_guided(const double* __restrict__ x_in, double* __restrict__ x_out, int ld, int* __restrict__ as,
                  double* __restrict__ lw, const double* __restrict__ y, double t1d, double t2d, int step,
                  const BatchFilter* __restrict__ filt, const PZParams* __restrict__ prms,
                  const int* __restrict__ blk2f, StepStats* stats, LwPartial* partials, unsigned* counters,
                  double* hist, int nf, int k, const float2* __restrict__ O) {
  const int f = __ldg(blk2f + blockIdx.x);
  const BatchFilter fd = filt[f];
  StepStats* st = stats + f;
  const int p = (blockIdx.x - fd.block0) * kPZBlock + threadIdx.x;
  const int resampled = st->resample;
  const bool ok = st->status == BPF_OK;
  const PZParams prm = prms[f];
  LwPartial part = lw_empty();
  if (ok && p < fd.n) {
    const int col = fd.off + p;
    const int src = resampled ? min(max(as[col], 0), fd.n - 1) : p;
    double P = __ldg(x_in + fd.off + src), Z = __ldg(x_in + (size_t)ld + fd.off + src);
    const float2 o = O[col];
    const double delta = (double)o.x;
    const double s = (double)fminf(fmaxf(o.y, kSMin), kSMax);
    // the standard normal of the particle's transition draw (pz_alpha's)
    const bpf_u32x4 r = bpf_draw(fd.seed, (uint32_t)p, (uint32_t)step, 0u, BPF_RNG_NOISE);
    double z0, z1;
    bpf_normal_pair_d(r.v[0], r.v[1], &z0, &z1);
    const double la = __fma_rn(bpf_exp(s), z0, prm.mu + delta);
    pz_advance<double>(P, Z, bpf_exp(la), t1d, t2d, prm);
    double l = resampled ? st->ll : lw[col];
    l += pz_obs_term<double>(P, __ldg(y + f), prm);
    const double u = (la - prm.mu) / prm.sigma;
    l += __fma_rn(-0.5, u * u, -bpf_log(prm.sigma)) + __fma_rn(0.5, z0 * z0, s);
    x_out[col] = P;
    x_out[(size_t)ld + col] = Z;
    lw[col] = l;
    if (resampled) as[col] = src;
    lw_push(part, l);
  }
  if (transition_reduce_tail(part, partials, blockIdx.x, fd.block0, fd.nblocks, counters + f, fd.n, st, ok,
                             resampled, true))
    batch_record(st, hist, nf, f, k);
}

}  // namespace

int launch_batch_pz_guided(ProposalNet& net, const BatchPZGuidedArgs& a, cudaStream_t st) {
  if (!net.pz || !a.O || !a.y) return BPF_E_INVALID;
  // the images are copied in bulk: 16-byte aligned starts
  if (((reinterpret_cast<uintptr_t>(net.packed) | (uintptr_t)net.pk_w1 | (uintptr_t)net.pk_w2 |
        (uintptr_t)net.pk_w3) & 15) != 0)
    return BPF_E_INVALID;
  static unsigned configured = 0;
  BPF_TRY(set_dyn_smem_once(k_pz_net, kNetSmem, configured));
  static int sms[64] = {0};
  int dev = 0;
  BPF_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return BPF_E_INVALID;
  if (!sms[dev]) BPF_TRY(cudaDeviceGetAttribute(&sms[dev], cudaDevAttrMultiProcessorCount, dev));
  PZNetArgs n;
  n.x_in = a.x_in;
  n.ld = a.ld;
  n.as = a.as;
  n.y = a.y;
  n.filt = a.filt;
  n.blk2f = a.blk2f;
  n.stats = a.stats;
  n.blocks = a.blocks;
  n.packed = net.packed;
  n.pk_w1 = net.pk_w1;
  n.pk_w2 = net.pk_w2;
  n.pk_w3 = net.pk_w3;
  n.b3 = net.b3();
  n.shift = net.shift;
  n.scale = net.scale;
  n.O = a.O;
  n.err = net.err;
  // one CTA per SM (its 206 KB of shared memory and 512 TMEM columns)
  const int need = (a.blocks + kNetGroups - 1) / kNetGroups;
  const int grid = need < sms[dev] ? need : sms[dev];
  k_pz_net<<<grid, kNetThreads, kNetSmem, st>>>(n);
  BPF_TRY(cudaGetLastError());
  k_batch_pz_guided<<<a.blocks, kPZBlock, 0, st>>>(a.x_in, a.x_out, a.ld, a.as, a.lw, a.y, a.t1, a.t2, a.step,
                                                   a.filt, a.prms, a.blk2f, a.stats, a.partials, a.counters,
                                                   a.hist, a.nf, a.k, a.O);
  BPF_TRY(cudaGetLastError());
  return BPF_OK;
}

}  // namespace bpf
