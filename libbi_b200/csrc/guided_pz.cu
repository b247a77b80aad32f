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
//                 CTA loads the layer-1 and layer-2 weight images once
//                 (bulk copies, 36 KB), then for each 128-particle block of
//                 the batch stages the standardised BF16 inputs (the three
//                 features padded to one K step of 16), runs layer 1
//                 (128 x 128 x 16) and layer 2 (128 x 128 x 128) as tcgen05
//                 MMAs into tensor memory with the bias/ReLU/BF16 epilogue
//                 between them, and computes the two outputs of layer 3 on
//                 the CUDA cores from its accumulator row (FP32 FMAs over
//                 BF16 weights): 8 bytes per particle leave the kernel,
//                 nothing of the hidden layers touches HBM;
//   k_batch_pz_guided  the batched PZ transition with the proposal's draw
//                 and the weight correction, ending in the same per-filter
//                 reduction tail.
// The ODE kernel keeps its own occupancy (FP64 RK4(3), 128 threads, no
// shared memory); the network kernel's occupancy is set by its 69 KB of
// shared memory (three CTAs per SM).  No counterpart in the reference,
// whose bootstrap filter proposes from the transition.
#include "internal.cuh"
#include "model_body.cuh"
#include "batch.cuh"
#include "mlp.cuh"
#include "proposal.cuh"
#include "guided_tc.cuh"

namespace bpf {
namespace {

constexpr int kNetK1 = 16;  // layer-1 K: the three inputs padded to one MMA K step
constexpr uint32_t kNetW1B = kProposalHidden * kNetK1 * 2;            // 4 KB
constexpr uint32_t kNetW2B = kProposalHidden * kProposalHidden * 2;   // 32 KB
constexpr int kNetSmem = (int)(kNetW1B + kNetW2B) + kGTileBytes + 1024;  // + alignment slack
constexpr int kNetCtasPerSm = 3;

struct PZNetArgs {
  const double* x_in;
  int ld;
  const int* as;
  const double* y;  // nf observations
  const BatchFilter* filt;
  const int* blk2f;
  StepStats* stats;
  int blocks;
  const unsigned char* packed;  // weight images (ProposalNet::packed)
  int pk_w1, pk_w2;
  const float *b1, *b2, *b3, *shift, *scale;
  const __nv_bfloat16* w3;  // layer-3 weights, 2 x 128 BF16
  float2* O;                // (delta, raw s) per column
  int* err;
};

// the network of every particle of the batch (after its ancestor gather)
__global__ void __launch_bounds__(kGTile, kNetCtasPerSm) k_pz_net(PZNetArgs a) {
  constexpr int H = kProposalHidden;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  unsigned char* sW1 = smem;
  unsigned char* sW2 = smem + kNetW1B;
  unsigned char* sA = sW2 + kNetW2B;  // the block's activation tile
  __shared__ float sW3[2 * H];
  __shared__ uint64_t mbar, wbar;
  __shared__ uint32_t s_taddr;
  const int tid = threadIdx.x, warp = tid >> 5;
  if (warp == 0) tc::tmem_alloc(&s_taddr, H);
  if (tid == 0) {
    tc::mbar_init(&mbar, 1);
    tc::mbar_init(&wbar, 1);
  }
  for (int k = tid; k < 2 * H; k += kGTile) sW3[k] = __bfloat162float(a.w3[k]);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t taddr = s_taddr;
  const uint32_t trow = taddr + ((uint32_t)(warp * 32) << 16);  // this warp's 32 lanes
  if (tid == 0) {
    tc::mbar_expect_tx(&wbar, kNetW1B + kNetW2B);
    tc::bulk_g2s(sW1, a.packed + a.pk_w1, kNetW1B, &wbar);
    tc::bulk_g2s(sW2, a.packed + a.pk_w2, kNetW2B, &wbar);
  }
  const float b30 = __ldg(a.b3), b31 = __ldg(a.b3 + 1);
  bool ok = true;
  uint32_t phase = 0;
  for (int blk = blockIdx.x; blk < a.blocks; blk += gridDim.x) {
    const int f = __ldg(a.blk2f + blk);
    const BatchFilter fd = a.filt[f];
    StepStats* st = a.stats + f;
    // one filter per block; another CTA may mark the filter timed out
    // meanwhile, so the CTA agrees on one reading
    if (!__syncthreads_and(st->status == BPF_OK)) continue;
    if (!ok) {
      // a wait of an earlier block gave up: this block's filter stops too
      if (tid == 0) st->status = BPF_E_TIMEOUT;
      continue;
    }
    const int p = (blk - fd.block0) * kGTile + tid;
    const bool live = p < fd.n;
    const int col = fd.off + p;
    float u[8] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    if (live) {
      const int src = st->resample ? min(max(a.as[col], 0), fd.n - 1) : p;
      const double P = __ldg(a.x_in + fd.off + src), Z = __ldg(a.x_in + (size_t)a.ld + fd.off + src);
      const double lp = bpf_log(P);
      const float v[3] = {(float)lp, (float)bpf_log(Z), (float)(__ldg(a.y + f) - lp)};
#pragma unroll
      for (int j = 0; j < 3; ++j) u[j] = (v[j] - __ldg(a.shift + j)) * __ldg(a.scale + j);
    }
    *reinterpret_cast<uint4*>(sA + tc::kmajor_off(tid, 0, kNetK1)) = pack8(u);
    *reinterpret_cast<uint4*>(sA + tc::kmajor_off(tid, 8, kNetK1)) = make_uint4(0u, 0u, 0u, 0u);
    // layer 1, then its epilogue as layer 2's A operand
    ok = weights_ready(&wbar, 0u, ok);
    if (ok && tid == 0) issue_layer<1, kNetK1, H>(taddr, sA, sW1, &mbar);
    ok = layer_done(&mbar, phase, ok);
    phase ^= 1u;
    if (!ok) {
      if (tid == 0) st->status = BPF_E_TIMEOUT;
      continue;
    }
    hidden_epilogue(trow, a.b1, sA, tid);
    ok = weights_ready(&wbar, 0u, ok);
    if (ok && tid == 0) issue_layer<1, H, H>(taddr, sA, sW2, &mbar);
    ok = layer_done(&mbar, phase, ok);
    phase ^= 1u;
    if (!ok) {
      if (tid == 0) st->status = BPF_E_TIMEOUT;
      continue;
    }
    // layer 2's epilogue (bias, ReLU, BF16) straight into layer 3's two
    // dot products
    float o0 = 0.0f, o1 = 0.0f;
#pragma unroll 1
    for (int n0 = 0; n0 < H; n0 += 16) {
      float v[16];
      tc::tmem_ld16(trow + (uint32_t)n0, v);
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const float h = __bfloat162float(__float2bfloat16(fmaxf(v[j] + __ldg(a.b2 + n0 + j), 0.0f)));
        o0 = fmaf(h, sW3[n0 + j], o0);
        o1 = fmaf(h, sW3[H + n0 + j], o1);
      }
    }
    if (live) a.O[col] = make_float2(o0 + b30, o1 + b31);
    // the next block's layer 1 overwrites these accumulators: every thread's
    // loads are done before thread 0 issues it (weights_ready's barrier)
    tc::fence_before_sync();
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(taddr, H);
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
  if (net.din != 3 || net.dout != 2 || net.hidden != kProposalHidden || net.k1 != kNetK1 || !a.O || !a.y)
    return BPF_E_INVALID;
  // the weight images are copied in bulk: 16-byte aligned starts
  if (((reinterpret_cast<uintptr_t>(net.packed) | (uintptr_t)net.pk_w1 | (uintptr_t)net.pk_w2) & 15) != 0)
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
  n.b1 = net.b1();
  n.b2 = net.b2();
  n.b3 = net.b3();
  n.shift = net.shift;
  n.scale = net.scale;
  n.w3 = net.params_h + net.o_w3;
  n.O = a.O;
  n.err = net.err;
  const int grid = a.blocks < kNetCtasPerSm * sms[dev] ? a.blocks : kNetCtasPerSm * sms[dev];
  k_pz_net<<<grid, kGTile, kNetSmem, st>>>(n);
  BPF_TRY(cudaGetLastError());
  k_batch_pz_guided<<<a.blocks, kPZBlock, 0, st>>>(a.x_in, a.x_out, a.ld, a.as, a.lw, a.y, a.t1, a.t2, a.step,
                                                   a.filt, a.prms, a.blk2f, a.stats, a.partials, a.counters,
                                                   a.hist, a.nf, a.k, a.O);
  BPF_TRY(cudaGetLastError());
  return BPF_OK;
}

}  // namespace bpf
