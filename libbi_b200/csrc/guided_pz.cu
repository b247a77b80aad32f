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
// stays unbiased.  The network's three dense layers (BF16 operands, FP32
// accumulation, tensor cores: mlp.cu) run over all the batch's columns
// between an inputs kernel and the step kernel; the step kernel is the
// batched PZ transition with the proposal's draw and the weight correction,
// ending in the same per-filter reduction tail.  No counterpart in the
// reference, whose bootstrap filter proposes from the transition.
#include "internal.cuh"
#include "model_body.cuh"
#include "batch.cuh"
#include "mlp.cuh"
#include "proposal.cuh"

namespace bpf {
namespace {

// network inputs of every particle (after its ancestor gather)
__global__ void __launch_bounds__(kPZBlock)
k_batch_pz_guided_inputs(const double* __restrict__ x_in, int ld, const int* __restrict__ as,
                         const double* __restrict__ y, const BatchFilter* __restrict__ filt,
                         const int* __restrict__ blk2f, const StepStats* __restrict__ stats,
                         const float* __restrict__ shift, const float* __restrict__ scale, __nv_bfloat16* U) {
  const int f = __ldg(blk2f + blockIdx.x);
  const BatchFilter fd = filt[f];
  const StepStats* st = stats + f;
  const int p = (blockIdx.x - fd.block0) * kPZBlock + threadIdx.x;
  if (st->status != BPF_OK || p >= fd.n) return;
  const int col = fd.off + p;
  const int src = st->resample ? min(max(as[col], 0), fd.n - 1) : p;
  const double P = __ldg(x_in + fd.off + src), Z = __ldg(x_in + (size_t)ld + fd.off + src);
  const double lp = bpf_log(P);
  const float v[3] = {(float)lp, (float)bpf_log(Z), (float)(__ldg(y + f) - lp)};
#pragma unroll
  for (int j = 0; j < 3; ++j) U[(size_t)col * 3 + j] = __float2bfloat16((v[j] - shift[j]) * scale[j]);
}

// the step: proposal draw, ODE, observation and weight correction, per
// filter reduction tail (the batched PZ transition's layout)
__global__ void __launch_bounds__(kPZBlock)
k_batch_pz_guided(const double* __restrict__ x_in, double* __restrict__ x_out, int ld, int* __restrict__ as,
                  double* __restrict__ lw, const double* __restrict__ y, double t1d, double t2d, int step,
                  const BatchFilter* __restrict__ filt, const PZParams* __restrict__ prms,
                  const int* __restrict__ blk2f, StepStats* stats, LwPartial* partials, unsigned* counters,
                  double* hist, int nf, int k, const float* __restrict__ O) {
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
    const double delta = (double)O[(size_t)col * 2];
    const double s = (double)fminf(fmaxf(O[(size_t)col * 2 + 1], kSMin), kSMax);
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
  if (net.din != 3 || net.dout != 2 || !a.U || !a.H1 || !a.H2 || !a.O || !a.y) return BPF_E_INVALID;
  k_batch_pz_guided_inputs<<<a.blocks, kPZBlock, 0, st>>>(a.x_in, a.ld, a.as, a.y, a.filt, a.blk2f, a.stats,
                                                          net.shift, net.scale, a.U);
  BPF_TRY(cudaGetLastError());
  int rc = proposal_forward(net, a.U, a.ld, a.H1, a.H2, a.O, st);
  if (rc) return rc;
  k_batch_pz_guided<<<a.blocks, kPZBlock, 0, st>>>(a.x_in, a.x_out, a.ld, a.as, a.lw, a.y, a.t1, a.t2, a.step,
                                                   a.filt, a.prms, a.blk2f, a.stats, a.partials, a.counters,
                                                   a.hist, a.nf, a.k, a.O);
  BPF_TRY(cudaGetLastError());
  return BPF_OK;
}

}  // namespace bpf
