// The guided filter step: the bootstrap filter's predict + correct with the
// transition replaced by a learned proposal q(x_{t+1} | x_t, y_{t+1})
// (proposal.cu) and the weights corrected by importance sampling,
//   lw += log p(y | x') + log p(x' | x) - log q(x' | x, y),
// so the likelihood estimate stays unbiased.  For the Lorenz-96 model
// p(x' | x) = N(x'; m(x), sigma_eta^2 I) with m the deterministic RK4 step,
// and q = N(m(x) + delta, diag(exp(2 s))).  One step is five launches:
//   k_guided_prepare   gather the ancestor, RK4 mean m, network input row
//   3 x k_dense_tc     the network on the tensor cores (one 128-particle
//                      tile per CTA), output written structure-of-arrays
//   k_guided_finish    draw x' = m + delta + exp(s) z, the weight, the block
//                      partial of the log-weight reduction; the last block
//                      finalises ESS, lW and logLikelihood
// The resampling before it is the bootstrap filter's.  No counterpart in the
// reference.
#include "internal.cuh"
#include "reduce.cuh"
#include "model_body.cuh"
#include "mlp.cuh"
#include "proposal.cuh"

namespace bpf {

template <int D>
__global__ void __launch_bounds__(kL96Block, 8)
k_guided_prepare(const float* __restrict__ x_in, int ld, int n, const int* __restrict__ as,
                 const float* __restrict__ y, double t1, double t2, L96Params prm, const StepStats* st,
                 const float* __restrict__ shift, const float* __restrict__ scale, float* __restrict__ M,
                 __nv_bfloat16* __restrict__ U) {
  const int p = blockIdx.x * kL96Block + threadIdx.x;
  if (p >= n || st->status != BPF_OK) return;
  const int src = st->resample ? min(max(as[p], 0), n - 1) : p;
  __nv_bfloat16* u = U + (size_t)p * 2 * D;
  float m[D];
#pragma unroll
  for (int i = 0; i < D; ++i) {
    m[i] = __ldg(x_in + (size_t)i * ld + src);
    u[i] = __float2bfloat16((m[i] - __ldg(shift + i)) * __ldg(scale + i));
  }
  l96_rk4<float, D>(m, t1, t2, (float)prm.F, (float)prm.h);
#pragma unroll
  for (int i = 0; i < D; ++i) {
    M[(size_t)i * ld + p] = m[i];
    u[D + i] = __float2bfloat16(((__ldg(y + i) - m[i]) - __ldg(shift + D + i)) * __ldg(scale + D + i));
  }
}

template <int D>
__global__ void __launch_bounds__(kL96Block, 8)
k_guided_finish(float* __restrict__ x_out, int ld, int n, double* __restrict__ lw,
                const float* __restrict__ y, const float* __restrict__ M, const float* __restrict__ O,
                uint64_t seed, int step, L96Params prm, StepStats* st, LwPartial* partials, unsigned* counter) {
  const int p = blockIdx.x * kL96Block + threadIdx.x;
  const int resampled = st->resample;
  const bool ok = st->status == BPF_OK;
  LwPartial part = lw_empty();
  if (ok && p < n) {
    const float se = (float)prm.sigma_eta, ise = 1.0f / se, lse = logf(se);
    const float sy = (float)prm.sigma_y, isy = (float)prm.inv_sigma_y;
    const float c2 = (float)prm.c_half_log_2pi, ls = (float)prm.log_sigma_y;
    double l = resampled ? st->ll : lw[p];
    double corr = 0.0;  // log p(x' | x) - log q(x' | x, y), the 2 pi terms cancel
#pragma unroll 1
    for (int b = 0; b < (D + 3) / 4; ++b) {
      bpf_u32x4 r = bpf_draw(seed, (uint32_t)p, (uint32_t)step, (uint32_t)b, BPF_RNG_NOISE);
      float z[4];
      bpf_normal_pair_f(r.v[0], r.v[1], &z[0], &z[1]);
      bpf_normal_pair_f(r.v[2], r.v[3], &z[2], &z[3]);
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int i = 4 * b + j;
        if (i < D) {
          const float delta = O[(size_t)i * ld + p];
          const float s = fminf(fmaxf(O[(size_t)(D + i) * ld + p], kSMin), kSMax);
          const float dx = delta + expf(s) * z[j];  // x' - m
          const float xi = M[(size_t)i * ld + p] + dx;
          x_out[(size_t)i * ld + p] = xi;
          const float e = dx * ise;
          corr += (double)(-0.5f * e * e - lse) - (double)(-0.5f * z[j] * z[j] - s);
          if (y) {
            float dz = __ldg(y + i) - xi;
            dz = isy != 0.0f ? dz * isy : dz / sy;
            l += (double)(fmaf(-0.5f, dz * dz, -c2) - ls);
          }
        }
      }
    }
    l += corr;
    lw[p] = l;
    lw_push(part, l);
  }
  transition_reduce_tail(part, partials, blockIdx.x, 0, gridDim.x, counter, n, st, ok, resampled, y != nullptr);
}

static DenseArgs guided_dense(const __nv_bfloat16* A, int K, const __nv_bfloat16* W, const float* bias, int M,
                              int N, int relu, float* Df, long long df_rs, long long df_cs, __nv_bfloat16* Dh,
                              int* err) {
  DenseArgs g;
  g.A = A; g.a_rs = K; g.a_cs = 1;
  g.B = W; g.b_rs = K; g.b_cs = 1;
  g.M = M; g.N = N; g.K = K;
  g.bias = bias; g.relu = relu;
  g.Df = Df; g.df_rs = df_rs; g.df_cs = df_cs;
  g.Dh = Dh; g.dh_rs = N;
  g.err = err;
  return g;
}

int launch_guided(ProposalNet& net, const GuidedArgs& a, cudaStream_t st) {
  if (a.n <= 0 || !a.y) return BPF_E_INVALID;  // the proposal needs the observation
  const int blocks = (a.n + kL96Block - 1) / kL96Block;
  if (blocks > a.max_partials) return BPF_E_INVALID;
  const L96Params prm = l96_params<float>(a.theta, a.h);
  k_guided_prepare<40><<<blocks, kL96Block, 0, st>>>((const float*)a.x_in, a.ld, a.n, a.as, (const float*)a.y,
                                                     a.t1, a.t2, prm, a.stats, net.shift, net.scale, a.M, a.U);
  BPF_TRY(cudaGetLastError());
  const int H = net.hidden;
  int rc = launch_dense(guided_dense(a.U, net.din, net.w1h(), net.b1(), a.n, H, 1, nullptr, 0, 1, a.H1, net.err), st);
  if (!rc) rc = launch_dense(guided_dense(a.H1, H, net.w2h(), net.b2(), a.n, H, 1, nullptr, 0, 1, a.H2, net.err), st);
  // output structure-of-arrays: O(p, j) at O[j*ld + p]
  if (!rc) rc = launch_dense(guided_dense(a.H2, H, net.w3h(), net.b3(), a.n, net.dout, 0, a.O, 1, a.ld, nullptr,
                                          net.err), st);
  if (rc) return rc;
  k_guided_finish<40><<<blocks, kL96Block, 0, st>>>((float*)a.x_out, a.ld, a.n, a.lw, (const float*)a.y, a.M,
                                                    a.O, a.seed, a.step, prm, a.stats, a.partials, a.counter);
  BPF_TRY(cudaGetLastError());
  return BPF_OK;
}

}  // namespace bpf
