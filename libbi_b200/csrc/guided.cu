// The guided filter step: the bootstrap filter's predict + correct with the
// transition replaced by a learned proposal q(x_{t+1} | x_t, y_{t+1})
// (proposal.cu) and the weights corrected by importance sampling,
//   lw += log p(y | x') + log p(x' | x) - log q(x' | x, y),
// so the likelihood estimate stays unbiased.  For the Lorenz-96 model
// p(x' | x) = N(x'; m(x), sigma_eta^2 I) with m the deterministic RK4 step,
// and q = N(m(x) + delta, diag(exp(2 s))).  No counterpart in the reference;
// the resampling before it is the bootstrap filter's.
//
// One launch per step, one CTA per tile of 128 particles (thread r owns
// particle m0 + r, which is also TMEM lane r of the accumulator):
//   1. the layer-1 weights start streaming into shared memory; each thread
//      gathers its ancestor, runs the RK4 mean m (kept in registers) and
//      writes its network input row [x, y - m] (standardised, BF16) into the
//      canonical K-major A tile
//   2. three tcgen05 MMA chains 128 x 128 x 80, 128 x 128 x 128 and
//      128 x 80 x 128 into one 128-column FP32 accumulator; between them the
//      epilogue (bias, ReLU, BF16) moves the accumulator row of each thread
//      back into shared memory as the next layer's A tile while the next
//      layer's weights are staged
//   3. the last epilogue reads (delta, s) from tensor memory, draws
//      x' = m + delta + exp(s) z, writes x' and the weight, and pushes the
//      weight into the block partial of the log-weight reduction; the last
//      block finalises ESS, lW and the log-likelihood.
// Shared memory: three 32 KB tiles (weights, two activations), so two CTAs
// (256 TMEM columns) share an SM.
#include "internal.cuh"
#include "reduce.cuh"
#include "model_body.cuh"
#include "tc.cuh"
#include "proposal.cuh"

namespace bpf {

namespace {

constexpr int kGTile = 128;                        // particles per CTA
constexpr int kGTileBytes = 128 * 128 * 2;         // one BF16 tile
constexpr int kGSmem = 3 * kGTileBytes + 1024;     // + alignment slack
constexpr long long kGWaitCycles = 2000000000ll;   // ~1 s at 2 GHz

// rows x K BF16 matrix (K-contiguous rows, 16-byte aligned) into the
// canonical K-major layout with K columns
template <int ROWS, int K>
__device__ __forceinline__ void stage_weights(unsigned char* s, const __nv_bfloat16* __restrict__ w) {
  constexpr int C8 = K / 8;
#pragma unroll 2
  for (int e = threadIdx.x; e < ROWS * C8; e += kGTile) {
    const int r = e / C8, c = e % C8;
    const uint4 v = __ldg(reinterpret_cast<const uint4*>(w + r * K + 8 * c));
    *reinterpret_cast<uint4*>(s + tc::kmajor_off(r, 8 * c, K)) = v;
  }
}

// 8 FP32 values rounded to BF16, one 16-byte core-matrix row
__device__ __forceinline__ uint4 pack8(const float* v) {
  uint4 u;
  __nv_bfloat162 b;
  b = __floats2bfloat162_rn(v[0], v[1]); u.x = *reinterpret_cast<uint32_t*>(&b);
  b = __floats2bfloat162_rn(v[2], v[3]); u.y = *reinterpret_cast<uint32_t*>(&b);
  b = __floats2bfloat162_rn(v[4], v[5]); u.z = *reinterpret_cast<uint32_t*>(&b);
  b = __floats2bfloat162_rn(v[6], v[7]); u.w = *reinterpret_cast<uint32_t*>(&b);
  return u;
}

// one thread issues the MMA chain D = A * B^T over K (multiple of 16) and
// commits it to the mbarrier
template <int K, int N>
__device__ __forceinline__ void issue_layer(uint32_t taddr, const unsigned char* sA, const unsigned char* sB,
                                            uint64_t* mbar) {
  constexpr uint32_t idesc = tc::idesc_bf16(128, N);
  tc::fence_after_sync();
#pragma unroll
  for (int ks = 0; ks < K / 16; ++ks) {
    const uint64_t ad = tc::smem_desc(tc::smem_u32(sA) + ks * 256, 128, K * 16);
    const uint64_t bd = tc::smem_desc(tc::smem_u32(sB) + ks * 256, 128, K * 16);
    tc::mma_bf16(taddr, ad, bd, idesc, ks > 0 ? 1u : 0u);
  }
  tc::mma_commit(mbar);
}

// hidden-layer epilogue: this thread's accumulator row + bias, ReLU, BF16,
// into row r of the next layer's A tile (K = 128)
__device__ __forceinline__ void hidden_epilogue(uint32_t trow, const float* __restrict__ bias, unsigned char* sOut,
                                                int r) {
#pragma unroll 1
  for (int n0 = 0; n0 < kProposalHidden; n0 += 16) {
    float v[16];
    tc::tmem_ld16(trow + (uint32_t)n0, v);
#pragma unroll
    for (int j = 0; j < 16; ++j) v[j] = fmaxf(v[j] + __ldg(bias + n0 + j), 0.0f);
    *reinterpret_cast<uint4*>(sOut + tc::kmajor_off(r, n0, kProposalHidden)) = pack8(v);
    *reinterpret_cast<uint4*>(sOut + tc::kmajor_off(r, n0 + 8, kProposalHidden)) = pack8(v + 8);
  }
}

// wait for the MMA chain's commit; all threads agree on the outcome
__device__ __forceinline__ bool layer_done(uint64_t* mbar, uint32_t parity, bool ok) {
  const bool done = ok && tc::mbar_wait(mbar, parity, kGWaitCycles);
  ok = __syncthreads_and(done) != 0;
  tc::fence_after_sync();
  return ok;
}

template <int D>
__global__ void __launch_bounds__(kGTile, 2)
k_guided_fused(const float* __restrict__ x_in, float* __restrict__ x_out, int ld, int n,
               const int* __restrict__ as, double* __restrict__ lw, const float* __restrict__ y, double t1,
               double t2, uint64_t seed, int step, L96Params prm, StepStats* st, LwPartial* partials,
               unsigned* counter, const __nv_bfloat16* __restrict__ w1, const __nv_bfloat16* __restrict__ w2,
               const __nv_bfloat16* __restrict__ w3, const float* __restrict__ b1, const float* __restrict__ b2,
               const float* __restrict__ b3, const float* __restrict__ shift, const float* __restrict__ scale,
               int* err) {
  constexpr int DIN = 2 * D, DOUT = 2 * D, H = kProposalHidden;
  static_assert(DIN % 16 == 0 && DOUT % 16 == 0 && DIN <= H && DOUT <= H, "tile shapes");
  extern __shared__ unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  unsigned char* sW = smem;                    // weights of the current layer
  unsigned char* sX = smem + kGTileBytes;      // network input, then layer-2 output
  unsigned char* sY = smem + 2 * kGTileBytes;  // layer-1 output
  __shared__ uint64_t mbar;
  __shared__ uint32_t s_taddr;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int p = blockIdx.x * kGTile + tid;
  const int resampled = st->resample;
  const bool ok_in = st->status == BPF_OK;
  if (warp == 0) tc::tmem_alloc(&s_taddr, H);
  if (tid == 0) tc::mbar_init(&mbar, 1);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t taddr = s_taddr;
  const uint32_t trow = taddr + ((uint32_t)(warp * 32) << 16);  // this warp's 32 lanes
  LwPartial part = lw_empty();
  bool ok = ok_in;
  if (ok) {
    stage_weights<H, DIN>(sW, w1);
    // 1. ancestor, RK4 mean, network input row
    const bool live = p < n;
    const int src = live ? (resampled ? min(max(as[p], 0), n - 1) : p) : 0;
    float m[D], u[8];
#pragma unroll
    for (int i = 0; i < D; ++i) m[i] = live ? __ldg(x_in + (size_t)i * ld + src) : 0.0f;
#pragma unroll
    for (int c = 0; c < D / 8; ++c) {
#pragma unroll
      for (int j = 0; j < 8; ++j) u[j] = (m[8 * c + j] - __ldg(shift + 8 * c + j)) * __ldg(scale + 8 * c + j);
      *reinterpret_cast<uint4*>(sX + tc::kmajor_off(tid, 8 * c, DIN)) = pack8(u);
    }
    l96_rk4<float, D>(m, t1, t2, (float)prm.F, (float)prm.h);
#pragma unroll
    for (int c = 0; c < D / 8; ++c) {
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int i = 8 * c + j;
        u[j] = ((__ldg(y + i) - m[i]) - __ldg(shift + D + i)) * __ldg(scale + D + i);
      }
      *reinterpret_cast<uint4*>(sX + tc::kmajor_off(tid, D + 8 * c, DIN)) = pack8(u);
    }
    // 2. the network
    tc::fence_proxy_async();
    __syncthreads();
    if (tid == 0) issue_layer<DIN, H>(taddr, sX, sW, &mbar);
    ok = layer_done(&mbar, 0u, ok);
    if (ok) {
      stage_weights<H, H>(sW, w2);
      hidden_epilogue(trow, b1, sY, tid);
      tc::fence_before_sync();
      tc::fence_proxy_async();
      __syncthreads();
      if (tid == 0) issue_layer<H, H>(taddr, sY, sW, &mbar);
      ok = layer_done(&mbar, 1u, ok);
    }
    if (ok) {
      stage_weights<DOUT, H>(sW, w3);
      hidden_epilogue(trow, b2, sX, tid);
      tc::fence_before_sync();
      tc::fence_proxy_async();
      __syncthreads();
      if (tid == 0) issue_layer<H, DOUT>(taddr, sX, sW, &mbar);
      ok = layer_done(&mbar, 0u, ok);
    }
    // 3. the draw and the weight
    if (ok) {
      float o[DOUT];
#pragma unroll
      for (int n0 = 0; n0 < DOUT; n0 += 16) {
        float v[16];
        tc::tmem_ld16(trow + (uint32_t)n0, v);
#pragma unroll
        for (int j = 0; j < 16; ++j) o[n0 + j] = v[j] + __ldg(b3 + n0 + j);
      }
      if (live) {
        const float se = (float)prm.sigma_eta, ise = 1.0f / se, lse = logf(se);
        const float sy = (float)prm.sigma_y, isy = (float)prm.inv_sigma_y;
        const float c2 = (float)prm.c_half_log_2pi, ls = (float)prm.log_sigma_y;
        double l = resampled ? st->ll : lw[p];
        double corr = 0.0;  // log p(x' | x) - log q(x' | x, y), the 2 pi terms cancel
#pragma unroll
        for (int b = 0; b < (D + 3) / 4; ++b) {
          bpf_u32x4 r = bpf_draw(seed, (uint32_t)p, (uint32_t)step, (uint32_t)b, BPF_RNG_NOISE);
          float z[4];
          bpf_normal_pair_f(r.v[0], r.v[1], &z[0], &z[1]);
          bpf_normal_pair_f(r.v[2], r.v[3], &z[2], &z[3]);
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const int i = 4 * b + j;
            if (i < D) {
              const float delta = o[i];
              const float s = fminf(fmaxf(o[D + i], kSMin), kSMax);
              const float dx = delta + expf(s) * z[j];  // x' - m
              const float xi = m[i] + dx;
              x_out[(size_t)i * ld + p] = xi;
              const float e = dx * ise;
              corr += (double)(-0.5f * e * e - lse) - (double)(-0.5f * z[j] * z[j] - s);
              float dz = __ldg(y + i) - xi;
              dz = isy != 0.0f ? dz * isy : dz / sy;
              l += (double)(fmaf(-0.5f, dz * dz, -c2) - ls);
            }
          }
        }
        l += corr;
        lw[p] = l;
        lw_push(part, l);
      }
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(taddr, H);
  if (ok_in && !ok && tid == 0) atomicExch(err, 1);
  transition_reduce_tail(part, partials, blockIdx.x, 0, gridDim.x, counter, n, st, ok_in && ok, resampled, true);
}

}  // namespace

int launch_guided(ProposalNet& net, const GuidedArgs& a, cudaStream_t st) {
  if (a.n <= 0 || !a.y) return BPF_E_INVALID;  // the proposal needs the observation
  if (net.dim != 40 || net.hidden != kProposalHidden || net.din != 80 || net.dout != 80) return BPF_E_INVALID;
  // the dense weights are read with 16-byte loads
  const uintptr_t al = reinterpret_cast<uintptr_t>(net.w1h()) | reinterpret_cast<uintptr_t>(net.w2h()) |
                       reinterpret_cast<uintptr_t>(net.w3h());
  if (al & 15) return BPF_E_INVALID;
  const int blocks = (a.n + kGTile - 1) / kGTile;
  if (blocks > a.max_partials) return BPF_E_INVALID;
  static bool configured = false;
  if (!configured) {
    BPF_TRY(cudaFuncSetAttribute(k_guided_fused<40>, cudaFuncAttributeMaxDynamicSharedMemorySize, kGSmem));
    configured = true;
  }
  const L96Params prm = l96_params<float>(a.theta, a.h);
  k_guided_fused<40><<<blocks, kGTile, kGSmem, st>>>(
      (const float*)a.x_in, (float*)a.x_out, a.ld, a.n, a.as, a.lw, (const float*)a.y, a.t1, a.t2, a.seed, a.step,
      prm, a.stats, a.partials, a.counter, net.w1h(), net.w2h(), net.w3h(), net.b1(), net.b2(), net.b3(), net.shift,
      net.scale, net.err);
  BPF_TRY(cudaGetLastError());
  return BPF_OK;
}

}  // namespace bpf
