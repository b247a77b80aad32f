// The guided filter step: the bootstrap filter's predict + correct with the
// transition replaced by a learned proposal q(x_{t+1} | x_t, y_{t+1})
// (proposal.cu) and the weights corrected by importance sampling,
//   lw += log p(y | x') + log p(x' | x) - log q(x' | x, y),
// so the likelihood estimate stays unbiased.  For the Lorenz-96 model
// p(x' | x) = N(x'; m(x), sigma_eta^2 I) with m the deterministic RK4 step,
// and q = N(m(x) + delta, diag(exp(2 s))).  No counterpart in the reference;
// the resampling before it is the bootstrap filter's.
//
// One launch per step.  A CTA holds TILES tiles of 128 particles (thread
// 128 j + r owns particle r of tile j, which is TMEM lane r of that tile's
// accumulator, columns [128 j, 128 j + 128)):
//   1. one thread starts the bulk copy of the layer-1 weight image (packed
//      once in the canonical K-major layout) into shared memory; each thread
//      gathers its ancestor, runs the RK4 mean m (kept in registers) and
//      writes its network input row [x, y - m] (standardised, BF16) into its
//      tile's A operand
//   2. three tcgen05 MMA chains 128 x 128 x 80, 128 x 128 x 128 and
//      128 x 80 x 128 per tile; as soon as a layer's MMAs are done the next
//      layer's weights start copying, and the epilogue (bias, ReLU, BF16)
//      moves each thread's accumulator row back into its tile as the next
//      layer's A operand
//   3. the last epilogue reads (delta, s) from tensor memory eight
//      components at a time, draws x' = m + delta + exp(s) z, writes x' and
//      the weight, and pushes the weight into the block partial of the
//      log-weight reduction; the last block finalises ESS, lW and the
//      log-likelihood.
// Shared memory: the weight buffer and one 32 KB activation tile per 128
// particles.  TILES = 2 (256 threads, 96 KB, 256 TMEM columns, at most 128
// registers) puts 512 particles on an SM, so 65536 particles run in one wave
// on 148 SMs; TILES = 1 spreads small filters over more SMs.
//
// The same kernel runs the guided step of a batch of filters (BATCH = true,
// TILES = 1): CTA c takes tile c of the batch's 128-particle tiles, finds its
// filter through the tile -> filter table, and uses that filter's columns,
// seed, constants, statistics and partial slots; since a filter of a batch
// has at most 32768 particles, its single-filter step would also use one
// tile per CTA, so the batched step reproduces it bit for bit.
#include "internal.cuh"
#include "reduce.cuh"
#include "model_body.cuh"
#include "tc.cuh"
#include "proposal.cuh"
#include "batch.cuh"
#include "guided_tc.cuh"

namespace bpf {

namespace {

template <int TILES>
constexpr int guided_smem() { return (1 + TILES) * kGTileBytes + 1024; }  // + alignment slack

struct GuidedWeights {
  const unsigned char* packed;  // shared-memory images of W1, W2, W3
  int pk_w1, pk_w2, pk_w3;
  const float *b1, *b2, *b3, *shift, *scale;
};

// Launch arguments of both forms: one filter (the per-filter fields) or a
// batch (the per-filter fields come from the batch's tables).
struct GuidedKernelArgs {
  const float* x_in;
  float* x_out;
  int ld;
  int* as;
  double* lw;
  const float* y;
  double t1, t2;
  int step;
  GuidedWeights w;
  int* err;
  LwPartial* partials;
  // one filter
  int n;
  uint64_t seed;
  L96Params prm;
  StepStats* st;
  unsigned* counter;
  // a batch: filter f owns tiles [tile0_f, tile0_f + ntiles_f)
  const BatchFilter* filt;
  const L96Params* prms;
  const int* tile2f;
  StepStats* stats;
  unsigned* counters;
  double* hist;
  int nf, k;
};

template <int D, int TILES, bool BATCH>
__global__ void __launch_bounds__(kGTile * TILES, TILES == 1 ? 3 : 2) k_guided_fused(GuidedKernelArgs a) {
  constexpr int DIN = 2 * D, DOUT = 2 * D, H = kProposalHidden;
  constexpr uint32_t W1B = H * DIN * 2, W2B = H * H * 2, W3B = DOUT * H * 2;
  static_assert(DIN % 16 == 0 && DOUT % 16 == 0 && DIN <= H && DOUT <= H && D % 8 == 0, "tile shapes");
  static_assert(!BATCH || TILES == 1, "a batch CTA holds one tile of one filter");
  extern __shared__ unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  unsigned char* sW = smem;                // weights of the current layer
  unsigned char* sA = smem + kGTileBytes;  // TILES activation tiles
  __shared__ uint64_t mbar, wbar;
  __shared__ uint32_t s_taddr;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int tile = tid / kGTile, r = tid % kGTile;
  unsigned char* sT = sA + tile * kGTileBytes;  // this thread's tile
  // this CTA's filter: particles, first column, tiles before this CTA's
  // within the filter, partial slots, draws, constants and statistics
  int f = 0, n, off, tbase, pidx, pbase, np;
  uint64_t seed;
  L96Params prm;
  StepStats* st;
  unsigned* counter;
  const float* y;
  if (BATCH) {
    f = __ldg(a.tile2f + blockIdx.x);
    const BatchFilter fd = a.filt[f];
    n = fd.n;
    off = fd.off;
    tbase = blockIdx.x - fd.tile0;
    pidx = fd.block0 + tbase;
    pbase = fd.block0;
    np = fd.ntiles;
    seed = fd.seed;
    prm = a.prms[f];
    st = a.stats + f;
    counter = a.counters + f;
    y = a.y + (size_t)f * D;
  } else {
    n = a.n;
    off = 0;
    tbase = blockIdx.x * TILES;
    pidx = blockIdx.x;
    pbase = 0;
    np = gridDim.x;
    seed = a.seed;
    prm = a.prm;
    st = a.st;
    counter = a.counter;
    y = a.y;
  }
  const float* __restrict__ x_in = a.x_in;
  float* __restrict__ x_out = a.x_out;
  double* __restrict__ lw = a.lw;
  const int ld = a.ld, step = a.step;
  const GuidedWeights& w = a.w;
  const int p = (tbase + tile) * kGTile + r;  // particle within the filter
  const int col = off + p;
  const int resampled = st->resample;
  // one reading for the whole CTA (a CTA of the same filter that timed out
  // may be writing the status meanwhile)
  const bool ok_in = __syncthreads_and(st->status == BPF_OK) != 0;
  if (warp == 0) tc::tmem_alloc(&s_taddr, 128 * TILES);
  if (tid == 0) {
    tc::mbar_init(&mbar, 1);
    tc::mbar_init(&wbar, 1);
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t taddr = s_taddr;
  // this warp's 32 lanes of its tile's accumulator
  const uint32_t trow = taddr + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)(128 * tile);
  LwPartial part = lw_empty();
  bool ok = ok_in;
  if (ok) {
    if (tid == 0) {
      tc::mbar_expect_tx(&wbar, W1B);
      tc::bulk_g2s(sW, w.packed + w.pk_w1, W1B, &wbar);
    }
    // 1. ancestor, RK4 mean, network input row
    const bool live = p < n;
    const int src = live ? (resampled ? min(max(a.as[col], 0), n - 1) : p) : 0;
    if (BATCH && live && resampled) a.as[col] = src;
    float m[D], u[8];
#pragma unroll
    for (int i = 0; i < D; ++i) m[i] = live ? __ldg(x_in + (size_t)i * ld + off + src) : 0.0f;
#pragma unroll
    for (int c = 0; c < D / 8; ++c) {
#pragma unroll
      for (int j = 0; j < 8; ++j) u[j] = (m[8 * c + j] - __ldg(w.shift + 8 * c + j)) * __ldg(w.scale + 8 * c + j);
      *reinterpret_cast<uint4*>(sT + tc::kmajor_off(r, 8 * c, DIN)) = pack8(u);
    }
    l96_rk4<float, D>(m, a.t1, a.t2, (float)prm.F, (float)prm.h);
#pragma unroll
    for (int c = 0; c < D / 8; ++c) {
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int i = 8 * c + j;
        u[j] = ((__ldg(y + i) - m[i]) - __ldg(w.shift + D + i)) * __ldg(w.scale + D + i);
      }
      *reinterpret_cast<uint4*>(sT + tc::kmajor_off(r, D + 8 * c, DIN)) = pack8(u);
    }
    // 2. the network; the activations of each layer overwrite its input tile
    ok = weights_ready(&wbar, 0u, ok);
    if (ok && tid == 0) issue_layer<TILES, DIN, H>(taddr, sA, sW, &mbar);
    ok = layer_done(&mbar, 0u, ok);
    if (ok) {
      if (tid == 0) {
        tc::mbar_expect_tx(&wbar, W2B);
        tc::bulk_g2s(sW, w.packed + w.pk_w2, W2B, &wbar);
      }
      hidden_epilogue(trow, w.b1, sT, r);
      ok = weights_ready(&wbar, 1u, ok);
      if (ok && tid == 0) issue_layer<TILES, H, H>(taddr, sA, sW, &mbar);
      ok = layer_done(&mbar, 1u, ok);
    }
    if (ok) {
      if (tid == 0) {
        tc::mbar_expect_tx(&wbar, W3B);
        tc::bulk_g2s(sW, w.packed + w.pk_w3, W3B, &wbar);
      }
      hidden_epilogue(trow, w.b2, sT, r);
      ok = weights_ready(&wbar, 0u, ok);
      if (ok && tid == 0) issue_layer<TILES, H, DOUT>(taddr, sA, sW, &mbar);
      ok = layer_done(&mbar, 0u, ok);
    }
    // 3. the draw and the weight, eight components at a time.  The tile's
    //    activations are dead once layer 3 is done: m moves there (row r,
    //    FP32), so that the loop over components stays rolled (one copy of
    //    the draw in the instruction stream)
    if (ok) {
      float* mrow = reinterpret_cast<float*>(sT) + r * (D + 1);  // odd row stride: conflict-free
#pragma unroll
      for (int i = 0; i < D; ++i) mrow[i] = m[i];
      const float se = (float)prm.sigma_eta, ise = 1.0f / se, lse = logf(se);
      const float sy = (float)prm.sigma_y, isy = (float)prm.inv_sigma_y;
      const float c2 = (float)prm.c_half_log_2pi, ls = (float)prm.log_sigma_y;
      double l = live ? (resampled ? st->ll : lw[col]) : 0.0;
      double corr = 0.0;  // log p(x' | x) - log q(x' | x, y), the 2 pi terms cancel
#pragma unroll 1
      for (int c = 0; c < D / 8; ++c) {
        float dl[8], sr[8];
        tc::tmem_ld8(trow + (uint32_t)(8 * c), dl);
        tc::tmem_ld8(trow + (uint32_t)(D + 8 * c), sr);
        if (live) {
#pragma unroll 1
          for (int h = 0; h < 2; ++h) {
            bpf_u32x4 rr = bpf_draw(seed, (uint32_t)p, (uint32_t)step, (uint32_t)(2 * c + h), BPF_RNG_NOISE);
            float z[4];
            bpf_normal_pair_f(rr.v[0], rr.v[1], &z[0], &z[1]);
            bpf_normal_pair_f(rr.v[2], rr.v[3], &z[2], &z[3]);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              const int q = 4 * h + j, i = 8 * c + q;
              const float delta = (h ? dl[4 + j] : dl[j]) + __ldg(w.b3 + i);
              const float s = fminf(fmaxf((h ? sr[4 + j] : sr[j]) + __ldg(w.b3 + D + i), kSMin), kSMax);
              const float dx = delta + expf(s) * z[j];  // x' - m
              const float xi = mrow[i] + dx;
              x_out[(size_t)i * ld + col] = xi;
              const float e = dx * ise;
              corr += (double)(-0.5f * e * e - lse) - (double)(-0.5f * z[j] * z[j] - s);
              float dz = __ldg(y + i) - xi;
              dz = isy != 0.0f ? dz * isy : dz / sy;
              l += (double)(fmaf(-0.5f, dz * dz, -c2) - ls);
            }
          }
        }
      }
      if (live) {
        l += corr;
        lw[col] = l;
        lw_push(part, l);
      }
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(taddr, 128 * TILES);
  // a wait that gave up: the proposal's flag and the step's status (the
  // filter's next read of its statistics returns it)
  if (ok_in && !ok && tid == 0) {
    atomicExch(a.err, 1);
    st->status = BPF_E_TIMEOUT;
  }
  if (transition_reduce_tail(part, a.partials, pidx, pbase, np, counter, n, st, ok_in && ok, resampled, true) &&
      BATCH)
    batch_record(st, a.hist, a.nf, f, a.k);
}

template <int TILES, bool BATCH>
int launch_fused(const GuidedKernelArgs& ka, int blocks, cudaStream_t st) {
  static unsigned configured = 0;
  BPF_TRY(set_dyn_smem_once(k_guided_fused<40, TILES, BATCH>, guided_smem<TILES>(), configured));
  k_guided_fused<40, TILES, BATCH><<<blocks, kGTile * TILES, guided_smem<TILES>(), st>>>(ka);
  BPF_TRY(cudaGetLastError());
  return BPF_OK;
}

int check_net(const ProposalNet& net) {
  if (net.dim != 40 || net.hidden != kProposalHidden || net.din != 80 || net.dout != 80 || !net.packed)
    return BPF_E_INVALID;
  // the weight images are copied in bulk: 16-byte aligned starts and sizes
  if (((reinterpret_cast<uintptr_t>(net.packed) | (uintptr_t)net.pk_w1 | (uintptr_t)net.pk_w2 |
        (uintptr_t)net.pk_w3) & 15) != 0)
    return BPF_E_INVALID;
  return BPF_OK;
}

GuidedWeights weights_of(const ProposalNet& net) {
  return GuidedWeights{net.packed, net.pk_w1, net.pk_w2, net.pk_w3, net.b1(), net.b2(), net.b3(), net.shift,
                       net.scale};
}

}  // namespace

int launch_guided(ProposalNet& net, const GuidedArgs& a, cudaStream_t st) {
  if (a.n <= 0 || !a.y) return BPF_E_INVALID;  // the proposal needs the observation
  int rc = check_net(net);
  if (rc) return rc;
  GuidedKernelArgs ka{};
  ka.x_in = (const float*)a.x_in;
  ka.x_out = (float*)a.x_out;
  ka.ld = a.ld;
  ka.as = const_cast<int*>(a.as);
  ka.lw = a.lw;
  ka.y = (const float*)a.y;
  ka.t1 = a.t1;
  ka.t2 = a.t2;
  ka.step = a.step;
  ka.w = weights_of(net);
  ka.err = net.err;
  ka.partials = a.partials;
  ka.n = a.n;
  ka.seed = a.seed;
  ka.prm = l96_params<float>(a.theta, a.h);
  ka.st = a.stats;
  ka.counter = a.counter;
  // two tiles per CTA once single-tile CTAs would need more than one wave
  // at three CTAs per SM
  const int tiles = (a.n + kGTile - 1) / kGTile;
  const int tiles_per_cta = tiles > 3 * 148 ? 2 : 1;
  const int blocks = (tiles + tiles_per_cta - 1) / tiles_per_cta;
  if (blocks > a.max_partials) return BPF_E_INVALID;
  return tiles_per_cta == 2 ? launch_fused<2, false>(ka, blocks, st) : launch_fused<1, false>(ka, blocks, st);
}

int launch_batch_guided(ProposalNet& net, const BatchGuidedArgs& a, cudaStream_t st) {
  if (a.tiles <= 0 || !a.y || !a.tile2f) return BPF_E_INVALID;
  int rc = check_net(net);
  if (rc) return rc;
  GuidedKernelArgs ka{};
  ka.x_in = a.x_in;
  ka.x_out = a.x_out;
  ka.ld = a.ld;
  ka.as = a.as;
  ka.lw = a.lw;
  ka.y = a.y;
  ka.t1 = a.t1;
  ka.t2 = a.t2;
  ka.step = a.step;
  ka.w = weights_of(net);
  ka.err = net.err;
  ka.partials = a.partials;
  ka.filt = a.filt;
  ka.prms = a.prms;
  ka.tile2f = a.tile2f;
  ka.stats = a.stats;
  ka.counters = a.counters;
  ka.hist = a.hist;
  ka.nf = a.nf;
  ka.k = a.k;
  return launch_fused<1, true>(ka, a.tiles, st);
}

}  // namespace bpf
