// Learned proposal for the Lorenz-96 filter: a small MLP, trained here on the
// GPU with the tensor-core dense layer (mlp.cu), that proposes
//   x_{t+1} ~ N(m(x_t) + delta, diag(exp(2 s))),   (delta, s) = MLP([x_t, y_{t+1} - m(x_t)]),
// where m(x_t) is the deterministic RK4 step of the model over the
// observation interval.  The network sees the particle state and the next
// observation as [x_t, y_{t+1} - m(x_t)] (the observation enters through its
// innovation against the transition's mean, so that the optimal correction
// is a near-linear function of the input; 2d values, standardised with the
// training data's per-feature mean and deviation),
// two hidden layers of 128 ReLU units, output (delta, s) (2d values); BF16
// weights and activations, FP32 accumulation, FP32 master weights and Adam.
// No counterpart in the reference (LibBi's bootstrap filter proposes from the
// transition); the guided filter step that uses it is in guided.cu.
//
// Training minimises the Gaussian negative log-likelihood of x_{t+1}:
//   L = mean_b sum_i [ s_i + (x_{t+1,i} - m_i - delta_i)^2 exp(-2 s_i) / 2 ],
// s clamped to [kSMin, kSMax] (zero gradient outside).  One step: gather a
// minibatch (indices from the counter-based stream, tag BPF_RNG_DATA),
// three dense layers forward, the loss gradient, five dense layers backward
// (weight gradients are dense layers over the batch dimension; the operands
// are read transposed through strides), bias gradients by column sums, and
// an Adam update that also refreshes the BF16 weight copies.
#include "internal.cuh"
#include "model_body.cuh"
#include "mlp.cuh"
#include "tc.cuh"
#include "proposal.cuh"

#include <cmath>
#include <new>
#include <vector>

namespace bpf {

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------
template <int D>
__global__ void k_rk4_mean(const float* __restrict__ x, float* __restrict__ m, int n, double dt, double F,
                           double h) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  float v[D];
#pragma unroll
  for (int i = 0; i < D; ++i) v[i] = x[(size_t)p * D + i];
  l96_rk4<float, D>(v, 0.0, dt, (float)F, (float)h);
#pragma unroll
  for (int i = 0; i < D; ++i) m[(size_t)p * D + i] = v[i];
}

// minibatch row b <- dataset row idx(b): standardised input [x_t, y - m]
// (BF16) and the regression target r0 = x_{t+1} - m(x_t)
__global__ void k_gather_batch(const float* __restrict__ xt, const float* __restrict__ mt,
                               const float* __restrict__ xt1, const float* __restrict__ yt1, int n, int D, int B,
                               uint64_t seed, int step, const float* __restrict__ shift,
                               const float* __restrict__ scale, __nv_bfloat16* U, float* r0) {
  const int b = blockIdx.x;
  if (b >= B) return;
  bpf_u32x4 w = bpf_draw(seed, (uint32_t)b, (uint32_t)step, 0u, BPF_RNG_DATA);
  const size_t row = (size_t)(((uint64_t)w.v[0] << 32 | w.v[1]) % (uint64_t)n);
  for (int j = threadIdx.x; j < 2 * D; j += blockDim.x) {
    const float v = j < D ? xt[row * D + j] : yt1[row * D + (j - D)] - mt[row * D + (j - D)];
    U[(size_t)b * 2 * D + j] = __float2bfloat16((v - shift[j]) * scale[j]);
  }
  for (int i = threadIdx.x; i < D; i += blockDim.x) r0[(size_t)b * D + i] = xt1[row * D + i] - mt[row * D + i];
}

// PZ training rows from states x_t (n x 2, FP64): the transition's log-noise
// la = mu + sigma z0 from its prior, the RK4(3) step over dt with
// alpha = exp(la), an observation y = log P' + sigma_y z1 (z0, z1 one
// Box-Muller pair of the data stream); inputs [log P, log Z, y - log P] and
// target la - mu
__global__ void k_pz_make_data(const double* __restrict__ xt, int n, uint64_t seed, PZParams prm, double dt,
                               float* __restrict__ feat, float* __restrict__ target) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  double P = xt[2 * (size_t)r], Z = xt[2 * (size_t)r + 1];
  const bpf_u32x4 w = bpf_draw(seed, (uint32_t)r, 1u, 0u, BPF_RNG_DATA);
  double z0, z1;
  bpf_normal_pair_d(w.v[0], w.v[1], &z0, &z1);
  const double la = __fma_rn(prm.sigma, z0, prm.mu);
  const double lp0 = bpf_log(P), lz0 = bpf_log(Z);
  pz_advance<double>(P, Z, bpf_exp(la), 0.0, dt, prm);
  const double y = __fma_rn(prm.sigma_y, z1, bpf_log(P));
  feat[3 * (size_t)r + 0] = (float)lp0;
  feat[3 * (size_t)r + 1] = (float)lz0;
  feat[3 * (size_t)r + 2] = (float)(y - lp0);
  target[r] = (float)(la - prm.mu);
}

// minibatch row b <- a precomputed training row (standardised BF16 inputs,
// FP32 targets)
__global__ void k_gather_rows(const float* __restrict__ feat, const float* __restrict__ target, int n, int din,
                              int D, int B, uint64_t seed, int step, const float* __restrict__ shift,
                              const float* __restrict__ scale, __nv_bfloat16* U, float* r0) {
  const int b = blockIdx.x;
  if (b >= B) return;
  bpf_u32x4 w = bpf_draw(seed, (uint32_t)b, (uint32_t)step, 0u, BPF_RNG_DATA);
  const size_t row = (size_t)(((uint64_t)w.v[0] << 32 | w.v[1]) % (uint64_t)n);
  for (int j = threadIdx.x; j < din; j += blockDim.x)
    U[(size_t)b * din + j] = __float2bfloat16((feat[row * din + j] - shift[j]) * scale[j]);
  for (int i = threadIdx.x; i < D; i += blockDim.x) r0[(size_t)b * D + i] = target[row * D + i];
}

__global__ void k_loss_grad(const float* __restrict__ O, const float* __restrict__ r0, int B, int D,
                            __nv_bfloat16* dO, double* loss_part) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  double l = 0.0;
  if (b < B) {
    const float invB = 1.0f / (float)B;
    for (int i = 0; i < D; ++i) {
      const float d = O[(size_t)b * 2 * D + i];
      const float sr = O[(size_t)b * 2 * D + D + i];
      const float s = fminf(fmaxf(sr, kSMin), kSMax);
      const float e = expf(-2.0f * s);
      const float r = r0[(size_t)b * D + i] - d;
      l += (double)(s + 0.5f * r * r * e);
      dO[(size_t)b * 2 * D + i] = __float2bfloat16(-r * e * invB);
      const bool inside = sr > kSMin && sr < kSMax;
      dO[(size_t)b * 2 * D + D + i] = __float2bfloat16(inside ? (1.0f - r * r * e) * invB : 0.0f);
    }
  }
  // block sum into this block's slot; k_loss_finish adds the slots in order
  __shared__ double s_l[8];
  for (int d = 16; d > 0; d >>= 1) l += __shfl_xor_sync(0xffffffffu, l, d);
  if ((threadIdx.x & 31) == 0) s_l[threadIdx.x >> 5] = l;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s_l[w];
    loss_part[blockIdx.x] = t;
  }
}

__global__ void k_loss_finish(const double* __restrict__ part, int nblocks, int B, double* loss) {
  double t = 0.0;
  for (int b = 0; b < nblocks; ++b) t += part[b];
  *loss = t / (double)B;
}

// dZ = dH where the layer's ReLU output is positive
__global__ void k_relu_back(const float* __restrict__ dH, const __nv_bfloat16* __restrict__ H, __nv_bfloat16* dZ,
                            size_t n) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dZ[i] = __float2bfloat16(__bfloat162float(H[i]) > 0.0f ? dH[i] : 0.0f);
}

// column sums out[j] = sum_b X[b, j] (the bias gradients) in a fixed order,
// so that training is reproducible: each block sums a chunk of kColChunk
// rows into part[block][j], then one block adds the chunks in block order
constexpr int kColChunk = 64;
__global__ void k_colsum(const __nv_bfloat16* __restrict__ X, int B, int N, float* __restrict__ part) {
  const int j = threadIdx.x;
  if (j >= N) return;
  const int r0 = blockIdx.x * kColChunk, r1 = min(B, r0 + kColChunk);
  float s = 0.0f;
  for (int r = r0; r < r1; ++r) s += __bfloat162float(X[(size_t)r * N + j]);
  part[(size_t)blockIdx.x * N + j] = s;
}

__global__ void k_colsum_finish(const float* __restrict__ part, int nchunks, int N, float* __restrict__ out) {
  const int j = threadIdx.x;
  if (j >= N) return;
  float s = 0.0f;
  for (int c = 0; c < nchunks; ++c) s += part[(size_t)c * N + j];
  out[j] = s;
}

static void colsum(const __nv_bfloat16* X, int B, int N, float* part, float* out, cudaStream_t st) {
  const int nchunks = (B + kColChunk - 1) / kColChunk;
  k_colsum<<<nchunks, 256, 0, st>>>(X, B, N, part);
  k_colsum_finish<<<1, 256, 0, st>>>(part, nchunks, N, out);
}

__global__ void k_adam(float* __restrict__ P, const float* __restrict__ G, float* __restrict__ M1,
                       float* __restrict__ M2, __nv_bfloat16* __restrict__ Ph, int n, float lr, float b1, float b2,
                       float eps, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float g = G[i];
  const float m = b1 * M1[i] + (1.0f - b1) * g;
  const float v = b2 * M2[i] + (1.0f - b2) * g * g;
  M1[i] = m;
  M2[i] = v;
  const float p = P[i] - lr * (m / c1) / (sqrtf(v / c2) + eps);
  P[i] = p;
  Ph[i] = __float2bfloat16(p);
}

// the three weight matrices into their shared-memory images
// (W1's image has k1 >= din columns, the ones past din zero from allocation)
__global__ void k_pack_weights(const __nv_bfloat16* __restrict__ Ph, int o_w1, int o_w2, int o_w3, int hidden,
                               int din, int k1, int dout, unsigned char* __restrict__ out, int pk_w1, int pk_w2,
                               int pk_w3) {
  const int n1 = hidden * din, n2 = hidden * hidden, n3 = dout * hidden;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n1) {
    *reinterpret_cast<__nv_bfloat16*>(out + pk_w1 + tc::kmajor_off(i / din, i % din, k1)) = Ph[o_w1 + i];
  } else if (i < n1 + n2) {
    const int j = i - n1;
    *reinterpret_cast<__nv_bfloat16*>(out + pk_w2 + tc::kmajor_off(j / hidden, j % hidden, hidden)) = Ph[o_w2 + j];
  } else if (i < n1 + n2 + n3) {
    const int j = i - n1 - n2;
    *reinterpret_cast<__nv_bfloat16*>(out + pk_w3 + tc::kmajor_off(j / hidden, j % hidden, hidden)) = Ph[o_w3 + j];
  }
}

// the FP32 value b as three BF16 pieces: piece j of hi + mid + lo
__device__ __forceinline__ __nv_bfloat16 bias_piece(float b, int j) {
  const __nv_bfloat16 hi = __float2bfloat16(b);
  if (j == 0) return hi;
  const float r1 = b - __bfloat162float(hi);
  const __nv_bfloat16 mid = __float2bfloat16(r1);
  if (j == 1) return mid;
  return __float2bfloat16(r1 - __bfloat162float(mid));
}

// the PZ network's images W1', W2', W3' (kPZNetK1 / kPZNetK2 columns)
__global__ void k_pack_pz(const __nv_bfloat16* __restrict__ Ph, const float* __restrict__ P, int o_w1, int o_b1,
                          int o_w2, int o_b2, int o_w3, unsigned char* __restrict__ out, int pk_w1, int pk_w2,
                          int pk_w3) {
  constexpr int H = kProposalHidden;
  constexpr int n1 = H * kPZNetK1, n2 = H * kPZNetK2, n3 = kPZNetN3 * kPZNetK2;
  const __nv_bfloat16 zero = __float2bfloat16(0.0f);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n1) {
    const int n = i / kPZNetK1, k = i % kPZNetK1;
    const __nv_bfloat16 v = k < 3 ? Ph[o_w1 + n * 3 + k] : k < 6 ? bias_piece(P[o_b1 + n], k - 3) : zero;
    *reinterpret_cast<__nv_bfloat16*>(out + pk_w1 + tc::kmajor_off(n, k, kPZNetK1)) = v;
  } else if (i < n1 + n2) {
    const int j = i - n1, n = j / kPZNetK2, k = j % kPZNetK2;
    const __nv_bfloat16 v = k < H ? Ph[o_w2 + n * H + k] : k < H + 3 ? bias_piece(P[o_b2 + n], k - H) : zero;
    *reinterpret_cast<__nv_bfloat16*>(out + pk_w2 + tc::kmajor_off(n, k, kPZNetK2)) = v;
  } else if (i < n1 + n2 + n3) {
    const int j = i - n1 - n2, n = j / kPZNetK2, k = j % kPZNetK2;
    const __nv_bfloat16 v = n < 2 && k < H ? Ph[o_w3 + n * H + k] : zero;
    *reinterpret_cast<__nv_bfloat16*>(out + pk_w3 + tc::kmajor_off(n, k, kPZNetK2)) = v;
  }
}

int pack_weights(ProposalNet& p, cudaStream_t st) {
  if (p.pz) {
    const int total = kProposalHidden * kPZNetK1 + kProposalHidden * kPZNetK2 + kPZNetN3 * kPZNetK2;
    k_pack_pz<<<(total + 255) / 256, 256, 0, st>>>(p.params_h, p.params, p.o_w1, p.o_b1, p.o_w2, p.o_b2, p.o_w3,
                                                   p.packed, p.pk_w1, p.pk_w2, p.pk_w3);
    BPF_TRY(cudaGetLastError());
    return BPF_OK;
  }
  const int total = p.hidden * p.din + p.hidden * p.hidden + p.dout * p.hidden;
  k_pack_weights<<<(total + 255) / 256, 256, 0, st>>>(p.params_h, p.o_w1, p.o_w2, p.o_w3, p.hidden, p.din, p.k1,
                                                      p.dout, p.packed, p.pk_w1, p.pk_w2, p.pk_w3);
  BPF_TRY(cudaGetLastError());
  return BPF_OK;
}

__global__ void k_to_bf16(const float* __restrict__ P, __nv_bfloat16* Ph, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) Ph[i] = __float2bfloat16(P[i]);
}

// ---------------------------------------------------------------------------
// forward and backward of one minibatch (U, r0 already in place)
// ---------------------------------------------------------------------------
static DenseArgs dense(const __nv_bfloat16* A, long long a_rs, long long a_cs, const __nv_bfloat16* B,
                       long long b_rs, long long b_cs, int M, int N, int K, const float* bias, int relu, float* Df,
                       __nv_bfloat16* Dh, int* err) {
  DenseArgs g;
  g.A = A; g.a_rs = a_rs; g.a_cs = a_cs;
  g.B = B; g.b_rs = b_rs; g.b_cs = b_cs;
  g.M = M; g.N = N; g.K = K;
  g.bias = bias; g.relu = relu;
  g.Df = Df; g.df_rs = N; g.df_cs = 1;
  g.Dh = Dh; g.dh_rs = N;
  g.err = err;
  return g;
}

// a training layer, with the split-K workspace
static int run_dense(ProposalNet& p, DenseArgs g, cudaStream_t st) {
  g.ws = p.ws;
  g.ws_floats = p.ws_floats;
  return launch_dense(g, st);
}

int proposal_forward(ProposalNet& p, const __nv_bfloat16* U, int B, __nv_bfloat16* H1, __nv_bfloat16* H2, float* O,
                     cudaStream_t st) {
  const int din = p.din, H = p.hidden, dout = p.dout;
  int rc = run_dense(p, dense(U, din, 1, p.w1h(), din, 1, B, H, din, p.b1(), 1, nullptr, H1, p.err), st);
  if (!rc) rc = run_dense(p, dense(H1, H, 1, p.w2h(), H, 1, B, H, H, p.b2(), 1, nullptr, H2, p.err), st);
  if (!rc) rc = run_dense(p, dense(H2, H, 1, p.w3h(), H, 1, B, dout, H, p.b3(), 0, O, nullptr, p.err), st);
  return rc;
}

static int loss_and_grad(ProposalNet& p, int B, cudaStream_t st) {
  const int din = p.din, H = p.hidden, dout = p.dout, D = p.dim;
  int rc = proposal_forward(p, p.U, B, p.H1, p.H2, p.O, st);
  if (rc) return rc;
  BPF_TRY(cudaMemsetAsync(p.grads, 0, (size_t)p.nparams * sizeof(float), st));
  const int lblocks = (B + 255) / 256;
  k_loss_grad<<<lblocks, 256, 0, st>>>(p.O, p.r0, B, D, p.dO, p.loss_part);
  k_loss_finish<<<1, 1, 0, st>>>(p.loss_part, lblocks, B, p.loss);
  float* g = p.grads;
  float *gW1 = g + p.o_w1, *gb1 = g + p.o_b1, *gW2 = g + p.o_w2, *gb2 = g + p.o_b2, *gW3 = g + p.o_w3,
        *gb3 = g + p.o_b3;
  // layer 3: O = H2 W3^T + b3
  rc = run_dense(p, dense(p.dO, 1, dout, p.H2, 1, H, dout, H, B, nullptr, 0, gW3, nullptr, p.err), st);
  if (rc) return rc;
  colsum(p.dO, B, dout, p.colpart, gb3, st);
  rc = run_dense(p, dense(p.dO, dout, 1, p.w3h(), 1, H, B, H, dout, nullptr, 0, p.dH, nullptr, p.err), st);
  if (rc) return rc;
  k_relu_back<<<(unsigned)(((size_t)B * H + 255) / 256), 256, 0, st>>>(p.dH, p.H2, p.dZ, (size_t)B * H);
  // layer 2: H2 = relu(H1 W2^T + b2)
  rc = run_dense(p, dense(p.dZ, 1, H, p.H1, 1, H, H, H, B, nullptr, 0, gW2, nullptr, p.err), st);
  if (rc) return rc;
  colsum(p.dZ, B, H, p.colpart, gb2, st);
  rc = run_dense(p, dense(p.dZ, H, 1, p.w2h(), 1, H, B, H, H, nullptr, 0, p.dH, nullptr, p.err), st);
  if (rc) return rc;
  k_relu_back<<<(unsigned)(((size_t)B * H + 255) / 256), 256, 0, st>>>(p.dH, p.H1, p.dZ, (size_t)B * H);
  // layer 1: H1 = relu(U W1^T + b1)
  rc = run_dense(p, dense(p.dZ, 1, H, p.U, 1, din, H, din, B, nullptr, 0, gW1, nullptr, p.err), st);
  if (rc) return rc;
  colsum(p.dZ, B, H, p.colpart, gb1, st);
  BPF_TRY(cudaGetLastError());
  return BPF_OK;
}

int ProposalNet::alloc(int d, int hid, int cap_batch, int din_) {
  dim = d;
  din = din_ > 0 ? din_ : 2 * d;
  dout = 2 * d;
  hidden = hid;
  o_w1 = 0;
  o_b1 = o_w1 + hidden * din;
  o_w2 = o_b1 + hidden;
  o_b2 = o_w2 + hidden * hidden;
  o_w3 = o_b2 + hidden;
  o_b3 = o_w3 + dout * hidden;
  nparams = o_b3 + dout;
  k1 = (din + 15) / 16 * 16;
  pz = din == 3 && dout == 2 && hidden == kProposalHidden;
  pk_w1 = 0;
  if (pz) {
    pk_w2 = pk_w1 + hidden * kPZNetK1 * 2;
    pk_w3 = pk_w2 + hidden * kPZNetK2 * 2;
    pk_bytes = pk_w3 + kPZNetN3 * kPZNetK2 * 2;
  } else {
    pk_w2 = pk_w1 + hidden * k1 * 2;
    pk_w3 = pk_w2 + hidden * hidden * 2;
    // W3's image holds whole 8-row core-matrix groups: dout rounded up to 16
    pk_bytes = pk_w3 + (dout + 15) / 16 * 16 * hidden * 2;
  }
  cap = cap_batch;
  auto A = [](void** p, size_t b) { return cudaMalloc(p, b) == cudaSuccess ? BPF_OK : BPF_E_NOMEM; };
  int rc = A((void**)&params, (size_t)nparams * 4);
  if (!rc) rc = A((void**)&params_h, (size_t)nparams * 2);
  if (!rc) rc = A((void**)&packed, (size_t)pk_bytes);
  if (!rc && cudaMemset(packed, 0, (size_t)pk_bytes) != cudaSuccess) rc = BPF_E_CUDA;  // W1's padding columns
  if (!rc) rc = A((void**)&grads, (size_t)nparams * 4);
  if (!rc) rc = A((void**)&m1, (size_t)nparams * 4);
  if (!rc) rc = A((void**)&m2, (size_t)nparams * 4);
  if (!rc) rc = A((void**)&shift, (size_t)din * 4);
  if (!rc) rc = A((void**)&scale, (size_t)din * 4);
  if (!rc) rc = A((void**)&err, sizeof(int));
  if (!rc) rc = A((void**)&loss, sizeof(double));
  if (!rc) rc = A((void**)&U, (size_t)cap * din * 2);
  if (!rc) rc = A((void**)&H1, (size_t)cap * hidden * 2);
  if (!rc) rc = A((void**)&H2, (size_t)cap * hidden * 2);
  if (!rc) rc = A((void**)&O, (size_t)cap * dout * 4);
  if (!rc) rc = A((void**)&dO, (size_t)cap * dout * 2);
  if (!rc) rc = A((void**)&dH, (size_t)cap * hidden * 4);
  if (!rc) rc = A((void**)&dZ, (size_t)cap * hidden * 2);
  if (!rc) rc = A((void**)&r0, (size_t)cap * dim * 4);
  if (!rc) rc = A((void**)&colpart, (size_t)((cap + kColChunk - 1) / kColChunk) * (hidden > dout ? hidden : dout) * 4);
  if (!rc) rc = A((void**)&loss_part, (size_t)((cap + 255) / 256) * sizeof(double));
  // room for one partial product per SM of the widest weight gradient
  ws_floats = 148ll * hidden * (hidden > din ? (hidden > dout ? hidden : dout) : (din > dout ? din : dout));
  if (!rc) rc = A((void**)&ws, (size_t)ws_floats * 4);
  if (rc) cudaGetLastError();
  return rc;
}

void ProposalNet::release() {
  void* ps[] = {params, params_h, packed, grads, m1, m2, shift, scale, err, loss, U, H1, H2, O, dO, dH, dZ, r0, mt,
                 colpart, loss_part, ws, feat, target};
  for (void* q : ps)
    if (q) cudaFree(q);
}

}  // namespace bpf

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
struct bpf_proposal {
  bpf::ProposalNet net;
  bpf_model_desc model;
  double dt = 0.0;
  uint64_t seed = 0;
  cudaStream_t stream = nullptr;
  // training data (caller-owned device arrays, n x d row-major)
  const float *xt = nullptr, *xt1 = nullptr, *yt1 = nullptr;
  int n = 0;
  int adam_step = 0;
  int train_step = 0;
};

namespace {

// He-uniform hidden layers; the output layer starts at zero weights with
// biases (0, log sigma_eta), so the untrained proposal is the transition
// itself (delta = 0, s = log sigma_eta) and the guided filter starts as the
// bootstrap filter
void init_params(bpf_proposal* q, std::vector<float>& P) {
  const bpf::ProposalNet& p = q->net;
  P.assign((size_t)p.nparams, 0.0f);
  auto u = [&](uint32_t i) {
    bpf_u32x4 w = bpf_draw(q->seed, i, 0u, 0u, BPF_RNG_DATA);
    return 2.0 * bpf_u01d(w.v[0], w.v[1]) - 1.0;
  };
  const double a1 = std::sqrt(6.0 / p.din), a2 = std::sqrt(6.0 / p.hidden);
  for (int i = 0; i < p.hidden * p.din; ++i) P[p.o_w1 + i] = (float)(a1 * u((uint32_t)(p.o_w1 + i)));
  for (int i = 0; i < p.hidden * p.hidden; ++i) P[p.o_w2 + i] = (float)(a2 * u((uint32_t)(p.o_w2 + i)));
  // the noise scale: sigma_eta of L96 (theta[1]), the log-noise deviation
  // sigma of PZ (theta[5])
  const double sn = q->model.kind == BPF_MODEL_PZ ? q->model.theta[5] : q->model.theta[1];
  for (int i = 0; i < p.dim; ++i) P[p.o_b3 + p.dim + i] = (float)std::log(sn > 0.0 ? sn : 1.0);
}

int upload_params(bpf_proposal* q, const float* P) {
  bpf::ProposalNet& p = q->net;
  BPF_TRY(cudaMemcpyAsync(p.params, P, (size_t)p.nparams * 4, cudaMemcpyHostToDevice, q->stream));
  bpf::k_to_bf16<<<(p.nparams + 255) / 256, 256, 0, q->stream>>>(p.params, p.params_h, p.nparams);
  BPF_TRY(cudaGetLastError());
  int rc = bpf::pack_weights(p, q->stream);
  if (rc) return rc;
  BPF_TRY(cudaStreamSynchronize(q->stream));
  return BPF_OK;
}

int check_err(bpf_proposal* q) {
  int e = 0;
  BPF_TRY(cudaMemcpyAsync(&e, q->net.err, sizeof(int), cudaMemcpyDeviceToHost, q->stream));
  BPF_TRY(cudaStreamSynchronize(q->stream));
  return e ? BPF_E_TIMEOUT : BPF_OK;
}

}  // namespace

extern "C" {

int bpf_proposal_create(const bpf_model_desc* model, double dt, int max_batch, uint64_t seed, void* stream,
                        bpf_proposal** out) {
  if (!out) return BPF_E_INVALID;
  *out = nullptr;
  if (!model || !(dt > 0.0) || !(model->h > 0.0) || max_batch < 128 || max_batch > (1 << 20)) return BPF_E_INVALID;
  const bool l96 = model->kind == BPF_MODEL_L96 && model->dim == 40 && model->precision == BPF_F32;
  const bool pz = model->kind == BPF_MODEL_PZ && model->dim == 2 && model->precision == BPF_F64 &&
                  model->integrator == BPF_ODE_RK43 && model->theta[5] > 0.0;
  if (!l96 && !pz) return BPF_E_INVALID;
  bpf_proposal* q = new (std::nothrow) bpf_proposal();
  if (!q) return BPF_E_NOMEM;
  q->model = *model;
  q->dt = dt;
  q->seed = seed;
  q->stream = (cudaStream_t)stream;
  // L96: the 40 state components from [x_t, y - m(x_t)] (80 inputs); PZ:
  // the one log-noise from [log P, log Z, y - log P]
  int rc = pz ? q->net.alloc(1, bpf::kProposalHidden, max_batch, 3)
              : q->net.alloc(model->dim, bpf::kProposalHidden, max_batch);
  std::vector<float> P;
  if (!rc) {
    init_params(q, P);
    rc = upload_params(q, P.data());
  }
  if (!rc) {
    std::vector<float> sh((size_t)q->net.din, 0.0f), sc((size_t)q->net.din, 1.0f);
    if (cudaMemcpy(q->net.shift, sh.data(), sh.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(q->net.scale, sc.data(), sc.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(q->net.err, 0, sizeof(int)) != cudaSuccess || cudaMemset(q->net.m1, 0, (size_t)q->net.nparams * 4) ||
        cudaMemset(q->net.m2, 0, (size_t)q->net.nparams * 4))
      rc = BPF_E_CUDA;
  }
  if (rc) {
    q->net.release();
    delete q;
    return rc;
  }
  *out = q;
  return BPF_OK;
}

int bpf_proposal_destroy(bpf_proposal* q) {
  if (!q) return BPF_OK;
  cudaStreamSynchronize(q->stream);
  q->net.release();
  delete q;
  return BPF_OK;
}

int bpf_proposal_set_states(bpf_proposal* q, const double* x_t, int n) {
  if (!q || !x_t || n <= 0 || q->model.kind != BPF_MODEL_PZ) return BPF_E_INVALID;
  bpf::ProposalNet& p = q->net;
  if (p.feat) cudaFree(p.feat);
  if (p.target) cudaFree(p.target);
  p.feat = p.target = nullptr;
  p.rows = 0;
  if (cudaMalloc((void**)&p.feat, (size_t)n * p.din * 4) != cudaSuccess ||
      cudaMalloc((void**)&p.target, (size_t)n * p.dim * 4) != cudaSuccess) {
    cudaGetLastError();
    return BPF_E_NOMEM;
  }
  p.rows = n;
  q->n = n;
  const bpf::PZParams prm = bpf::pz_params<double>(q->model.theta, q->model.h, q->model.atoler, q->model.rtoler);
  bpf::k_pz_make_data<<<(n + 127) / 128, 128, 0, q->stream>>>(x_t, n, q->seed, prm, q->dt, p.feat, p.target);
  BPF_TRY(cudaGetLastError());
  // input standardisation from (up to) the first 65536 rows
  const int ns = n < 65536 ? n : 65536;
  std::vector<float> h((size_t)ns * p.din);
  BPF_TRY(cudaMemcpyAsync(h.data(), p.feat, h.size() * 4, cudaMemcpyDeviceToHost, q->stream));
  BPF_TRY(cudaStreamSynchronize(q->stream));
  std::vector<float> sh((size_t)p.din), sc((size_t)p.din);
  for (int j = 0; j < p.din; ++j) {
    double s = 0.0, s2 = 0.0;
    for (int r = 0; r < ns; ++r) { const double v = h[(size_t)r * p.din + j]; s += v; s2 += v * v; }
    const double mean = s / ns, var = s2 / ns - mean * mean;
    sh[j] = (float)mean;
    sc[j] = (float)(1.0 / std::sqrt(var > 1e-12 ? var : 1.0));
  }
  BPF_TRY(cudaMemcpyAsync(p.shift, sh.data(), sh.size() * 4, cudaMemcpyHostToDevice, q->stream));
  BPF_TRY(cudaMemcpyAsync(p.scale, sc.data(), sc.size() * 4, cudaMemcpyHostToDevice, q->stream));
  BPF_TRY(cudaStreamSynchronize(q->stream));
  return BPF_OK;
}

int bpf_proposal_set_data(bpf_proposal* q, const float* x_t, const float* x_t1, const float* y_t1, int n) {
  if (!q || !x_t || !x_t1 || !y_t1 || n <= 0 || q->model.kind != BPF_MODEL_L96) return BPF_E_INVALID;
  bpf::ProposalNet& p = q->net;
  if (p.mt) cudaFree(p.mt);
  p.mt = nullptr;
  if (cudaMalloc((void**)&p.mt, (size_t)n * p.dim * 4) != cudaSuccess) { cudaGetLastError(); return BPF_E_NOMEM; }
  q->xt = x_t; q->xt1 = x_t1; q->yt1 = y_t1; q->n = n;
  bpf::k_rk4_mean<40><<<(n + 127) / 128, 128, 0, q->stream>>>(x_t, p.mt, n, q->dt, q->model.theta[0], q->model.h);
  BPF_TRY(cudaGetLastError());
  // input standardisation from (up to) the first 65536 rows of x_t and of
  // the innovation y - m
  const int ns = n < 65536 ? n : 65536;
  std::vector<float> hx((size_t)ns * p.dim), hy((size_t)ns * p.dim), hm((size_t)ns * p.dim);
  BPF_TRY(cudaMemcpyAsync(hx.data(), x_t, hx.size() * 4, cudaMemcpyDeviceToHost, q->stream));
  BPF_TRY(cudaMemcpyAsync(hy.data(), y_t1, hy.size() * 4, cudaMemcpyDeviceToHost, q->stream));
  BPF_TRY(cudaMemcpyAsync(hm.data(), p.mt, hm.size() * 4, cudaMemcpyDeviceToHost, q->stream));
  BPF_TRY(cudaStreamSynchronize(q->stream));
  for (size_t i = 0; i < hy.size(); ++i) hy[i] -= hm[i];
  std::vector<float> sh((size_t)p.din), sc((size_t)p.din);
  for (int j = 0; j < p.din; ++j) {
    const std::vector<float>& h = j < p.dim ? hx : hy;
    const int c = j < p.dim ? j : j - p.dim;
    double s = 0.0, s2 = 0.0;
    for (int r = 0; r < ns; ++r) { const double v = h[(size_t)r * p.dim + c]; s += v; s2 += v * v; }
    const double mean = s / ns, var = s2 / ns - mean * mean;
    sh[j] = (float)mean;
    sc[j] = (float)(1.0 / std::sqrt(var > 1e-12 ? var : 1.0));
  }
  BPF_TRY(cudaMemcpyAsync(p.shift, sh.data(), sh.size() * 4, cudaMemcpyHostToDevice, q->stream));
  BPF_TRY(cudaMemcpyAsync(p.scale, sc.data(), sc.size() * 4, cudaMemcpyHostToDevice, q->stream));
  BPF_TRY(cudaStreamSynchronize(q->stream));
  return BPF_OK;
}

int bpf_proposal_train(bpf_proposal* q, int steps, int batch, double lr, float* loss_trace) {
  if (!q || steps < 0 || batch < 1 || batch > q->net.cap || !(lr > 0.0) || q->n <= 0) return BPF_E_INVALID;
  bpf::ProposalNet& p = q->net;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  // learning rate: linear warm-up over the first 5% of the steps, then a
  // cosine decay to a tenth
  const int warm = steps / 20 > 1 ? steps / 20 : 1;
  for (int s = 0; s < steps; ++s) {
    const double w = s < warm ? (double)(s + 1) / warm : 1.0;
    const double c = 0.1 + 0.9 * 0.5 * (1.0 + std::cos(3.14159265358979323846 * s / (double)steps));
    const double lr_s = lr * w * c;
    if (p.feat)
      bpf::k_gather_rows<<<batch, 128, 0, q->stream>>>(p.feat, p.target, p.rows, p.din, p.dim, batch, q->seed,
                                                       q->train_step, p.shift, p.scale, p.U, p.r0);
    else
      bpf::k_gather_batch<<<batch, 128, 0, q->stream>>>(q->xt, p.mt, q->xt1, q->yt1, q->n, p.dim, batch, q->seed,
                                                        q->train_step, p.shift, p.scale, p.U, p.r0);
    int rc = bpf::loss_and_grad(p, batch, q->stream);
    if (rc) return rc;
    ++q->adam_step;
    ++q->train_step;
    const float c1 = 1.0f - std::pow(b1, (float)q->adam_step), c2 = 1.0f - std::pow(b2, (float)q->adam_step);
    bpf::k_adam<<<(p.nparams + 255) / 256, 256, 0, q->stream>>>(p.params, p.grads, p.m1, p.m2, p.params_h,
                                                               p.nparams, (float)lr_s, b1, b2, eps, c1, c2);
    BPF_TRY(cudaGetLastError());
    if (loss_trace) {
      double l = 0.0;
      BPF_TRY(cudaMemcpyAsync(&l, p.loss, sizeof(double), cudaMemcpyDeviceToHost, q->stream));
      BPF_TRY(cudaStreamSynchronize(q->stream));
      loss_trace[s] = (float)l;
    }
  }
  int rc = bpf::pack_weights(p, q->stream);
  if (rc) return rc;
  return check_err(q);
}

int bpf_proposal_loss_grad(bpf_proposal* q, const void* U, const float* r0, int batch, double* loss, float* grads) {
  if (!q || !U || !r0 || batch < 1 || batch > q->net.cap) return BPF_E_INVALID;
  bpf::ProposalNet& p = q->net;
  BPF_TRY(cudaMemcpyAsync(p.U, U, (size_t)batch * p.din * 2, cudaMemcpyDeviceToDevice, q->stream));
  BPF_TRY(cudaMemcpyAsync(p.r0, r0, (size_t)batch * p.dim * 4, cudaMemcpyDeviceToDevice, q->stream));
  int rc = bpf::loss_and_grad(p, batch, q->stream);
  if (rc) return rc;
  if (grads) BPF_TRY(cudaMemcpyAsync(grads, p.grads, (size_t)p.nparams * 4, cudaMemcpyDeviceToDevice, q->stream));
  double l = 0.0;
  BPF_TRY(cudaMemcpyAsync(&l, p.loss, sizeof(double), cudaMemcpyDeviceToHost, q->stream));
  BPF_TRY(cudaStreamSynchronize(q->stream));
  if (loss) *loss = l;
  return check_err(q);
}

int bpf_proposal_params(bpf_proposal* q, float* params, float* shift, float* scale, int* nparams) {
  if (!q) return BPF_E_INVALID;
  bpf::ProposalNet& p = q->net;
  if (nparams) *nparams = p.nparams;
  if (params) BPF_TRY(cudaMemcpyAsync(params, p.params, (size_t)p.nparams * 4, cudaMemcpyDeviceToHost, q->stream));
  if (shift) BPF_TRY(cudaMemcpyAsync(shift, p.shift, (size_t)p.din * 4, cudaMemcpyDeviceToHost, q->stream));
  if (scale) BPF_TRY(cudaMemcpyAsync(scale, p.scale, (size_t)p.din * 4, cudaMemcpyDeviceToHost, q->stream));
  BPF_TRY(cudaStreamSynchronize(q->stream));
  return BPF_OK;
}

int bpf_proposal_set_params(bpf_proposal* q, const float* params, const float* shift, const float* scale) {
  if (!q) return BPF_E_INVALID;
  bpf::ProposalNet& p = q->net;
  if (shift) BPF_TRY(cudaMemcpyAsync(p.shift, shift, (size_t)p.din * 4, cudaMemcpyHostToDevice, q->stream));
  if (scale) BPF_TRY(cudaMemcpyAsync(p.scale, scale, (size_t)p.din * 4, cudaMemcpyHostToDevice, q->stream));
  if (params) return upload_params(q, params);
  BPF_TRY(cudaStreamSynchronize(q->stream));
  return BPF_OK;
}

}  // extern "C"

namespace bpf {
ProposalNet* proposal_net(bpf_proposal* q) { return q ? &q->net : nullptr; }
double proposal_dt(bpf_proposal* q) { return q ? q->dt : 0.0; }
}  // namespace bpf
