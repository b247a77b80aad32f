// Dense layers on the fifth-generation tensor cores, the arithmetic of the
// learned proposal (forward inference inside the guided filter, forward and
// backward passes of its training).
//
// k_dense_tc computes, for one 128-row tile of A per CTA,
//   D[m, n] = act( sum_k A(m, k) * B(n, k) + bias[n] ),   n < N <= 256,
// with A and B read through arbitrary element strides (so transposed
// operands cost nothing extra), BF16 operands and FP32 accumulation in
// tensor memory.  The K dimension streams through shared memory in chunks of
// 64: the 128 threads stage a chunk in the canonical K-major layout, one
// thread issues four 128 x N x 16 MMAs and commits them to an mbarrier, and
// the chunk buffer is reused once that barrier's phase completes.  The
// epilogue reads each thread's accumulator row from tensor memory (warp w
// owns lanes 32w..32w+31), adds the bias, applies the activation and writes
// FP32 and/or BF16 results; row-major outputs go through shared memory so
// that warps write whole row segments.
//
// A layer with few row tiles and a long K (the weight gradients, K = the
// minibatch) splits K over a second grid dimension: each CTA writes its
// partial product to a workspace and k_splitk_reduce adds the partials in
// split order (deterministic) before the bias and activation.
#include "internal.cuh"
#include "tc.cuh"
#include "mlp.cuh"

#include <cuda_bf16.h>

namespace bpf {

constexpr int kTcKC = 64;                         // K per staged chunk
constexpr long long kTcWaitCycles = 2000000000ll;  // ~1 s at 2 GHz

// Stage rows [r0, r0 + ROWS) x columns [k0, k0 + KC) of an operand into the
// canonical K-major layout (zero outside rows < R, columns < K).  A
// K-contiguous operand with 16-byte aligned rows moves 8 elements per
// 16-byte load and store (a core-matrix row); a row-contiguous one (a
// transposed view) is read with consecutive threads on consecutive rows;
// any other goes element by element along K.
template <int ROWS>
__device__ __forceinline__ void stage_tile(unsigned char* sdst, const __nv_bfloat16* __restrict__ src, long long rs,
                                           long long cs, int r0, int R, int k0, int K, int vec, int rfast,
                                           __nv_bfloat16 zero) {
  constexpr int C8 = kTcKC / 8;
  if (vec) {
#pragma unroll 8
    for (int e = threadIdx.x; e < ROWS * C8; e += 128) {
      const int r = e / C8, c = e % C8;
      const int row = r0 + r, kk = k0 + 8 * c;
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      if (row < R) {
        if (kk + 8 <= K) {
          v = __ldg(reinterpret_cast<const uint4*>(src + row * rs + kk));
        } else if (kk < K) {
          __nv_bfloat16 t[8];
#pragma unroll
          for (int j = 0; j < 8; ++j) t[j] = kk + j < K ? src[row * rs + kk + j] : zero;
          v = *reinterpret_cast<const uint4*>(t);
        }
      }
      *reinterpret_cast<uint4*>(sdst + tc::kmajor_off(r, 8 * c, kTcKC)) = v;
    }
  } else if (rfast) {
#pragma unroll 8
    for (int e = threadIdx.x; e < ROWS * kTcKC; e += 128) {
      const int r = e % ROWS, k = e / ROWS;
      const int row = r0 + r, kk = k0 + k;
      const __nv_bfloat16 v = (row < R && kk < K) ? src[row * rs + kk * cs] : zero;
      *reinterpret_cast<__nv_bfloat16*>(sdst + tc::kmajor_off(r, k, kTcKC)) = v;
    }
  } else {
    for (int e = threadIdx.x; e < ROWS * kTcKC; e += 128) {
      const int r = e / kTcKC, k = e % kTcKC;
      const int row = r0 + r, kk = k0 + k;
      const __nv_bfloat16 v = (row < R && kk < K) ? src[row * rs + kk * cs] : zero;
      *reinterpret_cast<__nv_bfloat16*>(sdst + tc::kmajor_off(r, k, kTcKC)) = v;
    }
  }
}

__device__ __forceinline__ float dense_act(const DenseArgs& g, float x, int n) {
  x += g.bias ? __ldg(g.bias + n) : 0.0f;
  return g.relu ? fmaxf(x, 0.0f) : x;
}

template <int BN>
__global__ void __launch_bounds__(128) k_dense_tc(DenseArgs g) {
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char* sA = smem;                     // 128 x KC
  unsigned char* sB = smem + 128 * kTcKC * 2;   // BN x KC
  __shared__ uint64_t mbar;
  __shared__ uint32_t s_taddr;
  constexpr uint32_t NCOLS = BN <= 32 ? 32 : BN <= 64 ? 64 : BN <= 128 ? 128 : 256;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * 128;
  if (warp == 0) tc::tmem_alloc(&s_taddr, NCOLS);
  if (tid == 0) tc::mbar_init(&mbar, 1);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t taddr = s_taddr;
  constexpr uint32_t idesc = tc::idesc_bf16(128, BN);
  const __nv_bfloat16 zero = __float2bfloat16(0.0f);
  bool ok = true;
  // this CTA's share of the K chunks
  const int nchunks = (g.K + kTcKC - 1) / kTcKC;
  const int c0 = blockIdx.y * g.kchunks;
  const int c1 = min(nchunks, c0 + g.kchunks);
  for (int c = c0; c < c1; ++c) {
    const int k0 = c * kTcKC;
    stage_tile<128>(sA, g.A, g.a_rs, g.a_cs, m0, g.M, k0, g.K, g.a_vec, g.a_rfast, zero);
    stage_tile<BN>(sB, g.B, g.b_rs, g.b_cs, 0, g.N, k0, g.K, g.b_vec, g.b_rfast, zero);
    tc::fence_proxy_async();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after_sync();
#pragma unroll
      for (int ks = 0; ks < kTcKC / 16; ++ks) {
        const uint64_t ad = tc::smem_desc(tc::smem_u32(sA) + ks * 256, 128, kTcKC * 16);
        const uint64_t bd = tc::smem_desc(tc::smem_u32(sB) + ks * 256, 128, kTcKC * 16);
        tc::mma_bf16(taddr, ad, bd, idesc, (c > c0 || ks > 0) ? 1u : 0u);
      }
      tc::mma_commit(&mbar);
    }
    // the chunk buffers are reused once the MMAs that read them are done
    const bool done = tc::mbar_wait(&mbar, (uint32_t)((c - c0) & 1), kTcWaitCycles);
    ok = __syncthreads_and(done && ok) != 0;
    if (!ok) break;
  }
  tc::fence_after_sync();
  const uint32_t trow = taddr + ((uint32_t)(warp * 32) << 16);
  const bool split = g.ksplit > 1;
  if (ok && (split || !g.Df || g.df_cs == 1)) {
    // row-major outputs: each thread's row goes through shared memory (the
    // staging buffers are free), 32 columns at a time, and whole warps write
    // 32 consecutive columns of a row
    float* sO = reinterpret_cast<float*>(smem);  // 128 rows x 33 (odd stride: conflict-free)
    float* wsp = split ? g.ws + (size_t)blockIdx.y * g.M * g.N : nullptr;
#pragma unroll 1
    for (int n0 = 0; n0 < BN; n0 += 32) {
      const int nc = BN - n0 < 32 ? BN - n0 : 32;
      float v[16];
      tc::tmem_ld16(trow + (uint32_t)n0, v);
#pragma unroll
      for (int j = 0; j < 16; ++j) sO[tid * 33 + j] = v[j];
      if (nc > 16) {
        tc::tmem_ld16(trow + (uint32_t)(n0 + 16), v);
#pragma unroll
        for (int j = 0; j < 16; ++j) sO[tid * 33 + 16 + j] = v[j];
      }
      __syncthreads();
      const int n = n0 + lane;
#pragma unroll 4
      for (int rr = warp; rr < 128; rr += 4) {
        const int m = m0 + rr;
        if (lane < nc && m < g.M && n < g.N) {
          const float x = sO[rr * 33 + lane];
          if (split) {
            wsp[(size_t)m * g.N + n] = x;
          } else {
            const float y = dense_act(g, x, n);
            if (g.Df) g.Df[m * g.df_rs + n] = y;
            if (g.Dh) g.Dh[m * g.dh_rs + n] = __float2bfloat16(y);
          }
        }
      }
      __syncthreads();
    }
  } else if (ok) {
    // strided FP32 output (structure of arrays): thread m writes its row,
    // consecutive threads at consecutive addresses of each column
    const int m = m0 + warp * 32 + lane;
#pragma unroll 1
    for (int n0 = 0; n0 < BN; n0 += 16) {
      float v[16];
      tc::tmem_ld16(trow + (uint32_t)n0, v);
      if (m < g.M) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int n = n0 + j;
          if (n < g.N) {
            const float y = dense_act(g, v[j], n);
            g.Df[m * g.df_rs + n * g.df_cs] = y;
            if (g.Dh) g.Dh[m * g.dh_rs + n] = __float2bfloat16(y);
          }
        }
      }
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(taddr, NCOLS);
  if (!ok && tid == 0) atomicExch(g.err, 1);
}

// the split-K partial products added in split order, then bias, activation
// and the outputs
__global__ void k_splitk_reduce(DenseArgs g) {
  const long long mn = (long long)g.M * g.N;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= mn) return;
  const int m = (int)(i / g.N), n = (int)(i % g.N);
  float s = 0.0f;
  for (int k = 0; k < g.ksplit; ++k) s += g.ws[k * mn + i];
  const float y = dense_act(g, s, n);
  if (g.Df) g.Df[m * g.df_rs + n * g.df_cs] = y;
  if (g.Dh) g.Dh[m * g.dh_rs + n] = __float2bfloat16(y);
}

template <int BN>
static int launch_dense_bn(const DenseArgs& g, cudaStream_t st) {
  constexpr uint32_t NCOLS = BN <= 32 ? 32 : BN <= 64 ? 64 : BN <= 128 ? 128 : 256;
  // staging buffers, and at least enough shared memory that the CTAs
  // resident on one SM never ask for more than its 512 TMEM columns
  const size_t staging = (size_t)(128 + BN) * kTcKC * 2;
  const size_t tmem_cap = 233472 / (512 / NCOLS + 1) + 1024;
  const size_t smem = staging > tmem_cap ? staging : tmem_cap;
  static unsigned configured = 0;
  BPF_TRY(set_dyn_smem_once(k_dense_tc<BN>, (int)smem, configured));
  const dim3 grid((unsigned)((g.M + 127) / 128), (unsigned)g.ksplit);
  k_dense_tc<BN><<<grid, 128, smem, st>>>(g);
  BPF_TRY(cudaGetLastError());
  if (g.ksplit > 1) {
    const long long mn = (long long)g.M * g.N;
    k_splitk_reduce<<<(unsigned)((mn + 255) / 256), 256, 0, st>>>(g);
    BPF_TRY(cudaGetLastError());
  }
  return BPF_OK;
}

static int k_contiguous(const __nv_bfloat16* p, long long rs, long long cs) {
  return cs == 1 && rs % 8 == 0 && (reinterpret_cast<uintptr_t>(p) & 15) == 0;
}

int launch_dense(const DenseArgs& g0, cudaStream_t st) {
  DenseArgs g = g0;
  if (g.M <= 0 || g.N <= 0 || g.K <= 0 || !g.A || !g.B || !g.err || (!g.Df && !g.Dh)) return BPF_E_INVALID;
  g.a_vec = k_contiguous(g.A, g.a_rs, g.a_cs);
  g.b_vec = k_contiguous(g.B, g.b_rs, g.b_cs);
  g.a_rfast = !g.a_vec && g.a_rs == 1;
  g.b_rfast = !g.b_vec && g.b_rs == 1;
  // split K over CTAs when the 128-row tiles alone leave most SMs idle and
  // every split still gets two or more chunks
  const int mtiles = (g.M + 127) / 128;
  const int nchunks = (g.K + kTcKC - 1) / kTcKC;
  g.ksplit = 1;
  g.kchunks = nchunks;
  if (g.ws && mtiles < 64 && nchunks >= 4) {
    int target = nchunks / 2 < 148 / mtiles ? nchunks / 2 : 148 / mtiles;
    const long long cap = g.ws_floats / ((long long)g.M * g.N);
    if (target > cap) target = (int)cap;
    if (target > 1) {
      g.kchunks = (nchunks + target - 1) / target;
      g.ksplit = (nchunks + g.kchunks - 1) / g.kchunks;
    }
  }
  const int bn = (g.N + 15) / 16 * 16;
  switch (bn) {
    case 16: return launch_dense_bn<16>(g, st);
    case 32: return launch_dense_bn<32>(g, st);
    case 48: return launch_dense_bn<48>(g, st);
    case 64: return launch_dense_bn<64>(g, st);
    case 80: return launch_dense_bn<80>(g, st);
    case 96: return launch_dense_bn<96>(g, st);
    case 128: return launch_dense_bn<128>(g, st);
    case 160: return launch_dense_bn<160>(g, st);
    case 192: return launch_dense_bn<192>(g, st);
    case 256: return launch_dense_bn<256>(g, st);
    default: return BPF_E_INVALID;
  }
}

}  // namespace bpf

extern "C" int bpf_dense_bf16(const void* A, long long a_rs, long long a_cs, const void* B, long long b_rs,
                              long long b_cs, int M, int N, int K, const float* bias, int relu, float* Df,
                              long long df_rs, void* Dh, long long dh_rs, int* err, void* stream) {
  bpf::DenseArgs g;
  g.A = (const __nv_bfloat16*)A; g.a_rs = a_rs; g.a_cs = a_cs;
  g.B = (const __nv_bfloat16*)B; g.b_rs = b_rs; g.b_cs = b_cs;
  g.M = M; g.N = N; g.K = K;
  g.bias = bias; g.relu = relu;
  g.Df = Df; g.df_rs = df_rs; g.df_cs = 1;
  g.Dh = (__nv_bfloat16*)Dh; g.dh_rs = dh_rs;
  g.err = err;
  return bpf::launch_dense(g, (cudaStream_t)stream);
}
