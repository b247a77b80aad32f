// Pieces shared by the fused guided steps (guided.cu, guided_pz.cu): a CTA
// stages 128-row BF16 activation tiles in shared memory (canonical K-major
// layout, tc.cuh), one thread issues each layer's tcgen05 MMA chain into
// tensor memory, and every thread moves its own accumulator row (TMEM lane
// = particle) back into the tile as the next layer's A operand.
#pragma once
#include "internal.cuh"
#include "tc.cuh"
#include "proposal.cuh"

namespace bpf {
namespace {

constexpr int kGTile = 128;                     // particles per tile
constexpr int kGTileBytes = 128 * 128 * 2;      // one BF16 activation tile
constexpr long long kGWaitCycles = 2000000000ll;  // ~1 s at 2 GHz

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

// one thread issues, for every tile, the MMA chain D_j = A_j * W^T over K
// (a multiple of 16) and commits them all to the mbarrier
template <int TILES, int K, int N>
__device__ __forceinline__ void issue_layer(uint32_t taddr, const unsigned char* sA, const unsigned char* sW,
                                            uint64_t* mbar) {
  constexpr uint32_t idesc = tc::idesc_bf16(128, N);
  tc::fence_after_sync();
#pragma unroll
  for (int j = 0; j < TILES; ++j) {
#pragma unroll
    for (int ks = 0; ks < K / 16; ++ks) {
      const uint64_t ad = tc::smem_desc(tc::smem_u32(sA + j * kGTileBytes) + ks * 256, 128, K * 16);
      const uint64_t bd = tc::smem_desc(tc::smem_u32(sW) + ks * 256, 128, K * 16);
      tc::mma_bf16(taddr + (uint32_t)(128 * j), ad, bd, idesc, ks > 0 ? 1u : 0u);
    }
  }
  tc::mma_commit(mbar);
}

// hidden-layer epilogue: this thread's accumulator row + bias, ReLU, BF16,
// into row r of its tile (K = 128)
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

// thread 0 waits for the weight copy, then everyone agrees that the layer
// can be issued (the A operands written by all threads are visible to the
// tensor core once this returns true)
__device__ __forceinline__ bool weights_ready(uint64_t* wbar, uint32_t parity, bool ok) {
  tc::fence_before_sync();
  tc::fence_proxy_async();
  bool mine = ok;
  if (threadIdx.x == 0 && ok) mine = tc::mbar_wait(wbar, parity, kGWaitCycles);
  return __syncthreads_and(mine) != 0;
}

// wait for the MMA chain's commit; all threads agree on the outcome
__device__ __forceinline__ bool layer_done(uint64_t* mbar, uint32_t parity, bool ok) {
  const bool done = ok && tc::mbar_wait(mbar, parity, kGWaitCycles);
  ok = __syncthreads_and(done) != 0;
  tc::fence_after_sync();
  return ok;
}

}  // namespace
}  // namespace bpf
