// Declarations of the tensor-core dense layer (mlp.cu).
#pragma once
#include "internal.cuh"

#include <cuda_bf16.h>

namespace bpf {

struct DenseArgs {
  const __nv_bfloat16* A;
  long long a_rs, a_cs;  // A(m, k) = A[m*a_rs + k*a_cs]
  const __nv_bfloat16* B;
  long long b_rs, b_cs;  // B(n, k) = B[n*b_rs + k*b_cs]
  int M, N, K;
  const float* bias;     // N values, or null
  int relu;
  float* Df;             // D(m, n) = Df[m*df_rs + n*df_cs], or null
  long long df_rs;
  long long df_cs = 1;
  __nv_bfloat16* Dh;     // BF16 copy, or null
  long long dh_rs;
  int* err;              // set when a bounded wait gives up
  // split-K workspace (FP32), or null: a layer with few 128-row tiles and a
  // long K is split over CTAs whose partial products land here and are
  // added in a fixed order by a second kernel
  float* ws = nullptr;
  long long ws_floats = 0;
  // set by launch_dense: the operand is K-contiguous with 16-byte aligned
  // rows, so a chunk is staged with one 16-byte load per 8 elements
  // (*_vec), or row-contiguous, so consecutive threads take consecutive
  // rows (*_rfast); the K split and chunks per split
  int a_vec = 0, b_vec = 0, a_rfast = 0, b_rfast = 0;
  int ksplit = 1, kchunks = 0;
};

int launch_dense(const DenseArgs& g, cudaStream_t st);

}  // namespace bpf
