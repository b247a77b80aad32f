// The learned proposal's network and buffers (proposal.cu), shared with the
// guided filter step (guided.cu).
#pragma once
#include "internal.cuh"

#include <cuda_bf16.h>

namespace bpf {

constexpr int kProposalHidden = 128;
// clamp of the proposal's log-scale s
constexpr float kSMin = -7.0f, kSMax = 3.0f;
// the PZ network's shared-memory images (guided_pz.cu): W1' = [W1 | b1 | 0]
// (128 x 16), W2' = [W2 | b2 | 0] (128 x 144), W3' = [W3 | 0] (16 x 144);
// each bias as three BF16 pieces hi + mid + lo (24 significant bits, the
// FP32 value) in columns din .. din + 2, multiplied by constant-1 columns of
// the activations
constexpr int kPZNetK1 = 16, kPZNetK2 = kProposalHidden + 16, kPZNetN3 = 16;

struct ProposalNet {
  // dim: the proposed variables (the L96 state's 40 components; the PZ
  // model's one log-noise), din: network inputs, dout = 2 dim: (delta, s)
  int dim = 0, din = 0, dout = 0, hidden = 0;
  int k1 = 0;  // columns of W1's shared-memory image: din rounded up to a multiple of 16 (one MMA K step)
  // PZ network (din 3, dout 2): the images hold the biases of layers 1 and 2
  // as extra K columns (kPZNetK1, kPZNetK2) and W3 padded to 16 rows
  bool pz = false;
  // parameter vector: W1 [hidden x din], b1, W2 [hidden x hidden], b2,
  // W3 [dout x hidden], b3 (offsets in floats)
  int o_w1 = 0, o_b1 = 0, o_w2 = 0, o_b2 = 0, o_w3 = 0, o_b3 = 0, nparams = 0;
  float* params = nullptr;            // FP32 master copy
  __nv_bfloat16* params_h = nullptr;  // BF16 copy the dense layers read
  float *grads = nullptr, *m1 = nullptr, *m2 = nullptr;
  float *shift = nullptr, *scale = nullptr;  // input standardisation
  int* err = nullptr;
  double* loss = nullptr;
  // minibatch buffers (cap rows)
  int cap = 0;
  __nv_bfloat16 *U = nullptr, *H1 = nullptr, *H2 = nullptr, *dO = nullptr, *dZ = nullptr;
  float *O = nullptr, *dH = nullptr, *r0 = nullptr;
  float* mt = nullptr;  // RK4 means of the training inputs (L96)
  // precomputed training rows (PZ): inputs [rows x din] and targets
  // [rows x dim] in FP32
  float* feat = nullptr;
  float* target = nullptr;
  int rows = 0;
  // the BF16 weight matrices as shared-memory images in the canonical
  // K-major layout (tc.cuh): W1 at byte pk_w1, W2 at pk_w2, W3 at pk_w3;
  // rebuilt by pack_weights whenever params_h changes outside training and
  // at the end of every training call
  unsigned char* packed = nullptr;
  int pk_w1 = 0, pk_w2 = 0, pk_w3 = 0, pk_bytes = 0;
  float* colpart = nullptr;  // per-chunk column sums of the bias gradients
  float* ws = nullptr;       // split-K workspace of the weight-gradient layers
  long long ws_floats = 0;
  double* loss_part = nullptr;  // per-block loss sums

  const __nv_bfloat16* w1h() const { return params_h + o_w1; }
  const __nv_bfloat16* w2h() const { return params_h + o_w2; }
  const __nv_bfloat16* w3h() const { return params_h + o_w3; }
  const float* b1() const { return params + o_b1; }
  const float* b2() const { return params + o_b2; }
  const float* b3() const { return params + o_b3; }

  int alloc(int d, int hid, int cap_batch, int din_ = 0);  // din_ 0: 2 d
  void release();
};

// rebuild ProposalNet::packed from params_h
int pack_weights(ProposalNet& p, cudaStream_t st);

// O [B x dout] = MLP(U [B x din]); H1, H2 [B x hidden] hold the activations
int proposal_forward(ProposalNet& p, const __nv_bfloat16* U, int B, __nv_bfloat16* H1, __nv_bfloat16* H2, float* O,
                     cudaStream_t st);

// one guided filter step (guided.cu)
struct GuidedArgs {
  const void* x_in;  // state before the step (FP32 SoA, ld)
  void* x_out;
  int ld, n;
  const int* as;
  double* lw;
  const void* y;     // device observation (required)
  double t1, t2;
  uint64_t seed;
  int step;
  double theta[BPF_MAX_THETA];
  double h;
  StepStats* stats;
  LwPartial* partials;
  int max_partials;
  unsigned* counter;
};
int launch_guided(ProposalNet& net, const GuidedArgs& a, cudaStream_t st);

// the guided step of every filter of a batch (guided.cu, batch.cu)
struct BatchFilter;
struct L96Params;
struct BatchGuidedArgs {
  const float* x_in;
  float* x_out;
  int ld;
  int* as;
  double* lw;
  const float* y;  // nf x dim device observations
  double t1, t2;
  int step;
  const BatchFilter* filt;
  const L96Params* prms;
  const int* tile2f;  // 128-particle tile -> filter
  int tiles;
  StepStats* stats;
  LwPartial* partials;
  unsigned* counters;
  double* hist;
  int nf, k;
};
int launch_batch_guided(ProposalNet& net, const BatchGuidedArgs& a, cudaStream_t st);

// the guided step of every filter of a PZ batch (guided_pz.cu): the proposal
// over each particle's log-noise; the network of every particle in one
// launch, then the step
struct PZParams;
struct BatchPZGuidedArgs {
  const double* x_in;
  double* x_out;
  int ld;
  int* as;
  double* lw;
  const double* y;  // nf device observations
  double t1, t2;
  int step;
  const BatchFilter* filt;
  const PZParams* prms;
  const int* blk2f;  // transition block -> filter
  int blocks;
  StepStats* stats;
  LwPartial* partials;
  unsigned* counters;
  double* hist;
  int nf, k;
  float2* O;  // the network's (delta, raw s) per column, ld entries
};
int launch_batch_pz_guided(ProposalNet& net, const BatchPZGuidedArgs& a, cudaStream_t st);

}  // namespace bpf

struct bpf_proposal;
namespace bpf {
ProposalNet* proposal_net(bpf_proposal* q);
double proposal_dt(bpf_proposal* q);
}  // namespace bpf
