/*
 * libbi_b200 — a model compiled into the caller's own code (CUDA C++,
 * header-only, sm_100a).
 *
 * LibBi compiles a .bi model into a Model class whose pieces are C++ classes
 * (share/tt/cpp/model.hpp.tt, var.hpp.tt, var_coord.hpp.tt,
 * action_coord.hpp.tt): one VarN per variable (ID, START, SIZE, TYPE,
 * coord_type), one ActionN per action with static functions that the block
 * updaters call per particle and element,
 *   samples(rng, s, p, ix, cox, pax, x)        action/gaussian.hpp.tt (sample)
 *   logDensities(s, p, ix, cox, pax, x, lp)    action/gaussian.hpp.tt (logdensity)
 *   simulates(s, p, ix, cox, pax, x)           action/eval_.hpp.tt
 *   dfdt(t, s, p, cox, pax, dfdt)              action/ode_.hpp.tt
 * and type trees of actions per block (macro/create_action_typetree.hpp.tt).
 * The generated blocks call StaticSampler<B,S>::samples, RK4Integrator<B,S>
 * ::update / RK43Integrator<B,S>::update (block/ode.hpp.tt:39-54),
 * StaticUpdater<B,S>::update and SparseStaticLogDensity<B,S>::logDensities
 * (block/pdf_.hpp.tt:46-75), each a pass over the whole State.
 *
 * This header takes a model class of that shape, compiled with nvcc in the
 * caller's own translation unit, and runs its action functions inside ONE
 * fused kernel per filter step: ancestor gather, the transition's blocks in
 * order (noise draws, ODE, deterministic updates), the observation
 * log-density, and the block partial of the log-weight reduction, with the
 * state in registers (noise variables in shared memory).  bpf::model_ops<B>
 * packages the kernels as a bpf_model_ops table for bpf_create_model, so the
 * library's filter, resamplers and checkpoints drive the model with no
 * library change.  The bi:: updaters at the end of this header run the same
 * action functions one block per kernel on a device State<B, ON_DEVICE>,
 * with the same arithmetic and draws, for code that calls the block updaters
 * one by one as the generated blocks do.
 *
 * What the model class provides, beyond the generated classes:
 *   typedefs transition_type, observation_type and initial_type, each a
 *   bpf::blocks<...> of the block markers bpf::pdf_block<S> (noise or
 *   observation actions), bpf::eval_block<S> (deterministic actions) and
 *   bpf::ode_block<S, C> (C: alg = bpf::ODE_RK4 or bpf::ODE_RK43 and the
 *   ode block's h, atoler, rtoler, as block/ode.hpp.tt reads them), where S
 *   is the block's action type tree built with the generator's macros
 *   (BEGIN_TYPETREE, LEAF_NODE, BEGIN_NODE, JOIN_NODE, END_NODE,
 *   END_TYPETREE, GET_TYPETREE, all defined here).
 * Supported variable types: D_VAR (state, stored SoA in the filter's
 * buffers), DX_VAR (auxiliary state, stored after the D_VAR columns),
 * R_VAR (noise, redrawn every step), P_VAR (parameters, fixed for a filter:
 * bpf_create_model's params) and O_VAR (observations).  F_VAR inputs are
 * not supported.  Distributions: rng.gaussian(mu, sigma) and
 * rng.uniform(lo, hi).
 *
 * Arithmetic.  Compile the model's translation unit with -fmad=false for
 * results that follow the model source's expression order (so that a host
 * restatement of the same expressions, built without contraction,
 * reproduces every bit); with -fmad=true nvcc contracts products into
 * fused multiply-adds where it sees fit.  The integrators' own arithmetic
 * (stages, step control) uses explicit fused multiply-adds in the form of
 * the reference's host integrators compiled with contraction; bi::log,
 * bi::exp and bi::pow are the portable functions of bpf_math.h.
 *
 * Random draws: every normal of particle p in step k is a function of (seed,
 * p, k, draw index), Philox4x32-10 words through Box-Muller as the built-in
 * models draw them (bpf_philox.h, bpf_math.h): the i-th gaussian() of a step
 * uses block i/4, word pair (i%4)/2, member i%2.  The initial block draws
 * with step 0 and the tag BPF_RNG_INIT.  uniform() draws come from their own
 * counter in blocks (1 << 20) + j/4.
 */
#ifndef BPF_MODEL_CUH
#define BPF_MODEL_CUH

#include <cuda_runtime.h>
#include <stdint.h>
#include <type_traits>
#include <stdexcept>
#include <vector>

#include "libbi_b200.h"
#include "bpf_philox.h"
#include "bpf_math.h"
#include "bpf_device.cuh"

/* ---- the vocabulary the generated code uses ------------------------------ */

/* The model precision.  LibBi sets `real` for the whole build
 * (share/src/bi/math/scalar.hpp); here the model's translation unit does,
 * with -DBPF_REAL=float or the default double. */
#ifndef BPF_REAL
#define BPF_REAL double
#endif
typedef BPF_REAL real;

#ifndef CUDA_FUNC_BOTH
#define CUDA_FUNC_BOTH __host__ __device__ __forceinline__
#endif
#ifndef BI_UNUSED
#define BI_UNUSED __attribute__((unused))
#endif
#ifndef BI_REAL
#define BI_REAL(x) ((real)(x))
#endif
#ifndef BOOST_AUTO
#define BOOST_AUTO(var, expr) auto var = (expr)
#endif
#ifndef BI_INF
#define BI_INF (BI_REAL(1.0) / BI_REAL(0.0))
#endif
#ifndef BI_PI
#define BI_PI 3.1415926535897932384626433832795
#endif
#ifndef BI_HALF_LOG_TWO_PI
#define BI_HALF_LOG_TWO_PI 0.91893853320467274178032973640562
#endif
#ifndef BI_LOG_TWO_PI
#define BI_LOG_TWO_PI 1.83787706640934548356065947281123
#endif

namespace bi {

/* variable types and locations (share/src/bi/traits/var_traits.hpp,
 * share/src/bi/misc/location.hpp) */
enum VarType { R_VAR, D_VAR, P_VAR, F_VAR, O_VAR, DX_VAR, PX_VAR, B_VAR, RY_VAR, DY_VAR, PY_VAR, OY_VAR };
enum Location { ON_HOST, ON_DEVICE };

/* Action type trees: LEAF_NODE(reps, Action) repeats one action, a node
 * joins two subtrees; visited depth first, left to right. */
struct empty_typelist {};
template <int REPS, class A> struct tree_leaf {};
template <int REPS, class L, class R> struct tree_node {};

/* The device State of a model (State<B, ON_DEVICE>): a view of
 * structure-of-arrays buffers in device memory.  x: D_VAR then DX_VAR
 * columns, element j of particle p at x[j * ld + p]; r: R_VAR columns
 * likewise; prm: the P_VAR values (shared by all particles); y: the O_VAR
 * values of the current observation.  step addresses the random draws (the
 * seed comes with the sampler's Random); stream: where the updaters below
 * enqueue their kernels.  Inside the fused kernel the action functions receive a State
 * whose fields they do not use: every variable is fetched through pax and
 * x. */
template <class B, Location L> class State;
template <class B> class State<B, ON_DEVICE> {
 public:
  real* x = nullptr;
  real* r = nullptr;
  const real* prm = nullptr;
  const real* y = nullptr;
  int ld = 0;
  int n = 0;
  int step = 0;
  cudaStream_t stream = 0;
  CUDA_FUNC_BOTH int size() const { return n; }
};

/* elementary functions of the model code, on host and device */
CUDA_FUNC_BOTH float log(float x) { return bpf_logf(x); }
CUDA_FUNC_BOTH double log(double x) { return bpf_log(x); }
CUDA_FUNC_BOTH float exp(float x) { return bpf_expf(x); }
CUDA_FUNC_BOTH double exp(double x) { return bpf_exp(x); }
CUDA_FUNC_BOTH float sqrt(float x) { return ::sqrtf(x); }
CUDA_FUNC_BOTH double sqrt(double x) { return ::sqrt(x); }
CUDA_FUNC_BOTH float abs(float x) { return ::fabsf(x); }
CUDA_FUNC_BOTH double abs(double x) { return ::fabs(x); }
CUDA_FUNC_BOTH float max(float a, float b) { return ::fmaxf(a, b); }
CUDA_FUNC_BOTH double max(double a, double b) { return ::fmax(a, b); }
CUDA_FUNC_BOTH float min(float a, float b) { return ::fminf(a, b); }
CUDA_FUNC_BOTH double min(double a, double b) { return ::fmin(a, b); }
/* x^y: exact for y = 1 and 2, else exp(y log x) of bpf_math.h */
CUDA_FUNC_BOTH float pow(float x, float y) {
  if (y == 2.0f) return BPF_MATH_MULF(x, x);
  if (y == 1.0f) return x;
  return bpf_expf(BPF_MATH_MULF(y, bpf_logf(x)));
}
CUDA_FUNC_BOTH double pow(double x, double y) {
  if (y == 2.0) return BPF_MATH_MUL(x, x);
  if (y == 1.0) return x;
  return bpf_exp(BPF_MATH_MUL(y, bpf_log(x)));
}

}  // namespace bi

/* the generator's type tree macros (share/tt/cpp/macro/create_action_typetree.hpp.tt) */
#ifndef BEGIN_TYPETREE
#define BEGIN_TYPETREE(name) struct name { typedef
#define LEAF_NODE(reps, ...) bi::tree_leaf<reps, __VA_ARGS__>
#define BEGIN_NODE(reps) bi::tree_node<reps,
#define JOIN_NODE ,
#define END_NODE >
#define NULL_NODE bi::empty_typelist
#define END_TYPETREE() type; };
#define GET_TYPETREE(name) name::type
#endif

namespace bpf {

/* ---- block markers ------------------------------------------------------- */
enum { ODE_RK4 = 0, ODE_RK43 = 1 };
template <class S> struct pdf_block { typedef S action_typelist; };
template <class S> struct eval_block { typedef S action_typelist; };
template <class S, class C> struct ode_block { typedef S action_typelist; typedef C consts; };
template <class... Blocks> struct blocks {};

/* ---- visiting a type tree --------------------------------------------------- */
template <class S> struct tree;
template <> struct tree<bi::empty_typelist> {
  static constexpr int size = 0;
  template <class F> __device__ __forceinline__ static void each(F&) {}
};
template <int REPS, class A> struct tree<bi::tree_leaf<REPS, A>> {
  static constexpr int size = REPS * A::SIZE;
  template <class F> __device__ __forceinline__ static void each(F& f) {
#pragma unroll
    for (int r = 0; r < REPS; ++r) f.template visit<A>();
  }
};
template <int REPS, class L, class R> struct tree<bi::tree_node<REPS, L, R>> {
  static constexpr int size = REPS * (tree<L>::size + tree<R>::size);
  template <class F> __device__ __forceinline__ static void each(F& f) {
#pragma unroll
    for (int r = 0; r < REPS; ++r) {
      tree<L>::each(f);
      tree<R>::each(f);
    }
  }
};

/* ---- one particle's variables ------------------------------------------------ */
template <class B, class T>
struct ParticleVars {
  static constexpr int kND = B::ND > 0 ? B::ND : 1;
  static constexpr int kNDX = B::NDX > 0 ? B::NDX : 1;
  static constexpr int kNP = B::NP > 0 ? B::NP : 1;
  static constexpr int kNO = B::NO > 0 ? B::NO : 1;
  T d[kND];
  T dx[kNDX];
  T p[kNP];
  T o[kNO];
  T* r;        // R_VAR: element j at r[j * rstride]
  int rstride;
};

/* pax and x of the generated actions: every fetch resolves to a register
 * (or, for noise, this thread's shared-memory column) at compile time once
 * the loops over elements are unrolled. */
template <class B, class T>
struct VarAccess {
  ParticleVars<B, T>& v;
  template <class V, class S>
  __device__ __forceinline__ T& fetch(S&, const int, const int ix) const {
    if constexpr (V::TYPE == bi::D_VAR) return v.d[V::START + ix];
    else if constexpr (V::TYPE == bi::DX_VAR) return v.dx[V::START + ix];
    else if constexpr (V::TYPE == bi::R_VAR) return v.r[(V::START + ix) * v.rstride];
    else if constexpr (V::TYPE == bi::P_VAR) return v.p[V::START + ix];
    else {
      static_assert(V::TYPE == bi::O_VAR, "variable type not supported in a device model");
      return v.o[V::START + ix];
    }
  }
  /* the observed value of an O_VAR element (the OY_VAR buffer) */
  template <class V, class S>
  __device__ __forceinline__ T fetch_alt(S&, const int, const int ix) const {
    return v.o[V::START + ix];
  }
};

/* ---- the random draws of one particle in one step ---------------------------- */
template <class T>
struct ParticleRng {
  uint64_t seed;
  uint32_t p, step, tag;
  int ng = 0, nu = 0;  // gaussians and uniforms drawn so far
  int zblk = -1, ublk = -1;
  T z[4];
  bpf_u32x4 ur;
  __device__ __forceinline__ ParticleRng(uint64_t s, uint32_t pp, uint32_t k, uint32_t t, int ng0 = 0)
      : seed(s), p(pp), step(k), tag(t), ng(ng0) {}
  __device__ __forceinline__ T normal() {
    const int b = ng >> 2;
    if (b != zblk) {
      bpf_u32x4 r = bpf_draw(seed, p, step, (uint32_t)b, tag);
      normal_pair(r.v[0], r.v[1], z[0], z[1]);
      normal_pair(r.v[2], r.v[3], z[2], z[3]);
      zblk = b;
    }
    return z[ng++ & 3];
  }
  /* rng.gaussian(mu, sigma) = mu + sigma z, the product rounded on its own */
  __device__ __forceinline__ T gaussian(const T mu = (T)0, const T sigma = (T)1) {
    const T zz = normal();
    if constexpr (sizeof(T) == 4) return __fadd_rn(mu, __fmul_rn(sigma, zz));
    else return __dadd_rn(mu, __dmul_rn(sigma, zz));
  }
  /* rng.uniform(lo, hi) = lo + (hi - lo) u, u in (0, 1) */
  __device__ __forceinline__ T uniform(const T lo = (T)0, const T hi = (T)1) {
    const int b = (1 << 20) + (nu >> 2);
    if (b != ublk) {
      ur = bpf_draw(seed, p, step, (uint32_t)b, tag);
      ublk = b;
    }
    const uint32_t w = ur.v[nu++ & 3];
    if constexpr (sizeof(T) == 4) return __fadd_rn(lo, __fmul_rn(__fsub_rn(hi, lo), bpf_u01f(w)));
    else return __dadd_rn(lo, __dmul_rn(__dsub_rn(hi, lo), (double)bpf_u01f(w)));
  }
  __device__ __forceinline__ static void normal_pair(uint32_t a, uint32_t b, float& z0, float& z1) {
    bpf_normal_pair_f(a, b, &z0, &z1);
  }
  __device__ __forceinline__ static void normal_pair(uint32_t a, uint32_t b, double& z0, double& z1) {
    bpf_normal_pair_d(a, b, &z0, &z1);
  }
};

template <class T> struct Arith;
template <> struct Arith<float> {
  __device__ static float fma_(float a, float b, float c) { return __fmaf_rn(a, b, c); }
  __device__ static float mul_(float a, float b) { return __fmul_rn(a, b); }
};
template <> struct Arith<double> {
  __device__ static double fma_(double a, double b, double c) { return __fma_rn(a, b, c); }
  __device__ static double mul_(double a, double b) { return __dmul_rn(a, b); }
};

/* ---- the block visitors ------------------------------------------------------- */
/* noise (StaticSamplerHost's order: action by action, element by element) */
template <class B, class T>
struct SampleVisit {
  bi::State<B, bi::ON_DEVICE>& s;
  VarAccess<B, T>& acc;
  ParticleRng<T>& rng;
  int p;
  template <class A> __device__ __forceinline__ void visit() {
    typename A::coord_type cox;
#pragma unroll
    for (int ix = 0; ix < A::SIZE; ++ix) {
      A::samples(rng, s, p, ix, cox, acc, acc);
      ++cox;
    }
  }
};

/* deterministic updates (StaticUpdater) */
template <class B, class T>
struct SimulateVisit {
  bi::State<B, bi::ON_DEVICE>& s;
  VarAccess<B, T>& acc;
  int p;
  template <class A> __device__ __forceinline__ void visit() {
    typename A::coord_type cox;
#pragma unroll
    for (int ix = 0; ix < A::SIZE; ++ix) {
      A::simulates(s, p, ix, cox, acc, acc);
      ++cox;
    }
  }
};

/* observation log-density (SparseStaticLogDensity): lp accumulates in FP64
 * onto the particle's log-weight, term by term in element order; bit j of
 * mask (j the element's index over the O_VAR block) says whether it is
 * observed */
template <class B, class T>
struct LogDensityVisit {
  bi::State<B, bi::ON_DEVICE>& s;
  VarAccess<B, T>& acc;
  int p;
  uint64_t mask;
  double& lp;
  template <class A> __device__ __forceinline__ void visit() {
    typename A::coord_type cox;
#pragma unroll
    for (int ix = 0; ix < A::SIZE; ++ix) {
      const int j = A::target_type::START + cox.index();
      if (j >= 64 || ((mask >> j) & 1ull)) {
        T term = (T)0;
        A::logDensities(s, p, ix, cox, acc, acc, term);
        lp += (double)term;
      }
      ++cox;
    }
  }
};

/* ODE: element j of the integrated vector is the j-th (action, element) of
 * the block's type tree; slot(j) its index in the D_VAR (or DX_VAR)
 * registers */
template <class B, class T, int N>
struct OdeMap {
  int slot[N];
  bool dx[N];
  int j = 0;
  template <class A> __device__ __forceinline__ void visit() {
    typename A::coord_type cox;
#pragma unroll
    for (int ix = 0; ix < A::SIZE; ++ix) {
      slot[j] = A::target_type::START + cox.index();
      dx[j] = A::target_type::TYPE == bi::DX_VAR;
      ++j;
      ++cox;
    }
  }
};

template <class B, class T, int N>
struct DfdtVisit {
  bi::State<B, bi::ON_DEVICE>& s;
  VarAccess<B, T>& acc;
  int p;
  T t;
  T (&k)[N];
  int j = 0;
  template <class A> __device__ __forceinline__ void visit() {
    typename A::coord_type cox;
#pragma unroll
    for (int ix = 0; ix < A::SIZE; ++ix) {
      A::dfdt(t, s, p, cox, acc, k[j]);
      ++j;
      ++cox;
    }
  }
};

template <class B, class T, int N>
__device__ __forceinline__ T& ode_slot(ParticleVars<B, T>& v, const OdeMap<B, T, N>& m, int j) {
  return m.dx[j] ? v.dx[m.slot[j]] : v.d[m.slot[j]];
}

/* RK4IntegratorHost::update (share/src/bi/host/ode/RK4IntegratorHost.hpp:43-100)
 * with the stages of RK4Stage (share/src/bi/ode/RK4Stage.hpp:26-77): stage
 * times t, t + h/2, t + h/2, t + h; b = 1/6, 1/3, 1/3, 1/6; the last step
 * clipped to t2. */
template <class B, class T, class S>
__device__ __forceinline__ void ode_rk4(ParticleVars<B, T>& v, VarAccess<B, T>& acc, bi::State<B, bi::ON_DEVICE>& s,
                                        int p, double t1d, double t2d, double h0) {
  constexpr int N = tree<S>::size;
  OdeMap<B, T, N> m;
  tree<S>::each(m);
  typedef Arith<T> F;
  const T b1 = (T)(1.0 / 6.0), b2 = (T)(1.0 / 3.0), b3 = (T)(1.0 / 3.0), b4 = (T)(1.0 / 6.0);
  const T t2 = (T)t2d;
  T t = (T)t1d, h = (T)h0;
  T x0[N];
#pragma unroll
  for (int j = 0; j < N; ++j) x0[j] = ode_slot(v, m, j);
  while (t < t2) {
    if (F::fma_((T)1.01, h, t) - t2 > (T)0) {
      h = t2 - t;
      if (h <= (T)0) { t = t2; break; }
    }
    const T hh = (T)0.5 * h;
    T k[N], a[N];
    { DfdtVisit<B, T, N> f{s, acc, p, t, k}; tree<S>::each(f); }
#pragma unroll
    for (int j = 0; j < N; ++j) { a[j] = b1 * k[j]; ode_slot(v, m, j) = F::fma_(hh, k[j], x0[j]); }
    { DfdtVisit<B, T, N> f{s, acc, p, F::fma_((T)0.5, h, t), k}; tree<S>::each(f); }
#pragma unroll
    for (int j = 0; j < N; ++j) { a[j] = F::fma_(b2, k[j], a[j]); ode_slot(v, m, j) = F::fma_(hh, k[j], x0[j]); }
    { DfdtVisit<B, T, N> f{s, acc, p, F::fma_((T)0.5, h, t), k}; tree<S>::each(f); }
#pragma unroll
    for (int j = 0; j < N; ++j) { a[j] = F::fma_(b3, k[j], a[j]); ode_slot(v, m, j) = F::fma_(h, k[j], x0[j]); }
    { DfdtVisit<B, T, N> f{s, acc, p, t + h, k}; tree<S>::each(f); }
#pragma unroll
    for (int j = 0; j < N; ++j) {
      a[j] = F::fma_(b4, k[j], a[j]);
      x0[j] = F::fma_(h, a[j], x0[j]);
      ode_slot(v, m, j) = x0[j];
    }
    t += h;
  }
}

/* RK43IntegratorHost::update (share/src/bi/host/ode/RK43IntegratorHost.hpp:
 * 48-144), the low-storage RK4(3)5[2R+]C stages of RK43Stage
 * (share/src/bi/ode/RK43Stage.hpp:26-81), error norm
 * e2 = mean((err h / (atoler + rtoler max(|old|, |new|)))^2) and the
 * step-size control with the constants of IntegratorConstants
 * (share/src/bi/host/ode/IntegratorConstants.cpp:45-87): safety 0.9,
 * facl 0.2, facr 10, beta 0.04, at most 1000 steps. */
template <class B, class T, class S>
__device__ __forceinline__ void ode_rk43(ParticleVars<B, T>& v, VarAccess<B, T>& acc, bi::State<B, bi::ON_DEVICE>& s,
                                         int p, double t1d, double t2d, double h0, double atoler, double rtoler) {
  constexpr int N = tree<S>::size;
  OdeMap<B, T, N> m;
  tree<S>::each(m);
  typedef Arith<T> F;
  const T a21 = (T)0.225022458725713, b1 = (T)0.0512293066403392, e1 = (T)-0.0859880154628801;
  const T a32 = (T)0.544043312951405, b2 = (T)0.380954825726402, c2 = (T)0.225022458725713,
          e2c = (T)0.189074063397015;
  const T a43 = (T)0.144568243493995, b3 = (T)-0.373352596392383, c3 = (T)0.595272619591744,
          e3 = (T)-0.144145875232852;
  const T a54 = (T)0.786664342198357, b4 = (T)0.592501285026362, c4 = (T)0.576752375860736,
          e4 = (T)-0.0317933915175331;
  const T b5 = (T)0.34866717899928, c5 = (T)0.845495878172715, e5 = (T)0.0728532188162504;
  const T atol = (T)atoler, rtol = (T)rtoler;
  const T facl = (T)0.2, facr = (T)10.0, beta = (T)0.04;
  // h_ode_set_safe / h_ode_set_beta (IntegratorConstants.cpp:45-60) in T
  T logsafe, expo, logfacold;
  if constexpr (sizeof(T) == 4) {
    logsafe = bpf_logf(0.9f);
    expo = __fmul_rn(0.5f, __fmaf_rn(-0.04f, 0.75f, 0.2f));
    logfacold = bpf_logf(1.0e-4f);
  } else {
    logsafe = bpf_log(0.9);
    expo = __dmul_rn(0.5, __fma_rn(-0.04, 0.75, 0.2));
    logfacold = bpf_log(1.0e-4);
  }
  const T t2 = (T)t2d;
  T t = (T)t1d, h = (T)h0;
  T old[N], r1[N];
#pragma unroll
  for (int j = 0; j < N; ++j) { old[j] = ode_slot(v, m, j); r1[j] = old[j]; }
  int nst = 0;
  while (t < t2 && nst < 1000) {
    if (F::fma_((T)1.01, h, t) - t2 > (T)0) {
      h = t2 - t;
      if (h <= (T)0) { t = t2; break; }
    }
    T r2[N], k[N], err[N];
    // stage 1 at t, from r1
#pragma unroll
    for (int j = 0; j < N; ++j) ode_slot(v, m, j) = r1[j];
    { DfdtVisit<B, T, N> f{s, acc, p, t, k}; tree<S>::each(f); }
#pragma unroll
    for (int j = 0; j < N; ++j) {
      err[j] = e1 * k[j];
      r1[j] = F::fma_(a21 * h, k[j], r1[j]);
      r2[j] = F::fma_((b1 - a21) * h, k[j], r1[j]);
      ode_slot(v, m, j) = r1[j];
    }
    // stage 2
    { DfdtVisit<B, T, N> f{s, acc, p, F::fma_(c2, h, t), k}; tree<S>::each(f); }
#pragma unroll
    for (int j = 0; j < N; ++j) {
      err[j] = F::fma_(e2c, k[j], err[j]);
      r2[j] = F::fma_(a32 * h, k[j], r2[j]);
      r1[j] = F::fma_((b2 - a32) * h, k[j], r2[j]);
      ode_slot(v, m, j) = r2[j];
    }
    // stage 3
    { DfdtVisit<B, T, N> f{s, acc, p, F::fma_(c3, h, t), k}; tree<S>::each(f); }
#pragma unroll
    for (int j = 0; j < N; ++j) {
      err[j] = F::fma_(e3, k[j], err[j]);
      r1[j] = F::fma_(a43 * h, k[j], r1[j]);
      r2[j] = F::fma_((b3 - a43) * h, k[j], r1[j]);
      ode_slot(v, m, j) = r1[j];
    }
    // stage 4
    { DfdtVisit<B, T, N> f{s, acc, p, F::fma_(c4, h, t), k}; tree<S>::each(f); }
#pragma unroll
    for (int j = 0; j < N; ++j) {
      err[j] = F::fma_(e4, k[j], err[j]);
      r2[j] = F::fma_(a54 * h, k[j], r2[j]);
      r1[j] = F::fma_((b4 - a54) * h, k[j], r2[j]);
      ode_slot(v, m, j) = r2[j];
    }
    // stage 5
    { DfdtVisit<B, T, N> f{s, acc, p, F::fma_(c5, h, t), k}; tree<S>::each(f); }
#pragma unroll
    for (int j = 0; j < N; ++j) {
      err[j] = F::fma_(e5, k[j], err[j]);
      r1[j] = F::fma_(b5 * h, k[j], r1[j]);
    }
    // error norm
    T e2 = (T)0;
#pragma unroll
    for (int j = 0; j < N; ++j) {
      const T e = (err[j] * h) / F::fma_(rtol, bi::max(bi::abs(old[j]), bi::abs(r1[j])), atol);
      e2 = F::fma_(e, e, e2);
    }
    e2 = e2 / (T)N;
    if (e2 <= (T)1) {
      t += h;
      if (t < t2) {
#pragma unroll
        for (int j = 0; j < N; ++j) old[j] = r1[j];
      }
    } else {
#pragma unroll
      for (int j = 0; j < N; ++j) r1[j] = old[j];
    }
    if (t < t2) {
      const T logfac11 = F::mul_(expo, bi::log(e2));
      if (e2 > (T)1) {
        h = F::mul_(h, bi::max(facl, bi::exp(logsafe - logfac11)));
      } else {
        T fac = bi::exp(F::fma_(beta, logfacold, logsafe) - logfac11);
        fac = bi::min(facr, bi::max(facl, fac));
        h = F::mul_(h, fac);
        logfacold = F::mul_((T)0.5, bi::log(bi::max(e2, (T)1.0e-8)));
      }
    }
    ++nst;
  }
#pragma unroll
  for (int j = 0; j < N; ++j) ode_slot(v, m, j) = r1[j];
}

/* one block of a transition / initial block list */
template <class Blk> struct run_block;
template <class S> struct run_block<pdf_block<S>> {
  template <class B, class T>
  __device__ __forceinline__ static void sample(ParticleVars<B, T>&, VarAccess<B, T>& acc,
                                                bi::State<B, bi::ON_DEVICE>& s, ParticleRng<T>& rng, int p, double,
                                                double) {
    SampleVisit<B, T> f{s, acc, rng, p};
    tree<S>::each(f);
  }
};
template <class S> struct run_block<eval_block<S>> {
  template <class B, class T>
  __device__ __forceinline__ static void sample(ParticleVars<B, T>&, VarAccess<B, T>& acc,
                                                bi::State<B, bi::ON_DEVICE>& s, ParticleRng<T>&, int p, double,
                                                double) {
    SimulateVisit<B, T> f{s, acc, p};
    tree<S>::each(f);
  }
};
template <class S, class C> struct run_block<ode_block<S, C>> {
  template <class B, class T>
  __device__ __forceinline__ static void sample(ParticleVars<B, T>& v, VarAccess<B, T>& acc,
                                                bi::State<B, bi::ON_DEVICE>& s, ParticleRng<T>&, int p, double t1,
                                                double t2) {
    if constexpr (C::alg == ODE_RK4) ode_rk4<B, T, S>(v, acc, s, p, t1, t2, C::h);
    else ode_rk43<B, T, S>(v, acc, s, p, t1, t2, C::h, C::atoler, C::rtoler);
  }
};

template <class L> struct run_blocks;
template <class... Bs> struct run_blocks<blocks<Bs...>> {
  template <class B, class T>
  __device__ __forceinline__ static void sample(ParticleVars<B, T>& v, VarAccess<B, T>& acc,
                                                bi::State<B, bi::ON_DEVICE>& s, ParticleRng<T>& rng, int p,
                                                double t1, double t2) {
    (run_block<Bs>::template sample<B, T>(v, acc, s, rng, p, t1, t2), ...);
  }
  template <class B, class T>
  __device__ __forceinline__ static void log_density(VarAccess<B, T>& acc, bi::State<B, bi::ON_DEVICE>& s, int p,
                                                     uint64_t mask, double& lp) {
    (log_density_one<Bs>(acc, s, p, mask, lp), ...);
  }
  template <class Blk, class B, class T>
  __device__ __forceinline__ static void log_density_one(VarAccess<B, T>& acc, bi::State<B, bi::ON_DEVICE>& s, int p,
                                                         uint64_t mask, double& lp) {
    static_assert(std::is_same<Blk, pdf_block<typename Blk::action_typelist>>::value,
                  "an observation block holds pdf actions only");
    LogDensityVisit<B, T> f{s, acc, p, mask, lp};
    tree<typename Blk::action_typelist>::each(f);
  }
};

/* ---- the fused kernels --------------------------------------------------------- */
constexpr int kModelBlock = 128;

template <class B, class T>
struct ModelStepArgs {
  const T* x_in;
  T* x_out;
  int ld, n;
  int* as;
  double* lw;
  const T* y;
  uint64_t obs_mask;
  double t1, t2;
  uint64_t seed;
  int step;
  StepStats* stats;
  LwPartial* partials;
  unsigned* counter;
  T prm[ParticleVars<B, T>::kNP];
};

template <class B> constexpr int state_columns() { return B::ND + B::NDX; }

template <class B, class T>
__device__ __forceinline__ void load_particle(ParticleVars<B, T>& v, const T* __restrict__ x, int ld, int src) {
#pragma unroll
  for (int j = 0; j < B::ND; ++j) v.d[j] = __ldg(x + (size_t)j * ld + src);
#pragma unroll
  for (int j = 0; j < B::NDX; ++j) v.dx[j] = __ldg(x + (size_t)(B::ND + j) * ld + src);
}

template <class B, class T>
__device__ __forceinline__ void store_particle(const ParticleVars<B, T>& v, T* __restrict__ x, int ld, int p) {
#pragma unroll
  for (int j = 0; j < B::ND; ++j) x[(size_t)j * ld + p] = v.d[j];
#pragma unroll
  for (int j = 0; j < B::NDX; ++j) x[(size_t)(B::ND + j) * ld + p] = v.dx[j];
}

/* Resident blocks per SM the fused kernel is compiled for: 4 (at most 128
 * registers a thread) in FP32, 2 in FP64, where a particle's state takes
 * twice the registers.  A model with a larger state can specialise this. */
template <class B, class T> struct model_min_blocks {
  static constexpr int value = sizeof(T) == 4 ? 4 : 2;
};

/* One BootstrapPF::step of the model for every particle: gather from the
 * ancestor when the previous step resampled, transition blocks, observation
 * log-density, and the log-weight reduction of the step (bpf_device.cuh). */
template <class B, class T>
__global__ void __launch_bounds__(kModelBlock, (model_min_blocks<B, T>::value))
k_model_transition(const ModelStepArgs<B, T> a) {
  extern __shared__ unsigned char bpf_model_smem[];
  pdl_wait();  // the resampler's ancestors and statistics
  StepStats* st = a.stats;
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  const int resampled = st->resample;
  const bool ok = st->status == BPF_OK;
  LwPartial part = lw_empty();
  if (ok && p < a.n) {
    const int src = resampled ? a.as[p] : p;
    ParticleVars<B, T> v;
    v.r = reinterpret_cast<T*>(bpf_model_smem) + threadIdx.x;
    v.rstride = blockDim.x;
#pragma unroll
    for (int j = 0; j < ParticleVars<B, T>::kNP; ++j) v.p[j] = a.prm[j];
    load_particle<B, T>(v, a.x_in, a.ld, src);
    bi::State<B, bi::ON_DEVICE> s;
    VarAccess<B, T> acc{v};
    ParticleRng<T> rng(a.seed, (uint32_t)p, (uint32_t)a.step, BPF_RNG_NOISE);
    run_blocks<typename B::transition_type>::template sample<B, T>(v, acc, s, rng, p, a.t1, a.t2);
    store_particle<B, T>(v, a.x_out, a.ld, p);
    double l = resampled ? st->ll : a.lw[p];
    if (a.y) {
#pragma unroll
      for (int j = 0; j < B::NO; ++j) v.o[j] = __ldg(a.y + j);
      run_blocks<typename B::observation_type>::template log_density<B, T>(acc, s, p, a.obs_mask, l);
    }
    a.lw[p] = l;
    if (resampled) a.as[p] = src;
    lw_push(part, l);
  }
  pdl_trigger();
  transition_reduce_tail(part, a.partials, blockIdx.x, 0, gridDim.x, a.counter, a.n, st, ok, resampled,
                         a.y != nullptr);
}

/* Simulator::init through the model's initial block: draws with step 0 and
 * the tag BPF_RNG_INIT; log-weights zero. */
template <class B, class T>
__global__ void __launch_bounds__(kModelBlock) k_model_init(T* x, int ld, int n, double* lw, uint64_t seed,
                                                           const ModelStepArgs<B, T> a) {
  extern __shared__ unsigned char bpf_model_smem[];
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  ParticleVars<B, T> v;
  v.r = reinterpret_cast<T*>(bpf_model_smem) + threadIdx.x;
  v.rstride = blockDim.x;
#pragma unroll
  for (int j = 0; j < ParticleVars<B, T>::kNP; ++j) v.p[j] = a.prm[j];
#pragma unroll
  for (int j = 0; j < B::ND; ++j) v.d[j] = (T)0;
#pragma unroll
  for (int j = 0; j < B::NDX; ++j) v.dx[j] = (T)0;
  bi::State<B, bi::ON_DEVICE> s;
  VarAccess<B, T> acc{v};
  ParticleRng<T> rng(seed, (uint32_t)p, 0u, BPF_RNG_INIT);
  run_blocks<typename B::initial_type>::template sample<B, T>(v, acc, s, rng, p, 0.0, 0.0);
  store_particle<B, T>(v, x, ld, p);
  lw[p] = 0.0;
}

template <class B> constexpr size_t noise_smem_bytes() {
  return (size_t)(B::NR > 0 ? B::NR : 1) * kModelBlock * sizeof(real);
}

/* ---- the launchers behind bpf_model_ops ----------------------------------------- */
template <class B, class T>
inline void fill_params(ModelStepArgs<B, T>& a, const double* params, int nparams) {
  for (int j = 0; j < ParticleVars<B, T>::kNP; ++j) a.prm[j] = (T)(params && j < nparams ? params[j] : 0.0);
}

template <class B>
int model_transition_launch(const bpf_transition_args* t, void* stream) {
  typedef real T;
  ModelStepArgs<B, T> a;
  a.x_in = (const T*)t->x_in;
  a.x_out = (T*)t->x_out;
  a.ld = t->ld;
  a.n = t->n;
  a.as = t->ancestors;
  a.lw = t->lw;
  a.y = (const T*)t->y;
  a.obs_mask = t->obs_mask;
  a.t1 = t->t1;
  a.t2 = t->t2;
  a.seed = t->seed;
  a.step = t->step;
  a.stats = (StepStats*)t->stats;
  a.partials = (LwPartial*)t->partials;
  a.counter = t->counter;
  fill_params<B, T>(a, t->params, t->nparams);
  const int blocks = (t->n + kModelBlock - 1) / kModelBlock;
  if (blocks > t->max_partials) return BPF_E_INVALID;
  // a programmatic dependent of the resampler before it, as the library's
  // own transitions are
  return launch_pdl(k_model_transition<B, T>, dim3(blocks), dim3(kModelBlock), noise_smem_bytes<B>(),
                    (cudaStream_t)stream, a) == cudaSuccess
             ? BPF_OK
             : BPF_E_CUDA;
}

template <class B>
int model_init_launch(const bpf_init_args* t, void* stream) {
  typedef real T;
  ModelStepArgs<B, T> a{};
  fill_params<B, T>(a, t->params, t->nparams);
  const int blocks = (t->n + kModelBlock - 1) / kModelBlock;
  k_model_init<B, T><<<blocks, kModelBlock, noise_smem_bytes<B>(), (cudaStream_t)stream>>>((T*)t->x, t->ld, t->n,
                                                                                            t->lw, t->seed, a);
  return cudaGetLastError() == cudaSuccess ? BPF_OK : BPF_E_CUDA;
}

/* The table bpf_create_model takes for model class B in precision `real`. */
template <class B>
inline bpf_model_ops model_ops() {
  static_assert(B::NF == 0, "input (F_VAR) variables are not supported in a device model");
  static_assert(B::NO <= 64, "at most 64 observed elements (the step's observation mask)");
  static_assert(noise_smem_bytes<B>() <= 48 * 1024, "noise variables exceed the kernel's shared memory");
  bpf_model_ops o{};
  o.dim = state_columns<B>();
  o.nobs = B::NO;
  o.nparams = B::NP;
  o.precision = sizeof(real) == 4 ? BPF_F32 : BPF_F64;
  o.init = &model_init_launch<B>;
  o.transition = &model_transition_launch<B>;
  return o;
}

}  // namespace bpf

/* ---- the block updaters, one kernel each ------------------------------------------ */
namespace bpf {

/* one particle's variables from / to a device State<B, ON_DEVICE> */
template <class B, class T>
__device__ __forceinline__ void load_state(ParticleVars<B, T>& v, const bi::State<B, bi::ON_DEVICE>& s, int p) {
  v.r = nullptr;
#pragma unroll
  for (int j = 0; j < B::ND; ++j) v.d[j] = s.x[(size_t)j * s.ld + p];
#pragma unroll
  for (int j = 0; j < B::NDX; ++j) v.dx[j] = s.x[(size_t)(B::ND + j) * s.ld + p];
#pragma unroll
  for (int j = 0; j < B::NP; ++j) v.p[j] = s.prm[j];
}

template <class B, class T>
__device__ __forceinline__ void load_noise(ParticleVars<B, T>& v, const bi::State<B, bi::ON_DEVICE>& s, int p,
                                           T* smem) {
  v.r = smem + threadIdx.x;
  v.rstride = blockDim.x;
  if (s.r) {
#pragma unroll
    for (int j = 0; j < B::NR; ++j) v.r[j * v.rstride] = s.r[(size_t)j * s.ld + p];
  }
}

template <class B, class T>
__device__ __forceinline__ void store_state(const ParticleVars<B, T>& v, const bi::State<B, bi::ON_DEVICE>& s, int p) {
#pragma unroll
  for (int j = 0; j < B::ND; ++j) s.x[(size_t)j * s.ld + p] = v.d[j];
#pragma unroll
  for (int j = 0; j < B::NDX; ++j) s.x[(size_t)(B::ND + j) * s.ld + p] = v.dx[j];
  if (s.r) {
#pragma unroll
    for (int j = 0; j < B::NR; ++j) s.r[(size_t)j * s.ld + p] = v.r[j * v.rstride];
  }
}

/* kind: 0 noise draws (StaticSampler), 1 deterministic update
 * (StaticUpdater), 2 RK4, 3 RK4(3) */
template <class B, class T, class S, int KIND>
__global__ void __launch_bounds__(kModelBlock) k_block_update(bi::State<B, bi::ON_DEVICE> s, uint64_t seed,
                                                              double t1, double t2, double h, double atoler,
                                                              double rtoler) {
  extern __shared__ unsigned char bpf_model_smem[];
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= s.n) return;
  ParticleVars<B, T> v;
  load_state<B, T>(v, s, p);
  load_noise<B, T>(v, s, p, reinterpret_cast<T*>(bpf_model_smem));
  VarAccess<B, T> acc{v};
  if constexpr (KIND == 0) {
    ParticleRng<T> rng(seed, (uint32_t)p, (uint32_t)s.step, s.step == 0 ? BPF_RNG_INIT : BPF_RNG_NOISE);
    SampleVisit<B, T> f{s, acc, rng, p};
    tree<S>::each(f);
  } else if constexpr (KIND == 1) {
    SimulateVisit<B, T> f{s, acc, p};
    tree<S>::each(f);
  } else if constexpr (KIND == 2) {
    ode_rk4<B, T, S>(v, acc, s, p, t1, t2, h);
  } else {
    ode_rk43<B, T, S>(v, acc, s, p, t1, t2, h, atoler, rtoler);
  }
  store_state<B, T>(v, s, p);
}

template <class B, class T, class S>
__global__ void __launch_bounds__(kModelBlock) k_block_log_density(bi::State<B, bi::ON_DEVICE> s, uint64_t mask,
                                                                   double* lp) {
  extern __shared__ unsigned char bpf_model_smem[];
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= s.n) return;
  ParticleVars<B, T> v;
  load_state<B, T>(v, s, p);
  load_noise<B, T>(v, s, p, reinterpret_cast<T*>(bpf_model_smem));
#pragma unroll
  for (int j = 0; j < B::NO; ++j) v.o[j] = s.y[j];
  VarAccess<B, T> acc{v};
  double l = lp[p];
  LogDensityVisit<B, T> f{s, acc, p, mask, l};
  tree<S>::each(f);
  lp[p] = l;
}

template <class B, class S, int KIND>
inline void block_update(bi::State<B, bi::ON_DEVICE>& s, uint64_t seed, double t1, double t2, double h,
                         double atoler, double rtoler) {
  if (s.n <= 0) return;
  const int blocks = (s.n + kModelBlock - 1) / kModelBlock;
  k_block_update<B, real, S, KIND><<<blocks, kModelBlock, noise_smem_bytes<B>(), s.stream>>>(s, seed, t1, t2, h,
                                                                                             atoler, rtoler);
  if (cudaGetLastError() != cudaSuccess) throw std::runtime_error("block updater launch failed");
}

}  // namespace bpf

namespace bi {

/* The integrator constants the generated ode block sets before it integrates
 * (bi_ode_set, share/src/bi/ode/IntegratorConstants.hpp:38-57, called from
 * share/tt/cpp/block/ode.hpp.tt): the step h (initial step for RK4(3)) and
 * the tolerances. */
struct OdeConstants {
  double h = 1.0e-2, atoler = 1.0e-3, rtoler = 1.0e-3;
};
inline OdeConstants& ode_constants() {
  static OdeConstants c;
  return c;
}
inline void bi_ode_set(double h, double atoler, double rtoler) {
  ode_constants() = OdeConstants{h, atoler, rtoler};
}

/* StaticSampler<B,S>::samples (share/src/bi/updater/StaticSampler.hpp; block/pdf_.hpp.tt:46-75):
 * draws the actions of S for every particle of s into their targets (R_VAR
 * columns in s.r, D_VAR / DX_VAR columns in s.x), with the draws of the
 * particle's step s.step (0: the initial block's stream) under rng.seed,
 * the same numbers as the fused kernel's first noise block. */
template <class B, class S>
struct StaticSampler {
  template <class R1>
  static void samples(R1& rng, State<B, ON_DEVICE>& s) {
    bpf::block_update<B, S, 0>(s, rng.seed, 0.0, 0.0, 0.0, 0.0, 0.0);
  }
};

/* StaticUpdater<B,S>::update (block/eval_.hpp.tt): the deterministic actions of S */
template <class B, class S>
struct StaticUpdater {
  static void update(State<B, ON_DEVICE>& s) { bpf::block_update<B, S, 1>(s, 0, 0.0, 0.0, 0.0, 0.0, 0.0); }
};

/* RK4Integrator<B,S>::update (share/src/bi/ode/RK4Integrator.hpp;
 * block/ode.hpp.tt:39-54) from t1 to t2 with the step of bi_ode_set */
template <class B, class S, class T1 = real>
struct RK4Integrator {
  static void update(const T1 t1, const T1 t2, State<B, ON_DEVICE>& s) {
    const OdeConstants& c = ode_constants();
    bpf::block_update<B, S, 2>(s, 0, (double)t1, (double)t2, c.h, c.atoler, c.rtoler);
  }
};

/* RK43Integrator<B,S>::update (share/src/bi/ode/RK43Integrator.hpp) */
template <class B, class S, class T1 = real>
struct RK43Integrator {
  static void update(const T1 t1, const T1 t2, State<B, ON_DEVICE>& s) {
    const OdeConstants& c = ode_constants();
    bpf::block_update<B, S, 3>(s, 0, (double)t1, (double)t2, c.h, c.atoler, c.rtoler);
  }
};

/* SparseStaticLogDensity<B,S>::logDensities
 * (share/src/bi/updater/SparseStaticLogDensity.hpp; block/pdf_.hpp.tt:46-75):
 * adds each particle's observation terms to lp[p] (device, FP64), for the
 * O_VAR elements whose bit is set in mask, the observed values in s.y */
template <class B, class S>
struct SparseStaticLogDensity {
  static void logDensities(State<B, ON_DEVICE>& s, uint64_t mask, double* lp) {
    if (s.n <= 0) return;
    const int blocks = (s.n + bpf::kModelBlock - 1) / bpf::kModelBlock;
    bpf::k_block_log_density<B, real, S><<<blocks, bpf::kModelBlock, bpf::noise_smem_bytes<B>(), s.stream>>>(
        s, mask, lp);
    if (cudaGetLastError() != cudaSuccess) throw std::runtime_error("log-density launch failed");
  }
};

}  // namespace bi

namespace bi_b200 {

/* A model class compiled against this header, as the filter classes of
 * libbi_b200.hpp take it: BootstrapPFState<DeviceModel<Model>>,
 * BootstrapPF<DeviceModel<Model>, O, R>.  params: the P_VAR values. */
template <class B>
struct DeviceModel {
  typedef ::real real;
  std::vector<double> params;
  DeviceModel() = default;
  explicit DeviceModel(const std::vector<double>& p) : params(p) {}
  bpf_model_ops ops() const { return bpf::model_ops<B>(); }
  int nobs() const { return B::NO; }
  size_t esz() const { return sizeof(real); }
};

}  // namespace bi_b200

#endif
