// The models in the generated form (model_test_ar1.cuh,
// model_l96_generated.cuh) compiled into a shared library that hands their
// bpf_model_ops tables to a caller (the Python tests, through ctypes, pass
// them to bpf_create_model).  Built twice: -DBPF_REAL=double and
// -DBPF_REAL=float, both with -fmad=false (expression order of the model
// source).
#include "bpf_model.cuh"
#include "model_test_ar1.cuh"
#include "model_l96_generated.cuh"

extern "C" bpf_model_ops test_ar1_ops(void) { return bpf::model_ops<test_ar1::ModelTest>(); }
extern "C" bpf_model_ops test_l96_ops(void) { return bpf::model_ops<l96_gen::ModelL96>(); }

// One transition and observation of every particle through the unfused
// block updaters, in the order the generated transition and observation
// blocks call them (block/transition.hpp.tt, pdf_.hpp.tt, ode.hpp.tt,
// eval_.hpp.tt): all pointers are device pointers of a State<B, ON_DEVICE>
// (x: D_VAR columns, r: R_VAR columns, prm: P_VAR values, y: the
// observation, lp: FP64 log-densities added to).  Returns 0, or 2 when an
// updater threw, 3 on a CUDA error.
namespace {
struct SeedOnly {
  uint64_t seed;
};

template <class M, class Noise, class Ode, class Eval, class Obs>
int unfused_step(real* x, real* r, int ld, int n, const real* prm, const real* y, double t1, double t2,
                 uint64_t seed, int step, double* lp, double h) {
  bi::State<M, bi::ON_DEVICE> s;
  s.x = x;
  s.r = r;
  s.prm = prm;
  s.y = y;
  s.ld = ld;
  s.n = n;
  s.step = step;
  SeedOnly rng{seed};
  try {
    bi::StaticSampler<M, Noise>::samples(rng, s);
    if constexpr (!std::is_same<Ode, void>::value) {
      bi::bi_ode_set(h, 1.0e-3, 1.0e-3);
      bi::RK4Integrator<M, Ode>::update((real)t1, (real)t2, s);
    }
    bi::StaticUpdater<M, Eval>::update(s);
    bi::SparseStaticLogDensity<M, Obs>::logDensities(s, ~0ull, lp);
  } catch (const std::exception&) {
    return 2;
  }
  return cudaDeviceSynchronize() == cudaSuccess ? 0 : 3;
}
}  // namespace

extern "C" int test_l96_unfused_step(real* x, real* r, int ld, int n, const real* prm, const real* y, double t1,
                                     double t2, uint64_t seed, int step, double* lp) {
  using namespace l96_gen;
  return unfused_step<ModelL96, GET_TYPETREE(Block1ActionTypeList), GET_TYPETREE(Block2ActionTypeList),
                      GET_TYPETREE(Block3ActionTypeList), GET_TYPETREE(Block4ActionTypeList)>(
      x, r, ld, n, prm, y, t1, t2, seed, step, lp, Block2Ode::h);
}

extern "C" int test_ar1_unfused_step(real* x, real* r, int ld, int n, const real* prm, const real* y, double t1,
                                     double t2, uint64_t seed, int step, double* lp) {
  using namespace test_ar1;
  return unfused_step<ModelTest, GET_TYPETREE(Block2ActionTypeList), void, GET_TYPETREE(Block3ActionTypeList),
                      GET_TYPETREE(Block4ActionTypeList)>(x, r, ld, n, prm, y, t1, t2, seed, step, lp, 0.0);
}
