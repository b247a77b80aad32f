// Lorenz '96 (d = 40) as LibBi's code generator renders it, written out by
// hand from the generator's templates (share/tt/cpp/var.hpp.tt,
// var_coord.hpp.tt with a cyclic boundary, action_coord.hpp.tt,
// action/gaussian.hpp.tt, action/ode_.hpp.tt, action/eval_.hpp.tt,
// macro/fetch_parents.hpp.tt, macro/put_output.hpp.tt,
// macro/create_action_typetree.hpp.tt, the size constants of
// model.hpp.tt:67-78), for include/bpf_model.cuh:
//
//   model L96 {
//     const N = 40;  const SIGMA_ETA = 0.1;  const SIGMA_Y = 1.0;  const X0_STD = 0.01
//     dim n(size = N, boundary = 'cyclic')
//     param F
//     state x[n];  noise eta[n];  obs y[n]
//     sub initial { x[n] ~ gaussian(F, X0_STD) }
//     sub transition(delta = 0.05) {
//       eta[n] ~ gaussian(0.0, SIGMA_ETA)
//       ode(alg = 'RK4', h = 0.01) { dx[n]/dt = (x[n+1] - x[n-2])*x[n-1] - x[n] + F }
//       x[n] <- x[n] + eta[n]
//     }
//     sub observation { y[n] ~ gaussian(x[n], SIGMA_Y) }
//   }
//
// The forcing F is a parameter here (one value per filter, as in the batched
// workload), where docs/src/users.tex:354-358 keeps it a constant.
#pragma once
#include "bpf_model.cuh"

namespace l96_gen {

static const int N = 40;
class ModelL96;

/* variables and their cyclic coordinates (var.hpp.tt, var_coord.hpp.tt) */
#define L96_VAR(ID_, START_, TYPE_)                                             \
  class VarCoord##ID_ {                                                         \
   public:                                                                      \
    CUDA_FUNC_BOTH VarCoord##ID_() { i0 = 0; }                                  \
    CUDA_FUNC_BOTH VarCoord##ID_(const int i) { i0 = (i + N0) % N0; }          \
    CUDA_FUNC_BOTH void inc() { if (i0 < N0 - 1) ++i0; else i0 = 0; }          \
    CUDA_FUNC_BOTH int index() const { return i0; }                             \
    CUDA_FUNC_BOTH void setIndex(const int ix) { i0 = ix; }                     \
    CUDA_FUNC_BOTH VarCoord##ID_& operator++() { inc(); return *this; }        \
    int i0;                                                                     \
    static const int N0 = N;                                                    \
  };                                                                            \
  class Var##ID_ {                                                              \
   public:                                                                      \
    typedef VarCoord##ID_ coord_type;                                           \
    static const int ID = ID_;                                                  \
    static const int START = START_;                                            \
    static const int SIZE = N;                                                  \
    static const int NUM_DIMS = 1;                                              \
    static const bi::VarType TYPE = bi::TYPE_;                                  \
  };
L96_VAR(0, 0, D_VAR)  // state x[n]
L96_VAR(1, 0, R_VAR)  // noise eta[n]
L96_VAR(2, 0, O_VAR)  // obs y[n]
#undef L96_VAR

/* param F */
struct ScalarCoord {
  CUDA_FUNC_BOTH ScalarCoord() {}
  CUDA_FUNC_BOTH int index() const { return 0; }
  CUDA_FUNC_BOTH ScalarCoord& operator++() { return *this; }
};
class Var3 {
 public:
  typedef ScalarCoord coord_type;
  static const int ID = 3;
  static const int START = 0;
  static const int SIZE = 1;
  static const int NUM_DIMS = 0;
  static const bi::VarType TYPE = bi::P_VAR;
};

/* the action coordinate over the alias n (action_coord.hpp.tt) */
class ActionCoordN {
 public:
  CUDA_FUNC_BOTH ActionCoordN() { i0 = OFFSET0; }
  CUDA_FUNC_BOTH ActionCoordN(const int ix) { setIndex(ix); }
  CUDA_FUNC_BOTH void inc() { if (i0 < OFFSET0 + LEN0 - 1) ++i0; else i0 = OFFSET0; }
  CUDA_FUNC_BOTH int index() const { return i0; }
  CUDA_FUNC_BOTH void setIndex(const int ix) { i0 = OFFSET0 + ix; }
  CUDA_FUNC_BOTH ActionCoordN& operator++() { inc(); return *this; }
  int i0;
  static const int OFFSET0 = 0;
  static const int LEN0 = N;
  static const int N0 = N;
};

/* x[n] ~ gaussian(F, X0_STD)  (initial; gaussian.hpp.tt, sample) */
class Action0 {
 public:
  typedef Var0 target_type;
  typedef ActionCoordN coord_type;
  static const int SIZE = N;
  static const bool IS_MATRIX = false;
  template <class R1, bi::Location L, class CX, class PX, class OX>
  static CUDA_FUNC_BOTH void samples(R1& rng, bi::State<ModelL96, L>& s, const int p, const int ix, const CX& cox,
                                     const PX& pax, OX& x) {
    BI_UNUSED const int n_ = cox.i0;
    /* constants */
    const BOOST_AUTO(X0_STD, BI_REAL(0.01));
    /* variables */
    const BOOST_AUTO(F, pax.template fetch<Var3>(s, p, 0));
    const CX& cox_ = cox;
    real mu = F;
    real sigma = X0_STD;
    real u = rng.gaussian(mu, sigma);
    x.template fetch<target_type>(s, p, cox_.index()) = u;
  }
};

/* eta[n] ~ gaussian(0.0, SIGMA_ETA)  (transition; gaussian.hpp.tt, sample) */
class Action1 {
 public:
  typedef Var1 target_type;
  typedef ActionCoordN coord_type;
  static const int SIZE = N;
  static const bool IS_MATRIX = false;
  template <class R1, bi::Location L, class CX, class PX, class OX>
  static CUDA_FUNC_BOTH void samples(R1& rng, bi::State<ModelL96, L>& s, const int p, const int ix, const CX& cox,
                                     const PX& pax, OX& x) {
    BI_UNUSED const int n_ = cox.i0;
    /* constants */
    const BOOST_AUTO(SIGMA_ETA, BI_REAL(0.1));
    const CX& cox_ = cox;
    real mu = BI_REAL(0.0);
    real sigma = SIGMA_ETA;
    real u = rng.gaussian(mu, sigma);
    x.template fetch<target_type>(s, p, cox_.index()) = u;
  }
};

/* dx[n]/dt = (x[n+1] - x[n-2])*x[n-1] - x[n] + F  (transition; ode_.hpp.tt) */
class Action2 {
 public:
  typedef Var0 target_type;
  typedef ActionCoordN coord_type;
  static const int SIZE = N;
  static const bool IS_MATRIX = false;
  template <class T1, bi::Location L, class CX, class PX, class T2>
  static CUDA_FUNC_BOTH void dfdt(const T1 t, const bi::State<ModelL96, L>& s, const int p, const CX& cox,
                                  const PX& pax, T2& dfdt) {
    BI_UNUSED const int n_ = cox.i0;
    /* variables */
    const VarCoord0 cox0(n_ + 1);
    const BOOST_AUTO(x_n_plus_1, pax.template fetch<Var0>(s, p, cox0.index()));
    const VarCoord0 cox1(n_ - 2);
    const BOOST_AUTO(x_n_minus_2, pax.template fetch<Var0>(s, p, cox1.index()));
    const VarCoord0 cox2(n_ - 1);
    const BOOST_AUTO(x_n_minus_1, pax.template fetch<Var0>(s, p, cox2.index()));
    const VarCoord0 cox3(n_);
    const BOOST_AUTO(x_n, pax.template fetch<Var0>(s, p, cox3.index()));
    const BOOST_AUTO(F, pax.template fetch<Var3>(s, p, 0));
    dfdt = (x_n_plus_1 - x_n_minus_2) * x_n_minus_1 - x_n + F;
  }
};

/* x[n] <- x[n] + eta[n]  (transition; eval_.hpp.tt) */
struct Action3 {
  typedef Var0 target_type;
  typedef ActionCoordN coord_type;
  static const int SIZE = N;
  static const bool IS_MATRIX = false;
  template <bi::Location L, class CX, class PX, class OX>
  static CUDA_FUNC_BOTH void simulates(bi::State<ModelL96, L>& s, const int p, const int ix, const CX& cox,
                                       const PX& pax, OX& x) {
    BI_UNUSED const int n_ = cox.i0;
    const VarCoord0 cox0(n_);
    const BOOST_AUTO(x_n, pax.template fetch<Var0>(s, p, cox0.index()));
    const VarCoord1 cox1(n_);
    const BOOST_AUTO(eta_n, pax.template fetch<Var1>(s, p, cox1.index()));
    const CX& cox_ = cox;
    x.template fetch<target_type>(s, p, cox_.index()) = x_n + eta_n;
  }
};

/* y[n] ~ gaussian(x[n], SIGMA_Y)  (observation; gaussian.hpp.tt, logdensity) */
class Action4 {
 public:
  typedef Var2 target_type;
  typedef ActionCoordN coord_type;
  static const int SIZE = N;
  static const bool IS_MATRIX = false;
  template <bi::Location L, class CX, class PX, class OX, class T1>
  static CUDA_FUNC_BOTH void logDensities(bi::State<ModelL96, L>& s, const int p, const int ix, const CX& cox,
                                          const PX& pax, OX& x, T1& lp) {
    BI_UNUSED const int n_ = cox.i0;
    /* constants */
    const BOOST_AUTO(SIGMA_Y, BI_REAL(1.0));
    /* variables */
    const VarCoord0 cox0(n_);
    const BOOST_AUTO(x_n, pax.template fetch<Var0>(s, p, cox0.index()));
    const CX& cox_ = cox;
    real mu = x_n;
    real sigma = SIGMA_Y;
    real xy = pax.template fetch_alt<target_type>(s, p, cox_.index());
    if (sigma == 0) {
      if (xy == mu) {
        lp = BI_INF;
      } else {
        lp = -BI_INF;
      }
    } else {
      lp += BI_REAL(-0.5) * bi::pow((xy - mu) / sigma, BI_REAL(2.0)) - BI_REAL(BI_HALF_LOG_TWO_PI) -
            bi::log(sigma);
    }
    x.template fetch<target_type>(s, p, cox_.index()) = xy;
  }
};

BEGIN_TYPETREE(Block0ActionTypeList) LEAF_NODE(1, Action0) END_TYPETREE()
BEGIN_TYPETREE(Block1ActionTypeList) LEAF_NODE(1, Action1) END_TYPETREE()
BEGIN_TYPETREE(Block2ActionTypeList) LEAF_NODE(1, Action2) END_TYPETREE()
BEGIN_TYPETREE(Block3ActionTypeList) LEAF_NODE(1, Action3) END_TYPETREE()
BEGIN_TYPETREE(Block4ActionTypeList) LEAF_NODE(1, Action4) END_TYPETREE()

/* the ode block's arguments (block/ode.hpp.tt: alg, h, atoler, rtoler) */
struct Block2Ode {
  static const int alg = bpf::ODE_RK4;
  static constexpr double h = 0.01, atoler = 1.0e-3, rtoler = 1.0e-3;
};

class ModelL96 {
 public:
  static const int NR = N, ND = N, NP = 1, NF = 0, NO = N, NDX = 0, NPX = 0, NB = 0;
  static const int CR = 1, CD = 1, CP = 1, CF = 0, CO = 1, CDX = 0, CPX = 0, CB = 0;
  typedef bpf::blocks<bpf::pdf_block<GET_TYPETREE(Block0ActionTypeList)>> initial_type;
  typedef bpf::blocks<bpf::pdf_block<GET_TYPETREE(Block1ActionTypeList)>,
                      bpf::ode_block<GET_TYPETREE(Block2ActionTypeList), Block2Ode>,
                      bpf::eval_block<GET_TYPETREE(Block3ActionTypeList)>>
      transition_type;
  typedef bpf::blocks<bpf::pdf_block<GET_TYPETREE(Block4ActionTypeList)>> observation_type;
};

}  // namespace l96_gen
