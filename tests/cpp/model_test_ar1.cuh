// A model class in the shape LibBi's code generator emits for the
// reference's own example model Test.bi (an AR(1) process), rendered by hand
// from the generator's templates (share/tt/cpp/model.hpp.tt:60-78 size
// constants, var.hpp.tt, var_coord.hpp.tt, action/gaussian.hpp.tt sample
// and logdensity, action/eval_.hpp.tt, macro/fetch_parents.hpp.tt,
// macro/put_output.hpp.tt, macro/create_action_typetree.hpp.tt), with one
// addition that Test.bi lacks and a filter needs, an observation block:
//
//   model Test {
//     param theta, sigma2
//     noise w
//     state x
//     obs y                                   // added
//     sub initial { x ~ gaussian() }
//     sub transition { w ~ gaussian(0.0, sqrt(sigma2)); x <- theta*x + w }
//     sub observation { y ~ gaussian(x, 0.5) } // added
//   }
//
// (sub parameter draws theta and sigma2 from their priors; a filter takes
// them fixed, as the P_VAR values of bpf_create_model.)  The action bodies
// are the generator's, statement for statement; only the blocks' grouping
// into bpf::blocks<...> is added for include/bpf_model.cuh.
#pragma once
#include "bpf_model.cuh"

namespace test_ar1 {

class ModelTest;

/* scalar variables: a coordinate with no dimensions (var_coord.hpp.tt) */
struct ScalarCoord {
  CUDA_FUNC_BOTH ScalarCoord() {}
  CUDA_FUNC_BOTH ScalarCoord(const int) {}
  CUDA_FUNC_BOTH int index() const { return 0; }
  CUDA_FUNC_BOTH void setIndex(const int) {}
  CUDA_FUNC_BOTH ScalarCoord& operator++() { return *this; }
};

#define TEST_VAR(NAME, ID_, START_, TYPE_)         \
  class NAME {                                     \
   public:                                         \
    typedef ScalarCoord coord_type;                \
    static const int ID = ID_;                     \
    static const int START = START_;               \
    static const int SIZE = 1;                     \
    static const int NUM_DIMS = 0;                 \
    static const bi::VarType TYPE = bi::TYPE_;     \
  };
TEST_VAR(Var0, 0, 0, P_VAR)  // param theta
TEST_VAR(Var1, 1, 1, P_VAR)  // param sigma2
TEST_VAR(Var2, 2, 0, R_VAR)  // noise w
TEST_VAR(Var3, 3, 0, D_VAR)  // state x
TEST_VAR(Var4, 4, 0, O_VAR)  // obs y
#undef TEST_VAR

/* x ~ gaussian()  (initial; action/gaussian.hpp.tt, sample) */
class Action0 {
 public:
  typedef Var3 target_type;
  typedef ScalarCoord coord_type;
  static const int SIZE = 1;
  static const bool IS_MATRIX = false;
  template <class R1, bi::Location L, class CX, class PX, class OX>
  static CUDA_FUNC_BOTH void samples(R1& rng, bi::State<ModelTest, L>& s, const int p, const int ix,
                                     const CX& cox, const PX& pax, OX& x) {
    const CX& cox_ = cox;
    real mu = BI_REAL(0.0);
    real sigma = BI_REAL(1.0);
    real u = rng.gaussian(mu, sigma);
    x.template fetch<target_type>(s, p, cox_.index()) = u;
  }
};

/* w ~ gaussian(0.0, sqrt(sigma2))  (transition; gaussian.hpp.tt, sample) */
class Action1 {
 public:
  typedef Var2 target_type;
  typedef ScalarCoord coord_type;
  static const int SIZE = 1;
  static const bool IS_MATRIX = false;
  template <class R1, bi::Location L, class CX, class PX, class OX>
  static CUDA_FUNC_BOTH void samples(R1& rng, bi::State<ModelTest, L>& s, const int p, const int ix,
                                     const CX& cox, const PX& pax, OX& x) {
    /* variables */
    const BOOST_AUTO(sigma2, pax.template fetch<Var1>(s, p, 0));
    const CX& cox_ = cox;
    real mu = BI_REAL(0.0);
    real sigma = bi::sqrt(sigma2);
    real u = rng.gaussian(mu, sigma);
    x.template fetch<target_type>(s, p, cox_.index()) = u;
  }
};

/* x <- theta*x + w  (transition; action/eval_.hpp.tt) */
struct Action2 {
  typedef Var3 target_type;
  typedef ScalarCoord coord_type;
  static const int SIZE = 1;
  static const bool IS_MATRIX = false;
  template <bi::Location L, class CX, class PX, class OX>
  static CUDA_FUNC_BOTH void simulates(bi::State<ModelTest, L>& s, const int p, const int ix, const CX& cox,
                                       const PX& pax, OX& x) {
    /* variables */
    const BOOST_AUTO(theta, pax.template fetch<Var0>(s, p, 0));
    const BOOST_AUTO(x_, pax.template fetch<Var3>(s, p, 0));
    const BOOST_AUTO(w, pax.template fetch<Var2>(s, p, 0));
    const CX& cox_ = cox;
    x.template fetch<target_type>(s, p, cox_.index()) = theta * x_ + w;
  }
};

/* y ~ gaussian(x, 0.5)  (observation; gaussian.hpp.tt, logdensity) */
class Action3 {
 public:
  typedef Var4 target_type;
  typedef ScalarCoord coord_type;
  static const int SIZE = 1;
  static const bool IS_MATRIX = false;
  template <bi::Location L, class CX, class PX, class OX, class T1>
  static CUDA_FUNC_BOTH void logDensities(bi::State<ModelTest, L>& s, const int p, const int ix, const CX& cox,
                                          const PX& pax, OX& x, T1& lp) {
    /* variables */
    const BOOST_AUTO(x_, pax.template fetch<Var3>(s, p, 0));
    const CX& cox_ = cox;
    real mu = x_;
    real sigma = BI_REAL(0.5);
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

/* the blocks' action type trees (macro/create_action_typetree.hpp.tt) */
BEGIN_TYPETREE(Block1ActionTypeList) LEAF_NODE(1, Action0) END_TYPETREE()
BEGIN_TYPETREE(Block2ActionTypeList) LEAF_NODE(1, Action1) END_TYPETREE()
BEGIN_TYPETREE(Block3ActionTypeList) LEAF_NODE(1, Action2) END_TYPETREE()
BEGIN_TYPETREE(Block4ActionTypeList) LEAF_NODE(1, Action3) END_TYPETREE()

/* the model: size constants (model.hpp.tt:67-78) and its top-level blocks */
class ModelTest {
 public:
  static const int NR = 1, ND = 1, NP = 2, NF = 0, NO = 1, NDX = 0, NPX = 0, NB = 0;
  static const int CR = 1, CD = 1, CP = 2, CF = 0, CO = 1, CDX = 0, CPX = 0, CB = 0;
  typedef bpf::blocks<bpf::pdf_block<GET_TYPETREE(Block1ActionTypeList)>> initial_type;
  typedef bpf::blocks<bpf::pdf_block<GET_TYPETREE(Block2ActionTypeList)>,
                      bpf::eval_block<GET_TYPETREE(Block3ActionTypeList)>>
      transition_type;
  typedef bpf::blocks<bpf::pdf_block<GET_TYPETREE(Block4ActionTypeList)>> observation_type;
};

}  // namespace test_ar1
