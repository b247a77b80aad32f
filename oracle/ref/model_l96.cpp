// Oracle test infrastructure (never shipped, never timed as the product).
//
// The Lorenz-96 model as LibBi's code generator would render it, written out
// by hand from the generator's templates, so that the reference's OWN host
// updaters run unchanged on it:
//   RK4IntegratorHost         share/src/bi/host/ode/RK4IntegratorHost.hpp:43-100
//   StaticSamplerHost         share/src/bi/host/updater/StaticSamplerHost.hpp:44-65
//   StaticUpdaterHost         share/src/bi/host/updater/StaticUpdaterHost.hpp
//   SparseStaticLogDensityHost share/src/bi/host/updater/SparseStaticLogDensityHost.hpp:48-68
// The model, in LibBi's language (cf. docs/src/users.tex:354-358):
//
//   model L96 {
//     const N = 40;  const F = 8.0;  const SIGMA_ETA = 0.1;  const SIGMA_Y = 1.0
//     dim n(size = N, boundary = 'cyclic')
//     state x[n];  noise eta[n];  obs y[n]
//     sub transition(delta = 0.05) {
//       eta[n] ~ gaussian(0.0, SIGMA_ETA)
//       ode(alg = 'RK4', h = 0.01) { dx[n]/dt = (x[n+1] - x[n-2])*x[n-1] - x[n] + F }
//       x[n] <- x[n] + eta[n]
//     }
//     sub observation { y[n] ~ gaussian(x[n], SIGMA_Y) }
//   }
//
// Rendered pieces and their templates: VarN (share/tt/cpp/var.hpp.tt: ID,
// START, SIZE, NUM_DIMS, TYPE, coord_type), VarCoordN (var_coord.hpp.tt,
// cyclic boundary), ActionCoordN (action_coord.hpp.tt), ActionN
// (action/gaussian.hpp.tt, action/ode_.hpp.tt, action/eval_.hpp.tt with the
// macros fetch_parents, alias_dims, offset_coord, put_output), the action
// type trees (macro/create_action_typetree.hpp.tt) and the Model class's
// size constants (model.hpp.tt:67-78).  Members that nothing on the filter's
// hot path calls (names, input/output flags, dimension objects, the Model
// base class's registries) are not rendered.
//
// Every draw is served from the tape (oracle/shim/boost/random/tape.hpp):
// StaticSamplerHost draws eta particle by particle, component by component,
// so the tape holds the standard normals in that order.  Instantiated with
// real = double (the default of share/src/bi/math/scalar.hpp).
#include "bi/math/loc_temp_vector.hpp"
#include "bi/traits/var_traits.hpp"
#include "bi/traits/action_traits.hpp"
#include "bi/traits/block_traits.hpp"
#include "bi/state/State.hpp"
#include "bi/state/Mask.hpp"
#include "bi/random/Random.hpp"
#include "bi/typelist/macro_typelist.hpp"
#include "bi/typelist/macro_typetree.hpp"
#include "bi/math/scalar.hpp"
#include "bi/math/constant.hpp"
#include "bi/math/function.hpp"
#include "boost/typeof/typeof.hpp"

#include <stdexcept>

namespace l96 {

static const int N = 40;
class ModelL96;

/* ---- variables (var.hpp.tt, var_coord.hpp.tt) ---- */
#define L96_VAR(ID_, START_, TYPE_)                                            \
  class VarCoord##ID_ {                                                        \
   public:                                                                     \
    VarCoord##ID_() { i0 = 0; }                                                \
    VarCoord##ID_(const int i) { i0 = (i + N0) % N0; /* cyclic */ }           \
    void inc() { if (i0 < N0 - 1) ++i0; else i0 = 0; }                         \
    int index() const { return i0; }                                           \
    void setIndex(const int ix) { i0 = ix; }                                   \
    VarCoord##ID_& operator++() { inc(); return *this; }                      \
    int i0;                                                                    \
    static const int N0 = N;                                                   \
  };                                                                           \
  class Var##ID_ {                                                             \
   public:                                                                     \
    typedef VarCoord##ID_ coord_type;                                          \
    static const int ID = ID_;                                                 \
    static const int START = START_;                                           \
    static const int SIZE = N;                                                 \
    static const int NUM_DIMS = 1;                                             \
    static const bi::VarType TYPE = bi::TYPE_;                                 \
  };
L96_VAR(0, 0, D_VAR)  // state x[n]
L96_VAR(1, 0, R_VAR)  // noise eta[n]
L96_VAR(2, 0, O_VAR)  // obs y[n]
#undef L96_VAR

/* ---- action coordinates (action_coord.hpp.tt), one alias n over 0..N-1 ---- */
class ActionCoordN {
 public:
  ActionCoordN() { i0 = OFFSET0; }
  ActionCoordN(const int ix) { setIndex(ix); }
  void inc() { if (i0 < OFFSET0 + LEN0 - 1) ++i0; else i0 = OFFSET0; }
  void dec() { if (i0 > OFFSET0) --i0; else i0 = OFFSET0 + LEN0 - 1; }
  int index() const { return i0; }
  void setIndex(const int ix) { i0 = OFFSET0 + ix; }
  ActionCoordN& operator++() { inc(); return *this; }
  int i0;
  static const int OFFSET0 = 0;
  static const int LEN0 = N;
  static const int N0 = N;
};

/* ---- actions ---- */

/* eta[n] ~ gaussian(0.0, SIGMA_ETA)  (action/gaussian.hpp.tt, sample) */
class Action0 {
 public:
  typedef Var1 target_type;
  typedef ActionCoordN coord_type;
  static const int SIZE = N;
  static const bool IS_MATRIX = false;
  template <class R1, bi::Location L, class CX, class PX, class OX>
  static void samples(R1& rng, bi::State<ModelL96, L>& s, const int p, const int ix, const CX& cox,
                      const PX& pax, OX& x) {
    BI_UNUSED const int n_ = cox.i0;
    const CX& cox_ = cox;
    real mu = BI_REAL(0.0);
    real sigma = BI_REAL(0.1);
    real u = rng.gaussian(mu, sigma);
    x.template fetch<target_type>(s, p, cox_.index()) = u;
  }
};

/* dx[n]/dt = (x[n+1] - x[n-2])*x[n-1] - x[n] + F  (action/ode_.hpp.tt) */
class Action1 {
 public:
  typedef Var0 target_type;
  typedef ActionCoordN coord_type;
  static const int SIZE = N;
  static const bool IS_MATRIX = false;
  template <class T1, bi::Location L, class CX, class PX, class T2>
  static void dfdt(const T1 t, const bi::State<ModelL96, L>& s, const int p, const CX& cox, const PX& pax,
                   T2& dfdt) {
    BI_UNUSED const int n_ = cox.i0;
    /* constants */
    const BOOST_AUTO(F, BI_REAL(8.0));
    /* variables */
    const VarCoord0 cox0(n_ + 1);
    const BOOST_AUTO(x_n_plus_1, pax.template fetch<Var0>(s, p, cox0.index()));
    const VarCoord0 cox1(n_ - 2);
    const BOOST_AUTO(x_n_minus_2, pax.template fetch<Var0>(s, p, cox1.index()));
    const VarCoord0 cox2(n_ - 1);
    const BOOST_AUTO(x_n_minus_1, pax.template fetch<Var0>(s, p, cox2.index()));
    const VarCoord0 cox3(n_);
    const BOOST_AUTO(x_n, pax.template fetch<Var0>(s, p, cox3.index()));
    dfdt = (x_n_plus_1 - x_n_minus_2) * x_n_minus_1 - x_n + F;
  }
};

/* x[n] <- x[n] + eta[n]  (action/eval_.hpp.tt, static simulate) */
struct Action2 {
  typedef Var0 target_type;
  typedef ActionCoordN coord_type;
  static const int SIZE = N;
  static const bool IS_MATRIX = false;
  template <bi::Location L, class CX, class PX, class OX>
  static void simulates(bi::State<ModelL96, L>& s, const int p, const int ix, const CX& cox, const PX& pax,
                        OX& x) {
    BI_UNUSED const int n_ = cox.i0;
    const VarCoord0 cox0(n_);
    const BOOST_AUTO(x_n, pax.template fetch<Var0>(s, p, cox0.index()));
    const VarCoord1 cox1(n_);
    const BOOST_AUTO(eta_n, pax.template fetch<Var1>(s, p, cox1.index()));
    const CX& cox_ = cox;
    x.template fetch<target_type>(s, p, cox_.index()) = x_n + eta_n;
  }
};

/* y[n] ~ gaussian(x[n], SIGMA_Y)  (action/gaussian.hpp.tt, logdensity) */
class Action3 {
 public:
  typedef Var2 target_type;
  typedef ActionCoordN coord_type;
  static const int SIZE = N;
  static const bool IS_MATRIX = false;
  template <bi::Location L, class CX, class PX, class OX, class T1>
  static void logDensities(bi::State<ModelL96, L>& s, const int p, const int ix, const CX& cox, const PX& pax,
                           OX& x, T1& lp) {
    BI_UNUSED const int n_ = cox.i0;
    const VarCoord0 cox0(n_);
    const BOOST_AUTO(x_n, pax.template fetch<Var0>(s, p, cox0.index()));
    const CX& cox_ = cox;
    real mu = x_n;
    real sigma = BI_REAL(1.0);
    real xy = pax.template fetch_alt<target_type>(s, p, cox_.index());
    if (sigma == 0) {
      if (xy == mu) lp = BI_INF; else lp = -BI_INF;
    } else {
      lp += BI_REAL(-0.5) * bi::pow((xy - mu) / sigma, BI_REAL(2.0)) - BI_REAL(BI_HALF_LOG_TWO_PI) -
            bi::log(sigma);
    }
    x.template fetch<target_type>(s, p, cox_.index()) = xy;
  }
};

/* ---- blocks' action type trees (macro/create_action_typetree.hpp.tt) ---- */
BEGIN_TYPETREE(Block1ActionTypeList) LEAF_NODE(1, Action0) END_TYPETREE()
BEGIN_TYPETREE(Block2ActionTypeList) LEAF_NODE(1, Action1) END_TYPETREE()
BEGIN_TYPETREE(Block3ActionTypeList) LEAF_NODE(1, Action2) END_TYPETREE()
BEGIN_TYPETREE(Block4ActionTypeList) LEAF_NODE(1, Action3) END_TYPETREE()
typedef GET_TYPETREE(Block1ActionTypeList) noise_typelist;
typedef GET_TYPETREE(Block2ActionTypeList) ode_typelist;
typedef GET_TYPETREE(Block3ActionTypeList) eval_typelist;
typedef GET_TYPETREE(Block4ActionTypeList) obs_typelist;

/* ---- the model's size constants (model.hpp.tt:67-78) ---- */
class ModelL96 {
 public:
  static const int NR = N, ND = N, NP = 0, NF = 0, NO = N, NDX = 0, NPX = 0, NB = 0;
  static const int CR = 1, CD = 1, CP = 0, CF = 0, CO = 1, CDX = 0, CPX = 0, CB = 0;
};

}  // namespace l96

#include "bi/ode/IntegratorConstants.hpp"
#include "bi/host/ode/RK4IntegratorHost.hpp"
#include "bi/host/updater/StaticSamplerHost.hpp"
#include "bi/host/updater/StaticUpdaterHost.hpp"
#include "bi/host/updater/SparseStaticLogDensityHost.hpp"
#include "bi/traits/resampler_traits.hpp"
#include "bi/resampler/Resampler.hpp"
#include "bi/resampler/SystematicResampler.hpp"
#include "bi/host/resampler/ResamplerHost.hpp"
#include "bi/primitive/vector_primitive.hpp"

#include <chrono>
#include <vector>

namespace {
void ensure_init_l96() {
  static bool init = false;
  if (!init) {
    bi_omp_init(1);
    bi_ode_init();  // the integrator constants the generated client sets at start-up
    init = true;
  }
}
}

extern "C" {

/* One transition of the L96 model for P particles through the reference's
 * own updaters, in the order of the transition block (noise, ode, eval),
 * followed by the observation block's log-density when y != NULL.
 *   x      P x N state, particle-major (x[p*N + i]); updated in place
 *   z      P x N standard normals, in StaticSamplerHost's draw order
 *   y      N observations, or NULL
 *   lp     P log-densities (added to), or NULL when y is NULL
 * Returns 0, or 1 when the tape was not consumed exactly. */
int ref_l96_transition(double* x, int P, const double* z, double t1, double t2, const double* y, double* lp) {
  using namespace l96;
  ensure_init_l96();
  bi::State<ModelL96, bi::ON_HOST> s(P);
  for (int p = 0; p < P; ++p)
    for (int i = 0; i < N; ++i) s.get(bi::D_VAR)(p, i) = x[(size_t)p * N + i];
  static bi::Random rng(0);
  boost::random_tape::set(z, (size_t)P * N);
  bi::StaticSamplerHost<ModelL96, noise_typelist>::samples(rng, s);
  if (boost::random_tape::consumed() != (size_t)P * N) return 1;
  bi_ode_set(BI_REAL(0.01), BI_REAL(1.0e-3), BI_REAL(1.0e-3));
  bi::RK4IntegratorHost<ModelL96, ode_typelist, real>::update(t1, t2, s);
  bi::StaticUpdaterHost<ModelL96, eval_typelist>::update(s);
  if (y) {
    for (int i = 0; i < N; ++i) s.get(bi::OY_VAR)(0, i) = y[i];
    bi::Mask<bi::ON_HOST> mask(3);
    mask.addDenseMask(Var2::ID, N);
    bi::host_vector<real> l(P);
    for (int p = 0; p < P; ++p) l(p) = lp[p];
    bi::SparseStaticLogDensityHost<ModelL96, obs_typelist>::logDensities(s, mask, l);
    for (int p = 0; p < P; ++p) lp[p] = l(p);
  }
  for (int p = 0; p < P; ++p)
    for (int i = 0; i < N; ++i) x[(size_t)p * N + i] = s.get(bi::D_VAR)(p, i);
  return 0;
}

/* The reference's filter loop on this model, timed (the CPU baseline of
 * the benchmark): T steps of Filter<BootstrapPF>::filter
 * (share/src/bi/filter/Filter.hpp:58-70), each BootstrapPF::step
 * (share/src/bi/filter/BootstrapPF.hpp:158-181) run as
 *   resample  Resampler<R>::resample's test s.ess < essRel * P, then
 *             R::precompute and R::ancestorsPermute of the reference's
 *             SystematicResampler, State::gather and set_elements(lws, ll)
 *             (share/src/bi/resampler/Resampler.hpp:167-182)
 *   predict   the transition block: StaticSamplerHost (noise),
 *             RK4IntegratorHost (ode), StaticUpdaterHost (x <- x + eta)
 *   correct   the observation block through SparseStaticLogDensityHost,
 *             then ess_reduce for s.ess, lW and the log-likelihood
 * on `threads` OpenMP threads (the reference's own parallel loops).  Draws
 * come from the tape shim's cycling tables (nrm, uni: n values each), a
 * load per draw, so the reference's generator cost is not counted.
 *   x0  P x N initial states, particle-major;  y  T x N observations
 * Returns the wall-clock seconds of the T steps; *ll the log-likelihood. */
double ref_l96_filter_timed(const double* x0, int P, int T, const double* y, double dt, double ess_rel,
                            int threads, const double* nrm, const double* uni, int n, double* ll) {
  using namespace l96;
  ensure_init_l96();
  bi_omp_init(threads);
  boost::random_tape::set(nullptr, 0);  // this thread draws from the tables too
  boost::random_tape::cycle().nrm = nrm;
  boost::random_tape::cycle().uni = uni;
  boost::random_tape::cycle().n = (std::size_t)n;
  bi::State<ModelL96, bi::ON_HOST> s(P);
  for (int p = 0; p < P; ++p)
    for (int i = 0; i < N; ++i) s.get(bi::D_VAR)(p, i) = x0[(size_t)p * N + i];
  bi::host_vector<real> lws(P);
  bi::set_elements(lws, real(0));
  bi::Mask<bi::ON_HOST> mask(3);
  mask.addDenseMask(Var2::ID, N);
  static bi::Random rng(0);
  bi::SystematicResampler R;
  bi_ode_set(BI_REAL(0.01), BI_REAL(1.0e-3), BI_REAL(1.0e-3));
  double ess = P, logLik = 0.0;
  const auto t0 = std::chrono::steady_clock::now();
  for (int k = 0; k < T; ++k) {
    if (ess < ess_rel * P) {
      bi::ScanResamplerPrecompute<bi::ON_HOST> pre;
      bi::host_vector<int> as(P);
      R.precompute(lws, pre);
      R.ancestorsPermute(rng, lws, as, pre);
      s.gather(as);
      bi::set_elements(lws, real(logLik));
    }
    bi::StaticSamplerHost<ModelL96, noise_typelist>::samples(rng, s);
    bi::RK4IntegratorHost<ModelL96, ode_typelist, real>::update(k * dt, (k + 1) * dt, s);
    bi::StaticUpdaterHost<ModelL96, eval_typelist>::update(s);
    for (int i = 0; i < N; ++i) s.get(bi::OY_VAR)(0, i) = y[(size_t)k * N + i];
    bi::SparseStaticLogDensityHost<ModelL96, obs_typelist>::logDensities(s, mask, lws);
    double lW;
    ess = bi::ess_reduce(lws, &lW);
    logLik = lW;
  }
  const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  boost::random_tape::cycle() = boost::random_tape::Cycle();
  bi_omp_init(1);  // the parity entry points run on one thread
  if (ll) *ll = logLik;
  return secs;
}

}  // extern "C"
