// Oracle test infrastructure (never shipped, never timed as the product).
//
// The phytoplankton-zooplankton model as LibBi's code generator would render
// it, written out by hand from the generator's templates, so that the
// reference's OWN host updaters run unchanged on it:
//   RK43IntegratorHost        share/src/bi/host/ode/RK43IntegratorHost.hpp:48-144
//   StaticSamplerHost         share/src/bi/host/updater/StaticSamplerHost.hpp:44-65
//   SparseStaticLogDensityHost share/src/bi/host/updater/SparseStaticLogDensityHost.hpp:48-68
// The model, in LibBi's language (cf. docs/src/users.tex:40-84):
//
//   model PZ {
//     const c = 0.25;  const e = 0.3;  const m = 0.1;  const q = 0.1
//     state P, Z;  noise alpha;  obs y
//     sub transition(delta = 1.0) {
//       alpha ~ log_normal(log(0.3), 0.2)
//       ode(alg = 'RK4(3)', h = 0.1, atoler = 1.0e-3, rtoler = 1.0e-3) {
//         dP/dt = alpha*P - c*P*Z
//         dZ/dt = e*c*P*Z - m*Z - q*Z*Z
//       }
//     }
//     sub observation { y ~ gaussian(log(P), 0.2) }
//   }
//
// Rendered from share/tt/cpp/var.hpp.tt, var_coord.hpp.tt,
// action_coord.hpp.tt, action/gaussian.hpp.tt (log = 1 for log_normal),
// action/ode_.hpp.tt, macro/create_action_typetree.hpp.tt and the size
// constants of model.hpp.tt:67-78; members that nothing on the filter's hot
// path calls are not rendered.  Draws come from the tape
// (oracle/shim/boost/random/tape.hpp): one standard normal per particle.
// real = double.
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

namespace pz {

class ModelPZ;

/* ---- scalar variables (var.hpp.tt, var_coord.hpp.tt with no dimensions) ---- */
class VarCoordScalar {
 public:
  VarCoordScalar() {}
  VarCoordScalar(const int ix) {}
  void inc() {}
  void dec() {}
  int index() const { return 0; }
  void setIndex(const int ix) {}
  VarCoordScalar& operator++() { inc(); return *this; }
};
#define PZ_VAR(NAME, ID_, START_, TYPE_)   \
  class NAME {                              \
   public:                                  \
    typedef VarCoordScalar coord_type;      \
    static const int ID = ID_;              \
    static const int START = START_;        \
    static const int SIZE = 1;              \
    static const int NUM_DIMS = 0;          \
    static const bi::VarType TYPE = bi::TYPE_; \
  };
PZ_VAR(Var0, 0, 0, D_VAR)  // state P
PZ_VAR(Var1, 1, 1, D_VAR)  // state Z
PZ_VAR(Var2, 2, 0, R_VAR)  // noise alpha
PZ_VAR(Var3, 3, 0, O_VAR)  // obs y
#undef PZ_VAR

/* ---- action coordinates (action_coord.hpp.tt, no aliases) ---- */
class ActionCoordScalar {
 public:
  ActionCoordScalar() {}
  ActionCoordScalar(const int ix) {}
  void inc() {}
  void dec() {}
  int index() const { return 0; }
  void setIndex(const int ix) {}
  ActionCoordScalar& operator++() { inc(); return *this; }
};

/* alpha ~ log_normal(log(0.3), 0.2)  (action/gaussian.hpp.tt, log = 1) */
class Action0 {
 public:
  typedef Var2 target_type;
  typedef ActionCoordScalar coord_type;
  static const int SIZE = 1;
  static const bool IS_MATRIX = false;
  template <class R1, bi::Location L, class CX, class PX, class OX>
  static void samples(R1& rng, bi::State<ModelPZ, L>& s, const int p, const int ix, const CX& cox,
                      const PX& pax, OX& x) {
    const CX& cox_ = cox;
    real mu = bi::log(BI_REAL(0.3));
    real sigma = BI_REAL(0.2);
    real u = bi::exp(rng.gaussian(mu, sigma));
    x.template fetch<target_type>(s, p, cox_.index()) = u;
  }
};

/* dP/dt = alpha*P - c*P*Z  (action/ode_.hpp.tt) */
class Action1 {
 public:
  typedef Var0 target_type;
  typedef ActionCoordScalar coord_type;
  static const int SIZE = 1;
  static const bool IS_MATRIX = false;
  template <class T1, bi::Location L, class CX, class PX, class T2>
  static void dfdt(const T1 t, const bi::State<ModelPZ, L>& s, const int p, const CX& cox, const PX& pax,
                   T2& dfdt) {
    /* constants */
    const BOOST_AUTO(c, BI_REAL(0.25));
    /* variables */
    const BOOST_AUTO(alpha, pax.template fetch<Var2>(s, p, 0));
    const BOOST_AUTO(P, pax.template fetch<Var0>(s, p, 0));
    const BOOST_AUTO(Z, pax.template fetch<Var1>(s, p, 0));
    dfdt = alpha * P - c * P * Z;
  }
};

/* dZ/dt = e*c*P*Z - m*Z - q*Z*Z  (action/ode_.hpp.tt) */
class Action2 {
 public:
  typedef Var1 target_type;
  typedef ActionCoordScalar coord_type;
  static const int SIZE = 1;
  static const bool IS_MATRIX = false;
  template <class T1, bi::Location L, class CX, class PX, class T2>
  static void dfdt(const T1 t, const bi::State<ModelPZ, L>& s, const int p, const CX& cox, const PX& pax,
                   T2& dfdt) {
    /* constants */
    const BOOST_AUTO(c, BI_REAL(0.25));
    const BOOST_AUTO(e, BI_REAL(0.3));
    const BOOST_AUTO(m, BI_REAL(0.1));
    const BOOST_AUTO(q, BI_REAL(0.1));
    /* variables */
    const BOOST_AUTO(P, pax.template fetch<Var0>(s, p, 0));
    const BOOST_AUTO(Z, pax.template fetch<Var1>(s, p, 0));
    dfdt = e * c * P * Z - m * Z - q * Z * Z;
  }
};

/* y ~ gaussian(log(P), 0.2)  (action/gaussian.hpp.tt, logdensity) */
class Action3 {
 public:
  typedef Var3 target_type;
  typedef ActionCoordScalar coord_type;
  static const int SIZE = 1;
  static const bool IS_MATRIX = false;
  template <bi::Location L, class CX, class PX, class OX, class T1>
  static void logDensities(bi::State<ModelPZ, L>& s, const int p, const int ix, const CX& cox, const PX& pax,
                           OX& x, T1& lp) {
    const BOOST_AUTO(P, pax.template fetch<Var0>(s, p, 0));
    const CX& cox_ = cox;
    real mu = bi::log(P);
    real sigma = BI_REAL(0.2);
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

BEGIN_TYPETREE(Block1ActionTypeList) LEAF_NODE(1, Action0) END_TYPETREE()
BEGIN_TYPETREE(Block2ActionTypeList)
  BEGIN_NODE(1) LEAF_NODE(1, Action1) JOIN_NODE LEAF_NODE(1, Action2) END_NODE
END_TYPETREE()
BEGIN_TYPETREE(Block3ActionTypeList) LEAF_NODE(1, Action3) END_TYPETREE()
typedef GET_TYPETREE(Block1ActionTypeList) noise_typelist;
typedef GET_TYPETREE(Block2ActionTypeList) ode_typelist;
typedef GET_TYPETREE(Block3ActionTypeList) obs_typelist;

class ModelPZ {
 public:
  static const int NR = 1, ND = 2, NP = 0, NF = 0, NO = 1, NDX = 0, NPX = 0, NB = 0;
  static const int CR = 1, CD = 2, CP = 0, CF = 0, CO = 1, CDX = 0, CPX = 0, CB = 0;
};

}  // namespace pz

#include "bi/ode/IntegratorConstants.hpp"
#include "bi/host/ode/RK43IntegratorHost.hpp"
#include "bi/host/updater/StaticSamplerHost.hpp"
#include "bi/host/updater/SparseStaticLogDensityHost.hpp"
#include "bi/traits/resampler_traits.hpp"
#include "bi/resampler/Resampler.hpp"
#include "bi/resampler/SystematicResampler.hpp"
#include "bi/host/resampler/ResamplerHost.hpp"
#include "bi/primitive/vector_primitive.hpp"

#include <chrono>

namespace {
void ensure_init_pz() {
  static bool init = false;
  if (!init) {
    bi_omp_init(1);
    bi_ode_init();  // the integrator constants the generated client sets at start-up
    init = true;
  }
}
}

extern "C" {

/* One PZ transition for P particles through the reference's own updaters
 * (noise block, then the RK4(3) ode block), then the observation block's
 * log-density when y != NULL.
 *   x   P x 2 state (P, Z), particle-major; updated in place
 *   z   P standard normals (the log-normal alpha draws, in particle order)
 *   y   1 observation, or NULL;  lp  P log-densities (added to)
 * Returns 0, or 1 when the tape was not consumed exactly. */
int ref_pz_transition(double* x, int P, const double* z, double t1, double t2, const double* y, double* lp) {
  using namespace pz;
  ensure_init_pz();
  bi::State<ModelPZ, bi::ON_HOST> s(P);
  for (int p = 0; p < P; ++p)
    for (int i = 0; i < 2; ++i) s.get(bi::D_VAR)(p, i) = x[(size_t)p * 2 + i];
  static bi::Random rng(0);
  boost::random_tape::set(z, (size_t)P);
  bi::StaticSamplerHost<ModelPZ, noise_typelist>::samples(rng, s);
  if (boost::random_tape::consumed() != (size_t)P) return 1;
  bi_ode_set(BI_REAL(0.1), BI_REAL(1.0e-3), BI_REAL(1.0e-3));
  bi::RK43IntegratorHost<ModelPZ, ode_typelist, real>::update(t1, t2, s);
  if (y) {
    s.get(bi::OY_VAR)(0, 0) = y[0];
    bi::Mask<bi::ON_HOST> mask(4);
    mask.addDenseMask(Var3::ID, 1);
    bi::host_vector<real> l(P);
    for (int p = 0; p < P; ++p) l(p) = lp[p];
    bi::SparseStaticLogDensityHost<ModelPZ, obs_typelist>::logDensities(s, mask, l);
    for (int p = 0; p < P; ++p) lp[p] = l(p);
  }
  for (int p = 0; p < P; ++p)
    for (int i = 0; i < 2; ++i) x[(size_t)p * 2 + i] = s.get(bi::D_VAR)(p, i);
  return 0;
}

/* The reference's filter loop on this model, timed (the CPU baseline of the
 * plankton configuration): T steps of Filter<BootstrapPF>::filter
 * (share/src/bi/filter/Filter.hpp:58-70), each BootstrapPF::step
 * (share/src/bi/filter/BootstrapPF.hpp:158-181) run as Resampler<R>::resample's
 * test and the reference's SystematicResampler (precompute,
 * ancestorsPermute, State::gather, set_elements(lws, ll);
 * share/src/bi/resampler/Resampler.hpp:167-182), the transition block
 * (StaticSamplerHost for the log-normal growth rate, RK43IntegratorHost for
 * the ode) and the observation block through SparseStaticLogDensityHost,
 * then ess_reduce; on `threads` OpenMP threads.  Draws come from the tape
 * shim's cycling tables (a load each: the generator's cost is not counted).
 *   x0  P x 2 initial states (P, Z), particle-major;  y  T observations
 * Returns the wall-clock seconds of the T steps; *ll the log-likelihood. */
double ref_pz_filter_timed(const double* x0, int P, int T, const double* y, double dt, double ess_rel, int threads,
                           const double* nrm, const double* uni, int n, double* ll) {
  using namespace pz;
  ensure_init_pz();
  bi_omp_init(threads);
  boost::random_tape::set(nullptr, 0);  // this thread draws from the tables too
  boost::random_tape::cycle().nrm = nrm;
  boost::random_tape::cycle().uni = uni;
  boost::random_tape::cycle().n = (std::size_t)n;
  bi::State<ModelPZ, bi::ON_HOST> s(P);
  for (int p = 0; p < P; ++p)
    for (int i = 0; i < 2; ++i) s.get(bi::D_VAR)(p, i) = x0[(size_t)p * 2 + i];
  bi::host_vector<real> lws(P);
  bi::set_elements(lws, real(0));
  bi::Mask<bi::ON_HOST> mask(4);
  mask.addDenseMask(Var3::ID, 1);
  static bi::Random rng(0);
  bi::SystematicResampler R;
  bi_ode_set(BI_REAL(0.1), BI_REAL(1.0e-3), BI_REAL(1.0e-3));
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
    bi::StaticSamplerHost<ModelPZ, noise_typelist>::samples(rng, s);
    bi::RK43IntegratorHost<ModelPZ, ode_typelist, real>::update(k * dt, (k + 1) * dt, s);
    s.get(bi::OY_VAR)(0, 0) = y[k];
    bi::SparseStaticLogDensityHost<ModelPZ, obs_typelist>::logDensities(s, mask, lws);
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
