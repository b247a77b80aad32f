/* C++ host interface over the C ABI (libbi_b200.h), header-only.
 *
 * It mirrors the classes a generated LibBi filter client drives
 * (share/tt/cpp/client/filter_cpu.cpp.tt:105-192) with the same names and
 * call shapes:
 *   bi_b200::Filter<F>::filter(rng, first, last, s)      bi::Filter<F>::filter
 *       (share/src/bi/filter/Filter.hpp:58-70)
 *   bi_b200::BootstrapPF<B, O, R>: init, correct, step, term, samplePath
 *       (share/src/bi/filter/BootstrapPF.hpp:25-154)
 *   bi_b200::Resampler<R> with SystematicResampler, MultinomialResampler,
 *       MetropolisResampler (share/src/bi/resampler/Resampler.hpp:34-182)
 *   bi_b200::Schedule / ScheduleElement / ScheduleIterator and Observer
 *       (share/src/bi/state/Schedule.hpp:107-315,
 *        share/src/bi/simulator/Observer.hpp:97-126)
 *   bi_b200::BootstrapPFState<B> (share/src/bi/state/BootstrapPFState.hpp)
 *   bi_b200::ParticleFilterDegeneratedException
 *       (share/src/bi/misc/exception.hpp:47)
 * The models are the two built into the library (ModelL96, ModelPZ) with
 * the constants of their .bi files, or a model class in the shape LibBi's
 * code generator emits, compiled by the caller against bpf_model.cuh and
 * wrapped as DeviceModel<Model>.  Every call goes through the C ABI; the
 * particles stay in device memory.  Errors throw: a degenerate filter throws
 * ParticleFilterDegeneratedException as the reference does, any other
 * status BpfError. */
#ifndef LIBBI_B200_HPP
#define LIBBI_B200_HPP

#include "libbi_b200.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

namespace bi_b200 {

/* ---- errors ------------------------------------------------------------- */
struct ParticleFilterDegeneratedException {};

class BpfError : public std::runtime_error {
 public:
  BpfError(int status, const std::string& what)
      : std::runtime_error(what + ": " + bpf_status_string(status)), status_(status) {}
  int status() const { return status_; }

 private:
  int status_;
};

inline void check(int rc, const char* what) {
  if (rc == BPF_E_DEGENERATE) throw ParticleFilterDegeneratedException();
  if (rc != BPF_OK) throw BpfError(rc, what);
}

/* ---- models (B) ----------------------------------------------------------- */
/* Lorenz '96: transition(delta) { eta[i] ~ N(0, sigma_eta); ode RK4(h)
 * { dx[i]/dt = (x[i+1] - x[i-2]) x[i-1] - x[i] + F }; x += eta },
 * observation { y[i] ~ N(x[i], sigma_y) }, initial x[i] ~ N(x0_mean, x0_std)
 * (x0_mean defaults to F). */
struct ModelL96 {
  typedef float real;
  int dim = 40;
  double F = 8.0, sigma_eta = 0.1, sigma_y = 1.0, h = 0.01;
  double x0_mean = NAN, x0_std = 0.01;
  bool fp64 = false;
  bpf_model_desc desc() const {
    bpf_model_desc d{};
    d.kind = BPF_MODEL_L96;
    d.dim = dim;
    d.precision = fp64 ? BPF_F64 : BPF_F32;
    d.integrator = BPF_ODE_RK4;
    d.h = h;
    d.theta[0] = F;
    d.theta[1] = sigma_eta;
    d.theta[2] = sigma_y;
    d.theta[3] = std::isnan(x0_mean) ? F : x0_mean;
    d.theta[4] = x0_std;
    return d;
  }
  int nobs() const { return dim; }
  size_t esz() const { return fp64 ? 8 : 4; }
};

/* Phytoplankton-zooplankton (FP64, adaptive RK4(3)): transition(delta)
 * { alpha ~ log_normal(mu, sigma); ode { dP/dt = alpha P - c P Z;
 * dZ/dt = e c P Z - m Z - q Z^2 } }, observation { y ~ N(log P, sigma_y) },
 * initial { P ~ log_normal(p0_mu, p0_sigma), Z ~ log_normal(z0_mu, z0_sigma) }. */
struct ModelPZ {
  typedef double real;
  double c = 0.25, e = 0.3, m = 0.1, q = 0.1;
  double mu = -1.2039728043259361, sigma = 0.2, sigma_y = 0.2;  // mu = log 0.3
  double p0_mu = 0.69314718055994531, p0_sigma = 0.2;           // log 2
  double z0_mu = 0.69314718055994531, z0_sigma = 0.2;
  double h = 0.1, atoler = 1e-3, rtoler = 1e-3;
  bpf_model_desc desc() const {
    bpf_model_desc d{};
    d.kind = BPF_MODEL_PZ;
    d.dim = 2;
    d.precision = BPF_F64;
    d.integrator = BPF_ODE_RK43;
    d.h = h;
    d.atoler = atoler;
    d.rtoler = rtoler;
    const double th[] = {c, e, m, q, mu, sigma, sigma_y, p0_mu, p0_sigma, z0_mu, z0_sigma};
    for (int i = 0; i < 11; ++i) d.theta[i] = th[i];
    return d;
  }
  int nobs() const { return 1; }
  size_t esz() const { return 8; }
};

/* A model B is either one of the two built into the library (desc() gives
 * its bpf_model_desc) or a model class compiled by the caller against
 * bpf_model.cuh, wrapped as bi_b200::DeviceModel<Model> (ops() gives its
 * bpf_model_ops table, params its parameter values). */
template <class M>
auto create_handle(const M& m, const bpf_config& c, bpf_handle** h, int) -> decltype(m.desc(), int()) {
  bpf_model_desc d = m.desc();
  return bpf_create(&d, &c, h);
}
template <class M>
auto create_handle(const M& m, const bpf_config& c, bpf_handle** h, long) -> decltype(m.ops(), int()) {
  bpf_model_ops o = m.ops();
  return bpf_create_model(&o, m.params.empty() ? nullptr : m.params.data(), &c, h);
}
template <class M>
auto model_dim(const M& m, int) -> decltype(m.desc(), int()) { return m.desc().dim; }
template <class M>
auto model_dim(const M& m, long) -> decltype(m.ops(), int()) { return m.ops().dim; }

/* ---- random numbers ----------------------------------------------------- */
/* The reference's Random holds generator state; here every draw is a
 * counter-based Philox4x32-10 function of (seed, particle, step, stream), so
 * the seed is all there is. */
struct Random {
  uint64_t seed;
  explicit Random(uint64_t s = 0) : seed(s) {}
};

/* ---- resamplers (R) ------------------------------------------------------- */
struct SystematicResampler { static constexpr int kind = BPF_RESAMPLER_SYSTEMATIC; };
struct MultinomialResampler { static constexpr int kind = BPF_RESAMPLER_MULTINOMIAL; };
struct MetropolisResampler { static constexpr int kind = BPF_RESAMPLER_METROPOLIS; };

/* Resampler<R>: the filter's settings (essRel, Metropolis steps B) and the
 * stand-alone primitives on device vectors of log-weights. */
template <class R>
class Resampler : public R {
 public:
  explicit Resampler(double essRel = 0.5, int B = 0) : essRel_(essRel), B_(B) {}
  ~Resampler() {
    if (h_) bpf_resampler_destroy(h_);
  }
  Resampler(const Resampler&) = delete;
  Resampler& operator=(const Resampler&) = delete;
  double getEssRel() const { return essRel_; }
  int getB() const { return B_; }
  /* Resampler::reduce: returns the ESS, *lW = log mean exp(lws) */
  double reduce(const double* lws_device, int n, double* lW) {
    ensure(n);
    double ess = 0.0;
    check(bpf_ess_reduce(h_, lws_device, n, lW, &ess), "Resampler::reduce");
    return ess;
  }
  /* ancestorsPermute (permute = 1) or sorted ancestors (0) into as_device;
   * uniforms_device: the draws, or null for the library's own */
  void ancestors(const double* lws_device, int n, const double* uniforms_device, int permute, int* as_device,
                 int* Os_device = nullptr) {
    ensure(n);
    check(bpf_resampler_ancestors(h_, lws_device, n, uniforms_device, permute, as_device, Os_device),
          "Resampler::ancestors");
  }

 private:
  void ensure(int n) {
    if (h_ && n <= cap_) return;
    if (h_) bpf_resampler_destroy(h_);
    h_ = nullptr;
    check(bpf_resampler_create(R::kind, n, B_, nullptr, &h_), "bpf_resampler_create");
    cap_ = n;
  }
  double essRel_;
  int B_;
  bpf_resampler* h_ = nullptr;
  int cap_ = 0;
};

/* ---- schedule and observations (O) --------------------------------------- */
/* Observations in the sparse layout of a LibBi observation file: time,
 * component index and value per entry, grouped by time (Observer::update,
 * getMask). */
class Observer {
 public:
  Observer() = default;
  Observer(const std::vector<double>& times, const std::vector<int>& coords, const std::vector<double>& values) {
    if (times.size() != coords.size() || times.size() != values.size())
      throw std::invalid_argument("times, coords and values must have equal length");
    std::map<double, std::map<int, double>> g;
    for (size_t i = 0; i < times.size(); ++i) {
      if (coords[i] < 0) throw std::invalid_argument("component indices must be non-negative");
      auto& row = g[times[i]];
      if (row.count(coords[i])) throw std::invalid_argument("component observed twice at one time");
      row[coords[i]] = values[i];
    }
    for (const auto& kv : g) {
      times_.push_back(kv.first);
      std::vector<int> c;
      std::vector<double> v;
      for (const auto& cv : kv.second) {
        c.push_back(cv.first);
        v.push_back(cv.second);
      }
      coords_.push_back(c);
      values_.push_back(v);
    }
  }
  int size() const { return (int)times_.size(); }
  double time(int k) const { return times_[k]; }
  const std::vector<int>& mask(int k) const { return coords_[k]; }
  const std::vector<double>& values(int k) const { return values_[k]; }

 private:
  std::vector<double> times_;
  std::vector<std::vector<int>> coords_;
  std::vector<std::vector<double>> values_;
};

struct ScheduleElement {
  double time;
  bool observed;
  int indexObs;  // observation index when observed, else -1
  bool output;
  double getTime() const { return time; }
  bool hasObs() const { return observed; }
};
typedef std::vector<ScheduleElement>::const_iterator ScheduleIterator;

/* The ordered grid of a run: t0, the multiples of delta up to the last
 * time, observation and output times (which must lie on that grid: the
 * transition draws its noise once per delta). */
class Schedule {
 public:
  Schedule(double t0, double delta, const Observer* obs = nullptr, const std::vector<double>& outputs = {},
           double tol = 1e-9) {
    if (!(delta > 0.0)) throw std::invalid_argument("delta must be positive");
    double last = t0;
    if (obs)
      for (int k = 0; k < obs->size(); ++k) last = std::max(last, obs->time(k));
    for (double t : outputs) last = std::max(last, t);
    long nsteps = std::lround((last - t0) / delta);
    if (t0 + nsteps * delta < last - tol * std::max(1.0, std::fabs(last))) ++nsteps;
    elements_.resize((size_t)nsteps + 1);
    for (long k = 0; k <= nsteps; ++k) elements_[k] = ScheduleElement{t0 + delta * k, false, -1, false};
    auto on_grid = [&](double t, long* k) {
      *k = std::lround((t - t0) / delta);
      return *k >= 0 && *k <= nsteps && std::fabs(elements_[*k].time - t) <= tol * std::max(1.0, std::fabs(t));
    };
    if (obs)
      for (int i = 0; i < obs->size(); ++i) {
        long k = 0;
        if (!on_grid(obs->time(i), &k) || k == 0)
          throw std::invalid_argument("observation time is not a multiple of delta after t0");
        elements_[k].observed = true;
        elements_[k].indexObs = i;
      }
    for (double t : outputs) {
      long k = 0;
      if (!on_grid(t, &k)) throw std::invalid_argument("output time is not on the schedule's grid");
      elements_[k].output = true;
    }
  }
  ScheduleIterator begin() const { return elements_.begin(); }
  ScheduleIterator end() const { return elements_.end(); }
  int size() const { return (int)elements_.size(); }

 private:
  std::vector<ScheduleElement> elements_;
};

/* ---- state (S) ------------------------------------------------------------ */
/* BootstrapPFState: N particles of model B in device memory (the handle is
 * made when a filter binds its resampler and seed at init). */
template <class B>
class BootstrapPFState {
 public:
  BootstrapPFState(const B& m, int N, void* stream = nullptr) : m_(m), N_(N), stream_(stream) {}
  ~BootstrapPFState() {
    if (h_) bpf_destroy(h_);
  }
  BootstrapPFState(const BootstrapPFState&) = delete;
  BootstrapPFState& operator=(const BootstrapPFState&) = delete;
  int size() const { return N_; }
  bpf_handle* handle() const { return h_; }
  /* device structure-of-arrays state: component j of particle p at x[j*ld + p] */
  void* x() const { return ptrs().x; }
  double* logWeights() const { return ptrs().lw; }
  int* ancestors() const { return ptrs().as; }
  int ld() const { return ptrs().ld; }

  double logLikelihood = 0.0;
  double ess = 0.0;
  std::vector<double> logIncrements;

  /* the handle for these filter settings; kept when they do not change, so
   * that a path cache reserved before Filter::filter survives its init */
  void bind(int kind, double essRel, int msteps, uint64_t seed) {
    if (h_ && kind == kind_ && essRel == essRel_ && msteps == msteps_ && seed == seed_) return;
    if (h_) bpf_destroy(h_);
    h_ = nullptr;
    kind_ = kind;
    essRel_ = essRel;
    msteps_ = msteps;
    seed_ = seed;
    bpf_config c{};
    c.nparticles = N_;
    c.resampler = kind;
    c.metropolis_steps = msteps;
    c.ess_rel = essRel;
    c.seed = seed;
    c.stream = stream_;
    check(create_handle(m_, c, &h_, 0), "bpf_create");
  }

 private:
  struct Ptrs {
    void* x;
    double* lw;
    int* as;
    int ld;
  };
  Ptrs ptrs() const {
    Ptrs p{nullptr, nullptr, nullptr, 0};
    if (h_) check(bpf_state_ptrs(h_, &p.x, &p.lw, &p.as, &p.ld), "bpf_state_ptrs");
    return p;
  }
  B m_;
  int N_;
  void* stream_;
  bpf_handle* h_ = nullptr;
  int kind_ = -1, msteps_ = 0;
  double essRel_ = 0.0;
  uint64_t seed_ = 0;
};

/* ---- the filter ----------------------------------------------------------- */
template <class B, class O, class R>
class BootstrapPF {
 public:
  BootstrapPF(B& m, O& obs, R& resam) : m_(m), obs_(obs), resam_(resam) {}

  /* Simulator::init: initial draws, log-weights zero (and a reserved path
   * record restarted from the initial state) */
  template <class S1>
  void init(Random& rng, S1& s) {
    s.bind(R::kind, resam_.getEssRel(), resam_.getB(), rng.seed);
    check(bpf_init(s.handle()), "bpf_init");
    s.logLikelihood = 0.0;
    s.logIncrements.clear();
  }

  /* correct at the first element: an observation at t0 is not supported
   * (the schedule puts none there); nothing to do */
  template <class S1>
  void correct(Random&, const ScheduleElement now, S1&) {
    if (now.hasObs()) throw std::invalid_argument("an observation at the schedule's first time");
  }

  /* BootstrapPF::step: from *iter to the next observed element (or last):
   * resample if due, predict through every delta, correct at the
   * observation */
  template <class S1>
  void step(Random&, ScheduleIterator& iter, const ScheduleIterator last, S1& s) {
    do {
      const ScheduleElement prev = *iter;
      ++iter;
      const ScheduleElement& el = *iter;
      bpf_step_out out{};
      if (el.hasObs()) {
        const std::vector<int>& idx = obs_.mask(el.indexObs);
        const std::vector<double>& v = obs_.values(el.indexObs);
        std::vector<unsigned char> y(v.size() * m_.esz());
        for (size_t j = 0; j < v.size(); ++j) {
          if (m_.esz() == 4) reinterpret_cast<float*>(y.data())[j] = (float)v[j];
          else reinterpret_cast<double*>(y.data())[j] = v[j];
        }
        check(bpf_step_sparse(s.handle(), prev.time, el.time, y.data(), idx.data(), (int)idx.size(), &out),
              "BootstrapPF::step");
        s.logIncrements.push_back(out.log_increment);
        s.logLikelihood = out.log_likelihood;
        s.ess = out.ess;
      } else {
        check(bpf_step_sparse(s.handle(), prev.time, el.time, nullptr, nullptr, 0, &out), "BootstrapPF::step");
      }
    } while (iter + 1 != last && !iter->hasObs());
  }

  /* BootstrapPF::term: the log-likelihood estimate stays as accumulated */
  template <class S1>
  void term(S1&) {}

  /* BootstrapPF::samplePath with a path cache of max_steps steps reserved
   * before the run (recordPath); path: len x dim, oldest first */
  template <class S1>
  int samplePath(Random&, S1& s, std::vector<typename B::real>& path, int* particle = nullptr) {
    const int dim = model_dim(m_, 0);
    path.assign((size_t)(cap_ + 1) * dim, (typename B::real)0);
    int len = 0, p = 0;
    check(bpf_sample_path(s.handle(), nullptr, path.data(), &p, &len), "BootstrapPF::samplePath");
    path.resize((size_t)len * dim);
    if (particle) *particle = p;
    return len;
  }
  template <class S1>
  void recordPath(S1& s, int max_steps) {
    check(bpf_path_cache(s.handle(), max_steps), "bpf_path_cache");
    cap_ = max_steps;
  }

 private:
  B& m_;
  O& obs_;
  R& resam_;
  int cap_ = 0;
};

/* Filter<F>::filter: init, then step from element to element, then term */
template <class F>
class Filter : public F {
 public:
  using F::F;
  template <class S1>
  void filter(Random& rng, const ScheduleIterator first, const ScheduleIterator last, S1& s) {
    ScheduleIterator iter = first;
    this->init(rng, s);
    this->correct(rng, *iter, s);
    while (iter + 1 != last) this->step(rng, iter, last, s);
    this->term(s);
  }
};

}  // namespace bi_b200

#endif
