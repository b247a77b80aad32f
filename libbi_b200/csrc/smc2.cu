// SMC^2: sequential Monte Carlo over parameters, each parameter particle
// carrying its own particle filter (LibBi's MarginalSIR,
// share/src/bi/sampler/MarginalSIR.hpp:283-480).
//
// The P parameter particles' filters are one batch (batch.cu).  At each
// observation every filter takes one step (bpf_batch_step_device) and each
// parameter particle's log-weight grows by its filter's log-likelihood
// increment (MarginalSIR::step); the weights' ESS and the marginal
// likelihood increment follow (interact), and when the ESS falls below
// ess_rel * P the parameter particles are resampled (systematic) and each
// makes `moves` particle-marginal Metropolis-Hastings moves: a random-walk
// proposal, a fresh filter over the observations so far for all P proposals
// at once (a second batch), and MarginalMH's accept/reject (move,
// MarginalSIR.hpp:420-470).
//
// A filter's state at time t is a deterministic function of its parameters,
// its seed and the observations up to t (counter-based draws), so after a
// resample-move round the main batch simply replays the observations so far
// with the surviving (parameters, seed) pairs instead of copying particle
// states between filters; the replay reproduces each filter's
// log-likelihood bit for bit.
//
// Random numbers (tag BPF_RNG_PMMH, seed cfg.seed): parameter particle i at
// round r draws its random-walk normals as PMMH chain i at run r, its
// acceptance uniform from block 64; the systematic offset of the parameter
// resample after observation k uses chain index P, run 100000 + k; the
// initial parameters come from the priors as in PMMH.  Filter seeds:
// seed + 1 + r*P + i for the r-th filter run of slot i.
#include "internal.cuh"
#include "sampler_common.cuh"

#include <cmath>
#include <cstring>
#include <new>
#include <vector>

namespace {

using bpf::sampler::log_prior;
using bpf::sampler::normal_draw;
using bpf::sampler::uniform_draw;

struct Smc2 {
  bpf_model_desc model;
  bpf_smc2_config cfg;
  int P = 0, T = 0;
  double t0 = 0.0, dt = 0.0;
  size_t step_bytes = 0;     // one step's observations for all P filters
  void* y_dev = nullptr;     // T x P x nobs
  std::vector<unsigned char> y_host;
  bpf_batch* main = nullptr;
  bpf_batch* move = nullptr;
  std::vector<double> theta;  // P x BPF_MAX_THETA
  std::vector<uint64_t> seeds;
  std::vector<double> ll, lp, lw;
  int run = 0;                // filter runs so far (seed counter)

  ~Smc2() {
    if (main) bpf_batch_destroy(main);
    if (move) bpf_batch_destroy(move);
    if (y_dev) cudaFree(y_dev);
  }
};

double prior_of(const Smc2& s, const double* th) {
  double l = 0.0;
  for (int j = 0; j < s.cfg.nparams; ++j) l += log_prior(s.cfg.params[j], th[s.cfg.params[j].index]);
  return l;
}

// run batch b from t0 through observation k (1-based) with the given
// parameters and seeds; log-likelihoods (-inf when degenerate) into ll
int replay(Smc2& s, bpf_batch* b, const std::vector<double>& theta, const std::vector<uint64_t>& seeds, int k,
           std::vector<double>& ll) {
  int rc = bpf_batch_set_theta(b, theta.data());
  if (!rc) rc = bpf_batch_set_seeds(b, seeds.data());
  if (!rc) rc = bpf_batch_init(b);
  for (int j = 1; !rc && j <= k; ++j)
    rc = bpf_batch_step_device(b, s.t0 + (j - 1) * s.dt, s.t0 + j * s.dt,
                               (const char*)s.y_dev + (size_t)(j - 1) * s.step_bytes);
  if (rc) return rc;
  std::vector<int> status((size_t)s.P);
  rc = bpf_batch_stats(b, ll.data(), nullptr, status.data());
  if (rc != BPF_OK && rc != BPF_E_DEGENERATE) return rc;
  for (int i = 0; i < s.P; ++i)
    if (status[i] != BPF_OK) ll[i] = -INFINITY;
  return BPF_OK;
}

double log_sum_exp(const std::vector<double>& v) {
  double m = -INFINITY;
  for (double x : v) m = std::fmax(m, x);
  if (!std::isfinite(m)) return m;
  double s = 0.0;
  for (double x : v) s += std::exp(x - m);
  return m + std::log(s);
}

}  // namespace

extern "C" int bpf_smc2_run(const bpf_model_desc* model, const bpf_smc2_config* cfg, int T, double t0, double dt,
                            const void* y, void* stream, double* theta_out, double* log_weights_out,
                            double* log_evidence_increments, int* resample_steps, double* acceptance) {
  if (!model || !cfg || T <= 0 || !(dt > 0.0) || !y || cfg->ntheta <= 0 || cfg->nparams <= 0 ||
      cfg->nparams > BPF_MAX_THETA || cfg->nparticles <= 0 || cfg->nparticles > BPF_BATCH_MAX_PARTICLES ||
      cfg->moves < 0 || !(cfg->theta_ess_rel >= 0.0 && cfg->theta_ess_rel <= 1.0))
    return BPF_E_INVALID;
  for (int j = 0; j < cfg->nparams; ++j) {
    const bpf_pmmh_param& q = cfg->params[j];
    if (q.index < 0 || q.index >= BPF_MAX_THETA || !(q.step >= 0.0) || q.prior < BPF_PRIOR_UNIFORM ||
        q.prior > BPF_PRIOR_GAUSSIAN || (q.prior == BPF_PRIOR_UNIFORM ? !(q.b > q.a) : !(q.b > 0.0)))
      return BPF_E_INVALID;
  }
  Smc2* sp = new (std::nothrow) Smc2();
  if (!sp) return BPF_E_NOMEM;
  Smc2& s = *sp;
  s.model = *model;
  s.cfg = *cfg;
  s.P = cfg->ntheta;
  s.T = T;
  s.t0 = t0;
  s.dt = dt;
  const int P = s.P;
  const size_t nobs = model->kind == BPF_MODEL_L96 ? (size_t)model->dim : 1;
  const size_t esz = model->precision == BPF_F64 ? 8 : 4;
  s.step_bytes = (size_t)P * nobs * esz;
  s.y_host.resize((size_t)T * s.step_bytes);
  for (int k = 0; k < T; ++k)
    for (int i = 0; i < P; ++i)
      std::memcpy(&s.y_host[(size_t)k * s.step_bytes + (size_t)i * nobs * esz],
                  (const unsigned char*)y + (size_t)k * nobs * esz, nobs * esz);
  int rc = cudaMalloc(&s.y_dev, s.y_host.size()) == cudaSuccess ? BPF_OK : BPF_E_NOMEM;
  if (!rc && cudaMemcpy(s.y_dev, s.y_host.data(), s.y_host.size(), cudaMemcpyHostToDevice) != cudaSuccess)
    rc = BPF_E_CUDA;
  // initial parameters from the priors (MarginalSIR::init)
  s.theta.assign((size_t)P * BPF_MAX_THETA, 0.0);
  s.seeds.assign((size_t)P, 0);
  for (int i = 0; i < P; ++i) {
    double* th = &s.theta[(size_t)i * BPF_MAX_THETA];
    for (int m = 0; m < BPF_MAX_THETA; ++m) th[m] = model->theta[m];
    for (int j = 0; j < cfg->nparams; ++j) {
      const bpf_pmmh_param& q = cfg->params[j];
      double v;
      if (q.prior == BPF_PRIOR_UNIFORM) {
        v = q.a + (q.b - q.a) * uniform_draw(cfg->seed, i, 0, 32 + j);
      } else {
        const double z = normal_draw(cfg->seed, i, 0, 64 + 2 * j);
        v = q.prior == BPF_PRIOR_LOG_NORMAL ? std::exp(q.a + q.b * z) : q.a + q.b * z;
      }
      th[q.index] = v;
    }
    s.seeds[i] = cfg->seed + 1 + (uint64_t)i;
  }
  s.run = 1;
  std::vector<bpf_batch_filter> bf((size_t)P);
  for (int i = 0; i < P; ++i) {
    bf[i].nparticles = cfg->nparticles;
    bf[i].resampler = cfg->resampler;
    bf[i].metropolis_steps = cfg->metropolis_steps;
    bf[i].seed = s.seeds[i];
    for (int m = 0; m < BPF_MAX_THETA; ++m) bf[i].theta[m] = s.theta[(size_t)i * BPF_MAX_THETA + m];
  }
  if (!rc) rc = bpf_batch_create(model, P, bf.data(), cfg->ess_rel, stream, &s.main);
  if (!rc && cfg->moves > 0) rc = bpf_batch_create(model, P, bf.data(), cfg->ess_rel, stream, &s.move);
  if (rc) { delete sp; return rc; }
  s.ll.assign((size_t)P, 0.0);
  s.lw.assign((size_t)P, 0.0);
  s.lp.assign((size_t)P, 0.0);
  for (int i = 0; i < P; ++i) s.lp[i] = prior_of(s, &s.theta[(size_t)i * BPF_MAX_THETA]);
  int nres = 0, naccept = 0, ntotal = 0;
  std::vector<double> ll_new((size_t)P), prop_theta, prop_ll((size_t)P), prop_lp((size_t)P);
  std::vector<uint64_t> prop_seeds((size_t)P);
  std::vector<int> status((size_t)P);
  for (int k = 1; k <= T && !rc; ++k) {
    // MarginalSIR::step: every filter to observation k; weights += increments
    rc = bpf_batch_step_device(s.main, t0 + (k - 1) * dt, t0 + k * dt,
                               (const char*)s.y_dev + (size_t)(k - 1) * s.step_bytes);
    if (!rc) {
      int st = bpf_batch_stats(s.main, ll_new.data(), nullptr, status.data());
      if (st != BPF_OK && st != BPF_E_DEGENERATE) rc = st;
    }
    if (rc) break;
    const double before = log_sum_exp(s.lw);
    for (int i = 0; i < P; ++i) {
      if (status[i] != BPF_OK) ll_new[i] = -INFINITY;
      const double inc = std::isfinite(ll_new[i]) && std::isfinite(s.ll[i]) ? ll_new[i] - s.ll[i] : -INFINITY;
      s.lw[i] += inc;
      s.ll[i] = ll_new[i];
    }
    // interact: marginal likelihood increment and ESS of the parameter weights
    const double after = log_sum_exp(s.lw);
    if (log_evidence_increments) log_evidence_increments[k - 1] = after - before;
    double m = -INFINITY;
    for (double x : s.lw) m = std::fmax(m, x);
    double s1 = 0.0, s2 = 0.0;
    for (double x : s.lw) {
      const double e = std::isfinite(m) ? std::exp(x - m) : 0.0;
      s1 += e;
      s2 += e * e;
    }
    const double ess = s2 > 0.0 ? s1 * s1 / s2 : 0.0;
    if (!(s1 > 0.0)) { rc = BPF_E_DEGENERATE; break; }
    if (k == T || !(ess < cfg->theta_ess_rel * (double)P)) continue;
    // systematic resample of the parameter particles
    ++nres;
    bpf_u32x4 w = bpf_draw(cfg->seed, (uint32_t)P, (uint32_t)(100000 + k), 0u, BPF_RNG_PMMH);
    const double a = bpf_u01d(w.v[0], w.v[1]);
    std::vector<int> anc((size_t)P);
    {
      double cum = 0.0;
      int j = 0;
      for (int i = 0; i < P; ++i) {
        const double target = (i + a) / (double)P * s1;
        while (j < P - 1 && cum + std::exp(s.lw[j] - m) < target) cum += std::exp(s.lw[j++] - m);
        anc[i] = j;
      }
    }
    std::vector<double> th2(s.theta);
    std::vector<uint64_t> sd2(s.seeds);
    std::vector<double> ll2(s.ll), lp2(s.lp);
    for (int i = 0; i < P; ++i) {
      std::memcpy(&th2[(size_t)i * BPF_MAX_THETA], &s.theta[(size_t)anc[i] * BPF_MAX_THETA],
                  BPF_MAX_THETA * sizeof(double));
      sd2[i] = s.seeds[anc[i]];
      ll2[i] = s.ll[anc[i]];
      lp2[i] = s.lp[anc[i]];
    }
    s.theta.swap(th2);
    s.seeds.swap(sd2);
    s.ll.swap(ll2);
    s.lp.swap(lp2);
    const double lw_mean = after - std::log((double)P);
    for (int i = 0; i < P; ++i) s.lw[i] = lw_mean;
    // move: PMMH moves of every parameter particle over observations 1..k
    for (int mv = 0; mv < cfg->moves && !rc; ++mv) {
      const int r = s.run++;
      prop_theta = s.theta;
      for (int i = 0; i < P; ++i) {
        double* pr = &prop_theta[(size_t)i * BPF_MAX_THETA];
        for (int j = 0; j < cfg->nparams; ++j) {
          const bpf_pmmh_param& q = cfg->params[j];
          pr[q.index] += q.step * normal_draw(cfg->seed, i, r, j);
        }
        prop_lp[i] = prior_of(s, pr);
        prop_seeds[i] = cfg->seed + 1 + (uint64_t)r * (uint64_t)P + (uint64_t)i;
        if (!std::isfinite(prop_lp[i]))  // outside the prior: filter the current values, reject below
          std::memcpy(pr, &s.theta[(size_t)i * BPF_MAX_THETA], BPF_MAX_THETA * sizeof(double));
      }
      rc = replay(s, s.move, prop_theta, prop_seeds, k, prop_ll);
      if (rc) break;
      for (int i = 0; i < P; ++i) {
        bool acc;
        const double l2 = std::isfinite(prop_lp[i]) ? prop_ll[i] : -INFINITY;
        if (!std::isfinite(l2)) acc = false;
        else if (!std::isfinite(s.ll[i])) acc = true;
        else acc = std::log(uniform_draw(cfg->seed, i, r, 64)) < (l2 - s.ll[i]) + (prop_lp[i] - s.lp[i]);
        if (acc) {
          std::memcpy(&s.theta[(size_t)i * BPF_MAX_THETA], &prop_theta[(size_t)i * BPF_MAX_THETA],
                      BPF_MAX_THETA * sizeof(double));
          s.seeds[i] = prop_seeds[i];
          s.ll[i] = l2;
          s.lp[i] = prop_lp[i];
          ++naccept;
        }
        ++ntotal;
      }
    }
    if (rc) break;
    // the main batch continues from the surviving (parameters, seed) pairs
    std::vector<double> check((size_t)P);
    rc = replay(s, s.main, s.theta, s.seeds, k, check);
    if (rc) break;
    // (the replay must reproduce every log-likelihood exactly; a mismatch
    // would mean a non-deterministic filter and is reported as an error)
    for (int i = 0; i < P; ++i)
      if (!(check[i] == s.ll[i] || (!std::isfinite(check[i]) && !std::isfinite(s.ll[i])))) rc = BPF_E_CUDA;
  }
  if (!rc) {
    for (int i = 0; i < P; ++i) {
      if (theta_out)
        for (int j = 0; j < cfg->nparams; ++j)
          theta_out[(size_t)i * cfg->nparams + j] = s.theta[(size_t)i * BPF_MAX_THETA + cfg->params[j].index];
      if (log_weights_out) log_weights_out[i] = s.lw[i];
    }
    if (resample_steps) *resample_steps = nres;
    if (acceptance) *acceptance = ntotal > 0 ? (double)naccept / ntotal : 0.0;
  }
  delete sp;
  return rc;
}
