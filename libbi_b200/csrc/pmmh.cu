// Particle-marginal Metropolis-Hastings over many chains at once.
//
// LibBi's MarginalMH (share/src/bi/sampler/MarginalMH.hpp:190-271) runs one
// chain: init filters the initial parameters, then every iteration proposes
// (Simulator::propose, share/src/bi/simulator/Simulator.hpp:336-376), runs a
// full Filter<BootstrapPF>::filter for the proposal when its prior is finite,
// and accepts with probability min(1, exp(loglr + logpr + logqr))
// (acceptReject, MarginalMH.hpp:250-271).  Here C chains advance in
// lockstep: the C proposals of one iteration are filtered together as one
// batch (bpf_filter_batch, one CUDA graph), and the proposal, prior and
// accept/reject arithmetic runs on the host between graph launches.
//
// Random numbers are counter-based (include/bpf_philox.h, tag BPF_RNG_PMMH):
// chain c at filter run r (r = 0 for the initial filter, r = i for
// iteration i) draws the proposal normal of parameter j from block j/2
// (word pair j%2), its acceptance uniform from block 64, and (at r = 0) the
// initial value of parameter j from block 32 + j; the filter of run r uses
// seed  seed + 1 + r*C + c.
#include "internal.cuh"
#include "sampler_common.cuh"

#include <cmath>
#include <cstring>
#include <new>
#include <vector>

struct bpf_pmmh {
  bpf_model_desc model;
  bpf_pmmh_config cfg;
  int T = 0;
  double t0 = 0.0, dt = 0.0;
  std::vector<unsigned char> y;   // T x nchains x nobs (the same data for every chain)
  bpf_batch* batch = nullptr;
  int run = 0;                    // filter runs so far (0 = the initial one)
  std::vector<double> theta;      // current, nchains x BPF_MAX_THETA
  std::vector<double> ll, lp;     // current logLikelihood, logPrior per chain
  std::vector<int> accepted, total;
};

namespace {

using bpf::sampler::log_prior;
using bpf::sampler::normal_draw;
using bpf::sampler::uniform_draw;

int check_cfg(const bpf_model_desc* m, const bpf_pmmh_config* c) {
  if (!m || !c || c->nchains <= 0 || c->nparams <= 0 || c->nparams > BPF_MAX_THETA) return BPF_E_INVALID;
  if (c->nparticles <= 0 || c->nparticles > BPF_BATCH_MAX_PARTICLES) return BPF_E_INVALID;
  if (c->chain_nparticles)
    for (int k = 0; k < c->nchains; ++k)
      if (c->chain_nparticles[k] <= 0 || c->chain_nparticles[k] > BPF_BATCH_MAX_PARTICLES) return BPF_E_INVALID;
  for (int j = 0; j < c->nparams; ++j) {
    const bpf_pmmh_param& q = c->params[j];
    if (q.index < 0 || q.index >= BPF_MAX_THETA || !(q.step >= 0.0)) return BPF_E_INVALID;
    if (q.prior == BPF_PRIOR_UNIFORM && !(q.b > q.a)) return BPF_E_INVALID;
    if ((q.prior == BPF_PRIOR_LOG_NORMAL || q.prior == BPF_PRIOR_GAUSSIAN) && !(q.b > 0.0)) return BPF_E_INVALID;
    if (q.prior < BPF_PRIOR_UNIFORM || q.prior > BPF_PRIOR_GAUSSIAN) return BPF_E_INVALID;
  }
  return BPF_OK;
}

double chain_log_prior(const bpf_pmmh* s, const double* th) {
  double lp = 0.0;
  for (int j = 0; j < s->cfg.nparams; ++j) lp += log_prior(s->cfg.params[j], th[s->cfg.params[j].index]);
  return lp;
}

// filter every chain at `theta` with the seeds of run r; -inf for a
// degenerate filter (MarginalMH::propose catches
// ParticleFilterDegeneratedException, MarginalMH.hpp:241-243)
int filter_all(bpf_pmmh* s, const std::vector<double>& theta, int r, std::vector<double>& ll) {
  const int C = s->cfg.nchains;
  std::vector<uint64_t> seeds((size_t)C);
  for (int c = 0; c < C; ++c) seeds[c] = s->cfg.seed + 1 + (uint64_t)r * (uint64_t)C + (uint64_t)c;
  int rc = bpf_batch_set_seeds(s->batch, seeds.data());
  if (!rc) rc = bpf_batch_set_theta(s->batch, theta.data());
  if (rc) return rc;
  std::vector<int> status((size_t)C);
  rc = bpf_filter_batch(s->batch, s->T, s->t0, s->dt, s->y.data(), ll.data(), nullptr, nullptr, status.data());
  if (rc != BPF_OK && rc != BPF_E_DEGENERATE) return rc;
  for (int c = 0; c < C; ++c)
    if (status[c] != BPF_OK) ll[c] = -INFINITY;
  return BPF_OK;
}

}  // namespace

extern "C" {

int bpf_pmmh_create(const bpf_model_desc* model, const bpf_pmmh_config* cfg, int T, double t0, double dt,
                    const void* y, const double* theta0, void* stream, bpf_pmmh** out) {
  if (!out) return BPF_E_INVALID;
  *out = nullptr;
  if (check_cfg(model, cfg) || T <= 0 || !(dt > 0.0) || !y) return BPF_E_INVALID;
  bpf_pmmh* s = new (std::nothrow) bpf_pmmh();
  if (!s) return BPF_E_NOMEM;
  s->model = *model;
  s->cfg = *cfg;
  s->cfg.chain_nparticles = nullptr;  // copied into the batch below; the caller's array need not outlive create
  s->T = T;
  s->t0 = t0;
  s->dt = dt;
  const int C = cfg->nchains;
  const size_t nobs = model->kind == BPF_MODEL_L96 ? (size_t)model->dim : 1;
  const size_t esz = model->precision == BPF_F64 ? 8 : 4;
  // the same observations for every chain, laid out step-major, filter-major
  s->y.resize((size_t)T * C * nobs * esz);
  for (int k = 0; k < T; ++k)
    for (int c = 0; c < C; ++c)
      std::memcpy(&s->y[((size_t)k * C + c) * nobs * esz], (const unsigned char*)y + (size_t)k * nobs * esz,
                  nobs * esz);
  // initial parameters: theta0, or draws from the prior
  s->theta.assign((size_t)C * BPF_MAX_THETA, 0.0);
  for (int c = 0; c < C; ++c) {
    double* th = &s->theta[(size_t)c * BPF_MAX_THETA];
    for (int i = 0; i < BPF_MAX_THETA; ++i) th[i] = model->theta[i];
    for (int j = 0; j < cfg->nparams; ++j) {
      const bpf_pmmh_param& q = cfg->params[j];
      double v;
      if (theta0) {
        v = theta0[(size_t)c * cfg->nparams + j];
      } else if (q.prior == BPF_PRIOR_UNIFORM) {
        v = q.a + (q.b - q.a) * uniform_draw(cfg->seed, c, 0, 32 + j);
      } else {
        const double z = normal_draw(cfg->seed, c, 0, 64 + 2 * j);
        v = q.prior == BPF_PRIOR_LOG_NORMAL ? std::exp(q.a + q.b * z) : q.a + q.b * z;
      }
      th[q.index] = v;
    }
  }
  std::vector<bpf_batch_filter> bf((size_t)C);
  for (int c = 0; c < C; ++c) {
    bf[c].nparticles = cfg->chain_nparticles ? cfg->chain_nparticles[c] : cfg->nparticles;
    bf[c].resampler = cfg->resampler;
    bf[c].metropolis_steps = cfg->metropolis_steps;
    bf[c].seed = cfg->seed + 1 + (uint64_t)c;
    for (int i = 0; i < BPF_MAX_THETA; ++i) bf[c].theta[i] = s->theta[(size_t)c * BPF_MAX_THETA + i];
  }
  int rc = bpf_batch_create(model, C, bf.data(), cfg->ess_rel, stream, &s->batch);
  if (rc) { delete s; return rc; }
  // MarginalMH::init: filter the initial parameters (MarginalMH.hpp:218-228)
  s->ll.assign((size_t)C, -INFINITY);
  s->lp.assign((size_t)C, 0.0);
  for (int c = 0; c < C; ++c) s->lp[c] = chain_log_prior(s, &s->theta[(size_t)c * BPF_MAX_THETA]);
  rc = filter_all(s, s->theta, 0, s->ll);
  if (rc) { bpf_batch_destroy(s->batch); delete s; return rc; }
  s->run = 1;
  s->accepted.assign((size_t)C, 1);
  s->total.assign((size_t)C, 1);
  *out = s;
  return BPF_OK;
}

int bpf_pmmh_destroy(bpf_pmmh* s) {
  if (!s) return BPF_OK;
  bpf_batch_destroy(s->batch);
  delete s;
  return BPF_OK;
}

int bpf_pmmh_run(bpf_pmmh* s, int iterations, double* samples, double* log_likelihoods, double* log_priors,
                 double* proposal_log_likelihoods, int* accepted) {
  if (!s || iterations < 0) return BPF_E_INVALID;
  const int C = s->cfg.nchains, P = s->cfg.nparams;
  std::vector<double> prop(s->theta.size()), ll2((size_t)C), lp2((size_t)C);
  for (int it = 0; it < iterations; ++it) {
    const int r = s->run;
    // propose: Gaussian random walk on the sampled entries; a proposal
    // outside the prior's support keeps the current values for the filter
    // and is rejected without its likelihood (MarginalMH::propose)
    std::vector<char> finite((size_t)C);
    for (int c = 0; c < C; ++c) {
      const double* th = &s->theta[(size_t)c * BPF_MAX_THETA];
      double* pr = &prop[(size_t)c * BPF_MAX_THETA];
      for (int i = 0; i < BPF_MAX_THETA; ++i) pr[i] = th[i];
      for (int j = 0; j < P; ++j) {
        const bpf_pmmh_param& q = s->cfg.params[j];
        pr[q.index] = th[q.index] + q.step * normal_draw(s->cfg.seed, c, r, j);
      }
      lp2[c] = chain_log_prior(s, pr);
      finite[c] = std::isfinite(lp2[c]);
    }
    std::vector<double> filt_theta(prop);
    for (int c = 0; c < C; ++c)
      if (!finite[c])
        for (int i = 0; i < BPF_MAX_THETA; ++i)
          filt_theta[(size_t)c * BPF_MAX_THETA + i] = s->theta[(size_t)c * BPF_MAX_THETA + i];
    int rc = filter_all(s, filt_theta, r, ll2);
    if (rc) return rc;
    // acceptReject (MarginalMH.hpp:250-271); the random walk is symmetric,
    // so logqr = 0
    for (int c = 0; c < C; ++c) {
      if (!finite[c]) ll2[c] = -INFINITY;
      bool acc;
      if (!std::isfinite(ll2[c])) {
        acc = false;
      } else if (!std::isfinite(s->ll[c])) {
        acc = true;
      } else {
        const double logratio = (ll2[c] - s->ll[c]) + (lp2[c] - s->lp[c]);
        const double u = uniform_draw(s->cfg.seed, c, r, 64);
        acc = std::log(u) < logratio;
      }
      if (acc) {
        for (int j = 0; j < P; ++j) {
          const int i = s->cfg.params[j].index;
          s->theta[(size_t)c * BPF_MAX_THETA + i] = prop[(size_t)c * BPF_MAX_THETA + i];
        }
        s->ll[c] = ll2[c];
        s->lp[c] = lp2[c];
        ++s->accepted[c];
      }
      ++s->total[c];
      if (samples)
        for (int j = 0; j < P; ++j)
          samples[((size_t)it * C + c) * P + j] = s->theta[(size_t)c * BPF_MAX_THETA + s->cfg.params[j].index];
      if (log_likelihoods) log_likelihoods[(size_t)it * C + c] = s->ll[c];
      if (log_priors) log_priors[(size_t)it * C + c] = s->lp[c];
      if (proposal_log_likelihoods) proposal_log_likelihoods[(size_t)it * C + c] = ll2[c];
    }
    s->run = r + 1;
  }
  if (accepted)
    for (int c = 0; c < C; ++c) accepted[c] = s->accepted[c];
  return BPF_OK;
}

int bpf_pmmh_set_proposal(bpf_pmmh* s, bpf_proposal* p) {
  if (!s) return BPF_E_INVALID;
  return bpf_batch_set_proposal(s->batch, p);
}

int bpf_pmmh_state(bpf_pmmh* s, double* theta, double* log_likelihoods, double* log_priors, int* runs) {
  if (!s) return BPF_E_INVALID;
  const int C = s->cfg.nchains;
  for (int c = 0; c < C; ++c) {
    if (theta)
      for (int j = 0; j < s->cfg.nparams; ++j)
        theta[(size_t)c * s->cfg.nparams + j] = s->theta[(size_t)c * BPF_MAX_THETA + s->cfg.params[j].index];
    if (log_likelihoods) log_likelihoods[c] = s->ll[c];
    if (log_priors) log_priors[c] = s->lp[c];
  }
  if (runs) *runs = s->run;
  return BPF_OK;
}

}  // extern "C"
