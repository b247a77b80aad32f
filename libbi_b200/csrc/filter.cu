// Filter handle and the C ABI (include/libbi_b200.h).
//
// The handle owns what LibBi's generated filter client builds
// (share/tt/cpp/client/filter_cpu.cpp.tt:105-184): the particle State
// (structure of arrays, two buffers so that the ancestor gather is fused into
// the next transition's loads), the BootstrapPFState fields (log-weights,
// ancestors, ess, logLikelihood, logIncrements), the resampler's scratch and
// the counter-based RNG.  One BootstrapPF::step is a short, fixed sequence of
// kernels on the handle's stream; nothing returns to the host unless asked.
#include "internal.cuh"
#include "proposal.cuh"
#include "batch.cuh"
#include "resample_common.cuh"

#include <cstdio>
#include <map>
#include <mutex>
#include <cstring>
#include <new>
#include <cmath>
#include <vector>

static thread_local cudaError_t g_last_cuda_error = cudaSuccess;
void bpf_set_last_cuda_error(cudaError_t e) { g_last_cuda_error = e; }

struct bpf_handle {
  bpf::ModelArgs model;
  // a model compiled outside the library (bpf_create_model): its launchers
  // and parameters; model.kind is 0 then
  bool custom = false;
  bpf_model_ops ops{};
  std::vector<double> params;
  bpf_config cfg;
  int n = 0, ld = 0, dim = 0, esz = 0;
  void* x[2] = {nullptr, nullptr};
  int cur = 0;
  double* lw = nullptr;
  int* as = nullptr;
  void* y_dev = nullptr;
  size_t y_cap = 0;
  double* hist = nullptr;  // per-step (inc, ess, resampled) for bpf_filter
  int hist_cap = 0;
  bpf::ResampleScratch rs;
  cudaStream_t stream = nullptr;
  int step = 0;
  // optional device timing: 3 events per step (before resample, before
  // transition, after transition)
  bool timing = false;
  std::vector<cudaEvent_t> ev;
  int ev_steps = 0;
  // learned proposal (bpf_set_proposal), owned by the caller
  bpf_proposal* prop = nullptr;
  // pinned host copy of the step statistics (read back after every step)
  bpf::StepStats* host_stats = nullptr;
  // filters of at most kOneCtaMaxParticles resample in one CTA: the
  // batched resampler on a one-filter table (same ancestors, no grid
  // barriers); its CTA size is autotuned at create
  bpf::BatchFilter* one_filt = nullptr;
  int* one_order = nullptr;
  int one_threads = 1024;
  // path cache (bpf_path_cache): the pruned ancestry of the particles since
  // the record started (pc_len generations), at most pc_cap steps
  bpf::AncestryPool pc;
  bool pc_on = false;
  int pc_cap = 0;   // steps that may be recorded
  int pc_len = 0;   // generations recorded
  bool pc_full = false;
  // the Lorenz-96 step in one launch (resampling as its prologue), selected
  // by bpf_set_step_form: built-in L96 with the systematic resampler, every
  // block of the step resident at once
  bool fused = false;
  // bpf_filter's T steps as one CUDA graph: captured when a call repeats the
  // schedule of the call before it, replayed while the schedule stays
  struct FilterKey {
    int T = 0;
    double t0 = 0.0, dt = 0.0;
    const void* y = nullptr;
    const double* hist = nullptr;
    bool fused = false;
    long long wait_limit = 0;  // the one-launch step takes it as an argument
    bool operator==(const FilterKey& o) const {
      return T == o.T && t0 == o.t0 && dt == o.dt && y == o.y && hist == o.hist && fused == o.fused &&
             wait_limit == o.wait_limit;
    }
  };
  cudaGraphExec_t fgraph = nullptr;
  cudaStream_t capture_stream = nullptr;  // the graph is captured here (the
                                          // legacy default stream cannot
                                          // capture), launched on `stream`
  FilterKey fgraph_key;
  int fgraph_cur = 0;  // the state buffer the replayed steps end in
  FilterKey last_filter;
  bool last_filter_set = false;
};

struct bpf_resampler {
  int kind = 0, B = 0;
  int shape = -1;  // pinned tile shape of the one-launch systematic kernel
  cudaStream_t stream = nullptr;
  bpf::ResampleScratch rs;
  // optional device timing of the compute kernels of each call (events
  // after the status reset and before the read-back)
  bool timing = false;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  double timed_ms = 0.0;
  int timed_calls = 0;
};

namespace {

int check_model(const bpf_model_desc* m) {
  if (!m) return BPF_E_INVALID;
  if (m->precision != BPF_F32 && m->precision != BPF_F64) return BPF_E_INVALID;
  if (m->kind == BPF_MODEL_L96) {
    if (m->integrator != BPF_ODE_RK4) return BPF_E_INVALID;
    const int ok_dims[] = {4, 8, 16, 32, 40};
    bool ok = false;
    for (int d : ok_dims) ok |= (m->dim == d);
    if (!ok) return BPF_E_INVALID;
    if (!(m->h > 0.0) || !(m->theta[1] >= 0.0) || !(m->theta[2] > 0.0)) return BPF_E_INVALID;
  } else if (m->kind == BPF_MODEL_PZ) {
    if (m->integrator != BPF_ODE_RK43 || m->dim != 2 || m->precision != BPF_F64) return BPF_E_INVALID;
    if (!(m->h > 0.0) || !(m->theta[5] >= 0.0) || !(m->theta[6] > 0.0)) return BPF_E_INVALID;
    if (!(m->atoler > 0.0) || !(m->rtoler >= 0.0)) return BPF_E_INVALID;
  } else {
    return BPF_E_INVALID;
  }
  return BPF_OK;
}

// observed values per observation: every component for L96, log P for PZ
int nobs(const bpf_handle* h) {
  if (h->custom) return h->ops.nobs;
  return h->model.kind == BPF_MODEL_L96 ? h->dim : 1;
}

// the step's transition: the built-in model's fused kernel, or the
// launcher of a model compiled outside the library
int launch_model_transition(bpf_handle* h, const bpf::TransitionArgs& ta) {
  if (!h->custom) return bpf::launch_transition(h->model, ta, h->stream);
  bpf_transition_args a{};
  a.x_in = ta.x_in;
  a.x_out = ta.x_out;
  a.ld = ta.ld;
  a.n = ta.n;
  a.ancestors = const_cast<int*>(ta.as);
  a.lw = ta.lw;
  a.y = ta.y;
  a.obs_mask = ta.obs_mask;
  a.t1 = ta.t1;
  a.t2 = ta.t2;
  a.seed = ta.seed;
  a.step = ta.step;
  a.params = h->params.empty() ? nullptr : h->params.data();
  a.nparams = (int)h->params.size();
  a.stats = ta.stats;
  a.partials = ta.partials;
  a.max_partials = ta.max_partials;
  a.counter = ta.counter;
  return h->ops.transition(&a, h->stream);
}

int ensure_y(bpf_handle* h, size_t bytes) {
  if (bytes <= h->y_cap) return BPF_OK;
  if (h->y_dev) cudaFree(h->y_dev);
  h->y_dev = nullptr;
  h->y_cap = 0;
  if (cudaMalloc(&h->y_dev, bytes) != cudaSuccess) return BPF_E_NOMEM;
  h->y_cap = bytes;
  return BPF_OK;
}

int read_stats(bpf_handle* h, bpf::StepStats* out) {
  // through the handle's pinned copy: a direct DMA instead of a staged copy
  bpf::StepStats* dst = h->host_stats ? h->host_stats : out;
  BPF_TRY(cudaMemcpyAsync(dst, h->rs.stats, sizeof(*out), cudaMemcpyDeviceToHost, h->stream));
  BPF_TRY(cudaStreamSynchronize(h->stream));
  if (dst != out) *out = *dst;
  return BPF_OK;
}

// Resample (gated on the device flag set by the previous correct), then the
// fused transition + observation + reduction.  y_dev: device pointer or null.
int timing_event(bpf_handle* h, int which) {
  const size_t idx = (size_t)h->ev_steps * 3 + which;
  while (h->ev.size() <= idx) {
    cudaEvent_t e;
    BPF_TRY(cudaEventCreate(&e));
    h->ev.push_back(e);
  }
  BPF_TRY(cudaEventRecord(h->ev[idx], h->stream));
  return BPF_OK;
}

// append the handle's current state (and, after a step, its ancestors) to
// the path cache
int path_record(bpf_handle* h, bool after_step) {
  if (!h->pc_on || h->pc_full) return BPF_OK;
  if (h->pc_len > h->pc_cap) {
    h->pc_full = true;
    return BPF_OK;
  }
  int rc = after_step && h->pc_len > 0
               ? bpf::ancestry_append(h->pc, h->x[h->cur], h->ld, h->as, h->rs.stats, h->stream)
               : bpf::ancestry_reset(h->pc, h->n, h->dim, h->esz, h->x[h->cur], h->ld, h->stream);
  if (rc) return rc;
  ++h->pc_len;
  return BPF_OK;
}

// y_host, y_bytes: when given, the observation is copied from host memory
// into y_dev on the step's stream, after the resampling launch, so that the
// host issues the copy while the resampler runs; in stream order the copy
// itself runs between the resampler and the transition (a second stream for
// it, joined by events, measured slower end to end: the events cost more
// than the 160-byte copy)
int enqueue_step(bpf_handle* h, double t1, double t2, const void* y_dev, uint64_t mask = ~0ull,
                 const void* y_host = nullptr, size_t y_bytes = 0) {
  const int k = h->step + 1;
  if (h->timing) {
    int rc = timing_event(h, 0);
    if (rc) return rc;
  }
  const bool guided = h->prop && y_dev && (mask | ~((h->dim >= 64 ? 0ull : (1ull << h->dim)) - 1ull)) == ~0ull;
  if (h->fused && !guided) {
    // the whole step in one launch: the resampling (when due) as the
    // transition kernel's prologue
    if (y_host && y_dev)
      BPF_TRY(cudaMemcpyAsync(const_cast<void*>(y_dev), y_host, y_bytes, cudaMemcpyHostToDevice, h->stream));
    if (h->timing) {
      int rc = timing_event(h, 1);
      if (rc) return rc;
    }
    bpf::FusedStepArgs fa;
    fa.t.x_in = h->x[h->cur];
    fa.t.x_out = h->x[h->cur ^ 1];
    fa.t.ld = h->ld;
    fa.t.n = h->n;
    fa.t.as = h->as;
    fa.t.lw = h->lw;
    fa.t.y = y_dev;
    fa.t.t1 = t1;
    fa.t.t2 = t2;
    fa.t.seed = h->cfg.seed;
    fa.t.step = k;
    fa.t.stats = h->rs.stats;
    fa.t.partials = h->rs.partials;
    fa.t.max_partials = h->rs.max_partials;
    fa.t.counter = h->rs.counters + 4;
    fa.t.obs_mask = mask;
    fa.E = h->rs.E;
    fa.ecoarse = h->rs.etile;
    fa.pub = h->rs.pub;
    fa.max_pub = h->rs.pub_entries;
    fa.epoch_word = h->rs.counters + bpf::kEpochWord;
    int rc = bpf::launch_fused_step(h->model, fa, h->stream);
    if (rc) return rc;
    if (h->timing) {
      rc = timing_event(h, 2);
      if (rc) return rc;
      h->ev_steps += 1;
    }
    h->cur ^= 1;
    h->step = k;
    return path_record(h, true);
  }
  const int* gate = &h->rs.stats->resample;
  bpf::ResampleArgs ra;
  ra.kind = h->cfg.resampler;
  ra.n = h->n;
  ra.B = h->cfg.metropolis_steps;
  ra.lw = h->lw;
  ra.uniforms = nullptr;
  ra.seed = h->cfg.seed;
  ra.step = k;
  ra.permute = 1;
  ra.as = h->as;
  ra.Os_out = nullptr;
  ra.gate = gate;
  ra.max_known = true;
  int rc = h->one_filt ? bpf::launch_batch_resample(h->lw, h->as, h->one_filt, h->one_order, 1, h->n, h->rs.stats,
                                                    h->rs.lu, h->rs.Os, k, h->stream, h->one_threads)
                       : bpf::launch_resample(ra, h->rs, h->stream);
  if (rc) return rc;
  if (y_host && y_dev) BPF_TRY(cudaMemcpyAsync(const_cast<void*>(y_dev), y_host, y_bytes, cudaMemcpyHostToDevice,
                                               h->stream));
  if (h->timing) {
    rc = timing_event(h, 1);
    if (rc) return rc;
  }
  if (guided) {
    // guided step (every component observed): the learned proposal instead
    // of the transition
    const double dt = bpf::proposal_dt(h->prop);
    if (std::fabs((t2 - t1) - dt) > 1e-9 * dt) return BPF_E_INVALID;
    bpf::GuidedArgs ga;
    ga.x_in = h->x[h->cur];
    ga.x_out = h->x[h->cur ^ 1];
    ga.ld = h->ld;
    ga.n = h->n;
    ga.as = h->as;
    ga.lw = h->lw;
    ga.y = y_dev;
    ga.t1 = t1;
    ga.t2 = t2;
    ga.seed = h->cfg.seed;
    ga.step = k;
    for (int i = 0; i < BPF_MAX_THETA; ++i) ga.theta[i] = h->model.theta[i];
    ga.h = h->model.h;
    ga.stats = h->rs.stats;
    ga.partials = h->rs.partials;
    ga.max_partials = h->rs.max_partials;
    ga.counter = h->rs.counters + 4;
    rc = bpf::launch_guided(*bpf::proposal_net(h->prop), ga, h->stream);
    if (rc) return rc;
    if (h->timing) {
      rc = timing_event(h, 2);
      if (rc) return rc;
      h->ev_steps += 1;
    }
    h->cur ^= 1;
    h->step = k;
    return path_record(h, true);
  }
  bpf::TransitionArgs ta;
  ta.x_in = h->x[h->cur];
  ta.x_out = h->x[h->cur ^ 1];
  ta.ld = h->ld;
  ta.n = h->n;
  ta.as = h->as;
  ta.lw = h->lw;
  ta.y = y_dev;
  ta.t1 = t1;
  ta.t2 = t2;
  ta.seed = h->cfg.seed;
  ta.step = k;
  ta.stats = h->rs.stats;
  ta.partials = h->rs.partials;
  ta.max_partials = h->rs.max_partials;
  ta.counter = h->rs.counters + 4;
  ta.obs_mask = mask;
  rc = launch_model_transition(h, ta);
  if (rc) return rc;
  if (h->timing) {
    rc = timing_event(h, 2);
    if (rc) return rc;
    h->ev_steps += 1;
  }
  h->cur ^= 1;
  h->step = k;
  return path_record(h, true);
}

// point the step statistics at a whole-filter run's record (each step's
// last block then writes its entry), or at nothing
__global__ void k_set_hist(bpf::StepStats* st, double* hist, int n) {
  st->hist = hist;
  st->hist_n = n;
}

// the status back to BPF_OK, the grid-barrier word (counters[8..9]) to
// zero and the resampler's epoch (counters[kEpochWord]) one further: a
// cooperative launch that timed out can leave the barrier word part-counted
// and tagged words of the abandoned epoch behind
__global__ void k_set_status_ok(bpf::StepStats* st, unsigned* counters) {
  st->status = BPF_OK;
  counters[8] = 0u;
  counters[9] = 0u;
  counters[bpf::kEpochWord] += 1u;
}

// set_elements(s.logWeights(), s.logLikelihood), Resampler.hpp:177
__global__ void k_reset_lw(double* lw, int n, const bpf::StepStats* st) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) lw[i] = st->ll;
}

}  // namespace

// Largest filter resampled by one CTA.  On B200 (L96, d=40, a resampling
// at every step) one CTA takes 9.6 / 12.3 / 16.4 us per systematic
// resampling at N = 256 / 1024 / 4096 against 13.7 / 14.3 / 17.3 us for the
// grid-wide kernels (Metropolis at 4096: 14.3 against 29.8 us), but 62 us
// at 16384 against 17.8: past a few thousand particles the work needs more
// than one SM.
constexpr int kOneCtaMaxParticles = 4096;

// CTA size of the one-CTA resampler, timed once per process for each
// resampler and particle count (the sizes compute the same ancestors)
static int one_cta_threads(bpf_handle* h, int resampler) {
  static std::mutex mu;
  static std::map<std::pair<int, int>, int> tuned;
  const std::pair<int, int> key(resampler, h->n);
  {
    std::lock_guard<std::mutex> g(mu);
    auto it = tuned.find(key);
    if (it != tuned.end()) {
      h->one_threads = it->second;
      return BPF_OK;
    }
  }
  int rc = bpf::tune_batch_resample(h->one_filt, h->one_order, 1, h->n, h->ld, h->stream, &h->one_threads, nullptr);
  if (rc) return rc;
  std::lock_guard<std::mutex> g(mu);
  tuned[key] = h->one_threads;
  return BPF_OK;
}

extern "C" {

const char* bpf_version(void) { return "libbi_b200 0.1 (sm_100a)"; }

const char* bpf_status_string(int s) {
  switch (s) {
    case BPF_OK: return "ok";
    case BPF_E_DEGENERATE: return "particle filter degenerated (weights sum to zero or are not finite)";
    case BPF_E_INVALID: return "invalid argument";
    case BPF_E_CUDA: return cudaGetErrorString(g_last_cuda_error);
    case BPF_E_TIMEOUT: return "bounded device wait gave up";
    case BPF_E_NOMEM: return "device allocation failed";
    case BPF_E_TOO_LARGE: return "more particles than the static scratch holds (BPF_STATIC_MAX_PARTICLES)";
    default: return "unknown status";
  }
}

static int check_config(const bpf_config* config) {
  if (!config || config->nparticles <= 0) return BPF_E_INVALID;
  if (config->resampler < BPF_RESAMPLER_SYSTEMATIC || config->resampler > BPF_RESAMPLER_METROPOLIS)
    return BPF_E_INVALID;
  if (config->resampler == BPF_RESAMPLER_METROPOLIS && config->metropolis_steps < 0) return BPF_E_INVALID;
  // Resampler constructor pre-condition, share/src/bi/resampler/Resampler.hpp:129
  if (!(config->ess_rel >= 0.0 && config->ess_rel <= 1.0)) return BPF_E_INVALID;
  return BPF_OK;
}

// buffers, resampler and initial draw of a handle whose model fields are set
static int create_common(bpf_handle* h, const bpf_config* config, int dim, int precision, bpf_handle** out) {
  h->cfg = *config;
  h->stream = (cudaStream_t)config->stream;
  h->n = config->nparticles;
  // leading dimension rounded up to 32 particles (State::roundup for CUDA,
  // share/src/bi/state/State.hpp:40-57), so every component row is 128-byte aligned
  h->ld = ((h->n + 31) / 32) * 32;
  h->dim = dim;
  h->esz = precision == BPF_F64 ? 8 : 4;
  const size_t xb = (size_t)h->ld * h->dim * h->esz;
  if (cudaMalloc(&h->x[0], xb) != cudaSuccess || cudaMalloc(&h->x[1], xb) != cudaSuccess ||
      cudaMalloc((void**)&h->lw, (size_t)h->ld * sizeof(double)) != cudaSuccess ||
      cudaMalloc((void**)&h->as, (size_t)h->ld * sizeof(int)) != cudaSuccess) {
    bpf_destroy(h);
    return BPF_E_NOMEM;
  }
  int rc = bpf::scratch_alloc(h->rs, h->n);
  if (rc) { bpf_destroy(h); return rc; }
  if (cudaMallocHost((void**)&h->host_stats, sizeof(bpf::StepStats)) != cudaSuccess) {
    cudaGetLastError();
    h->host_stats = nullptr;  // read back through pageable memory instead
  }
  if (h->n <= kOneCtaMaxParticles) {
    // one CTA resamples the whole filter (the resampler reads n, off,
    // resampler, B and seed of the table entry)
    bpf::BatchFilter f{};
    f.n = h->n;
    f.off = 0;
    f.resampler = config->resampler;
    f.B = config->metropolis_steps;
    f.seed = config->seed;
    const int zero = 0;
    if (cudaMalloc((void**)&h->one_filt, sizeof(f)) != cudaSuccess ||
        cudaMalloc((void**)&h->one_order, sizeof(int)) != cudaSuccess ||
        cudaMemcpy(h->one_filt, &f, sizeof(f), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(h->one_order, &zero, sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess) {
      cudaGetLastError();
      bpf_destroy(h);
      return BPF_E_NOMEM;
    }
    rc = bpf::configure_batch_resample(h->n);
    if (!rc) rc = one_cta_threads(h, config->resampler);
    if (rc) { bpf_destroy(h); return rc; }
  } else if (config->resampler == BPF_RESAMPLER_SYSTEMATIC && bpf::autotuned_shape(h->n) == -1) {
    // the one-launch cooperative resampler's tile shape for this N, tuned
    // once per size class (the shapes compute the same ancestors, so only
    // the speed depends on it)
    int best = -1;
    if (bpf::autotune_systematic(h->n, h->stream, &best, nullptr) != BPF_OK) cudaGetLastError();
  }
  rc = bpf_init(h);
  if (rc) { bpf_destroy(h); return rc; }
  *out = h;
  return BPF_OK;
}

int bpf_create(const bpf_model_desc* model, const bpf_config* config, bpf_handle** out) {
  if (!out || !config) return BPF_E_INVALID;
  *out = nullptr;
  int rc = check_model(model);
  if (rc) return rc;
  if ((rc = check_config(config))) return rc;
  bpf_handle* h = new (std::nothrow) bpf_handle();
  if (!h) return BPF_E_NOMEM;
  h->model.kind = model->kind;
  h->model.dim = model->dim;
  h->model.precision = model->precision;
  h->model.integrator = model->integrator;
  h->model.h = model->h;
  h->model.atoler = model->atoler;
  h->model.rtoler = model->rtoler;
  for (int i = 0; i < BPF_MAX_THETA; ++i) h->model.theta[i] = model->theta[i];
  return create_common(h, config, model->dim, model->precision, out);
}

int bpf_set_step_form(bpf_handle* h, int fused) {
  if (!h) return BPF_E_INVALID;
  if (!fused) {
    h->fused = false;
    return BPF_OK;
  }
  if (h->custom || h->cfg.resampler != BPF_RESAMPLER_SYSTEMATIC || !bpf::fused_step_available(h->model, h->n))
    return BPF_E_INVALID;
  h->fused = true;
  return BPF_OK;
}

int bpf_step_form(bpf_handle* h, int* fused) {
  if (!h || !fused) return BPF_E_INVALID;
  *fused = h->fused ? 1 : 0;
  return BPF_OK;
}

int bpf_create_model(const bpf_model_ops* ops, const double* params, const bpf_config* config, bpf_handle** out) {
  if (!out || !config || !ops) return BPF_E_INVALID;
  *out = nullptr;
  if (ops->dim <= 0 || ops->nobs < 0 || ops->nobs > 64 || ops->nparams < 0 || ops->nparams > 4096 ||
      (ops->nparams > 0 && !params) || !ops->init || !ops->transition ||
      (ops->precision != BPF_F32 && ops->precision != BPF_F64))
    return BPF_E_INVALID;
  int rc = check_config(config);
  if (rc) return rc;
  bpf_handle* h = new (std::nothrow) bpf_handle();
  if (!h) return BPF_E_NOMEM;
  h->custom = true;
  h->ops = *ops;
  if (ops->nparams > 0) h->params.assign(params, params + ops->nparams);
  h->model.kind = 0;
  h->model.dim = ops->dim;
  h->model.precision = ops->precision;
  return create_common(h, config, ops->dim, ops->precision, out);
}

int bpf_destroy(bpf_handle* h) {
  if (!h) return BPF_OK;
  if (h->stream) cudaStreamSynchronize(h->stream); else cudaDeviceSynchronize();
  if (h->x[0]) cudaFree(h->x[0]);
  if (h->x[1]) cudaFree(h->x[1]);
  if (h->lw) cudaFree(h->lw);
  if (h->as) cudaFree(h->as);
  if (h->y_dev) cudaFree(h->y_dev);
  if (h->hist) cudaFree(h->hist);
  for (cudaEvent_t e : h->ev) cudaEventDestroy(e);
  if (h->host_stats) cudaFreeHost(h->host_stats);
  if (h->fgraph) cudaGraphExecDestroy(h->fgraph);
  if (h->capture_stream) cudaStreamDestroy(h->capture_stream);
  bpf::ancestry_free(h->pc);
  void* g[] = {h->one_filt, h->one_order};
  for (void* p : g)
    if (p) cudaFree(p);
  bpf::scratch_free(h->rs);
  delete h;
  return BPF_OK;
}

// ---- path cache and samplePath --------------------------------------------

}  // extern "C"

namespace {

constexpr int kPathThreads = 1024;

// p ~ multinomial(exp(lw)) from one uniform u, as RngHost::multinomial
// (share/src/bi/host/random/RngHost.hpp:120-139): Ps = inclusive scan of
// exp(lw - max) (here exact fixed-point sums rounded once), x = Ps_last * u,
// p = first index with Ps_p >= x; p = 0 when the weights sum to zero.
__global__ void __launch_bounds__(kPathThreads)
k_sample_index(const double* __restrict__ lw, int n, const double* u_in, uint64_t seed, int step, int* out) {
  __shared__ double s_max[kPathThreads / 32];
  __shared__ int s_best;
  const int IT = (n + kPathThreads - 1) / kPathThreads;
  const int i0 = min(n, (int)threadIdx.x * IT), i1 = min(n, i0 + IT);
  double m = -INFINITY;
  for (int i = i0; i < i1; ++i) m = bpf::nan_max(m, lw[i]);
  for (int d = 16; d > 0; d >>= 1) m = bpf::nan_max(m, __shfl_xor_sync(0xffffffffu, m, d));
  if ((threadIdx.x & 31) == 0) s_max[threadIdx.x >> 5] = m;
  if (threadIdx.x == 0) s_best = n;
  __syncthreads();
  double mx = -INFINITY;
  for (int w = 0; w < kPathThreads / 32; ++w) mx = bpf::nan_max(mx, s_max[w]);
  bpf::u128 acc = bpf::u128_zero();
  for (int i = i0; i < i1; ++i) {
    bpf::u128 q; q.lo = bpf::weight_to_fixed(bpf::nanexp(__dsub_rn(lw[i], mx))); q.hi = 0;
    acc = bpf::u128_add(acc, q);
  }
  bpf::u128 tot;
  bpf::u128 Q = bpf::block_exclusive_scan_u128_nt<kPathThreads>(acc, &tot);
  const double W = bpf::u128_to_weight(tot);
  double u;
  if (u_in) {
    u = *u_in;
  } else {
    bpf_u32x4 r = bpf_draw(seed, 0u, (uint32_t)step, 0u, BPF_RNG_PATH);
    u = bpf_u01d(r.v[0], r.v[1]);
  }
  if (!(W > 0.0)) {
    if (threadIdx.x == 0) *out = 0;
    return;
  }
  const double x = __dmul_rn(W, u);
  for (int i = i0; i < i1; ++i) {
    bpf::u128 q; q.lo = bpf::weight_to_fixed(bpf::nanexp(__dsub_rn(lw[i], mx))); q.hi = 0;
    Q = bpf::u128_add(Q, q);
    if (bpf::u128_to_weight(Q) >= x) {
      atomicMin(&s_best, i);
      break;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) *out = s_best < n ? s_best : n - 1;
}

}  // namespace

extern "C" {

int bpf_path_cache(bpf_handle* h, int max_steps) {
  if (!h || max_steps < 0) return BPF_E_INVALID;
  BPF_TRY(cudaStreamSynchronize(h->stream));
  bpf::ancestry_free(h->pc);
  h->pc_on = false;
  h->pc_cap = 0;
  h->pc_len = 0;
  h->pc_full = false;
  if (max_steps == 0) return BPF_OK;
  h->pc_on = true;
  h->pc_cap = max_steps;
  return path_record(h, false);  // the current state opens the record
}

int bpf_path_cache_nodes(bpf_handle* h, int* nodes, int* capacity) {
  if (!h || !h->pc_on || h->pc_len == 0) return BPF_E_INVALID;
  return bpf::ancestry_nodes(h->pc, h->stream, nodes, capacity);
}

int bpf_sample_path(bpf_handle* h, const double* u, void* path, int* particle, int* len) {
  if (!h || !h->pc_on || h->pc_len == 0) return BPF_E_INVALID;
  if (h->pc_full) return BPF_E_TOO_LARGE;
  if (len) *len = h->pc_len;
  int* d_p = nullptr;
  void* d_path = nullptr;
  const size_t pb = (size_t)h->pc_len * h->dim * h->esz;
  if (cudaMalloc((void**)&d_p, sizeof(int)) != cudaSuccess || cudaMalloc(&d_path, pb) != cudaSuccess) {
    cudaGetLastError();
    if (d_p) cudaFree(d_p);
    return BPF_E_NOMEM;
  }
  k_sample_index<<<1, kPathThreads, 0, h->stream>>>(h->lw, h->n, u, h->cfg.seed, h->step, d_p);
  cudaError_t e = cudaGetLastError();
  int rc = e == cudaSuccess ? bpf::ancestry_trace(h->pc, h->pc_len, d_p, d_path, h->stream) : BPF_E_CUDA;
  int p = 0;
  if (!rc) e = cudaMemcpyAsync(&p, d_p, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
  if (!rc && e == cudaSuccess && path) e = cudaMemcpyAsync(path, d_path, pb, cudaMemcpyDeviceToHost, h->stream);
  if (!rc && e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  cudaFree(d_p);
  cudaFree(d_path);
  if (rc) return rc;
  if (e != cudaSuccess) { bpf_set_last_cuda_error(e); return BPF_E_CUDA; }
  if (particle) *particle = p;
  return BPF_OK;
}

int bpf_set_proposal(bpf_handle* h, bpf_proposal* p) {
  if (!h) return BPF_E_INVALID;
  if (p) {
    if (h->model.kind != BPF_MODEL_L96 || h->model.dim != 40 || h->model.precision != BPF_F32) return BPF_E_INVALID;
    const bpf::ProposalNet& net = *bpf::proposal_net(p);
    if (net.dim != h->dim || net.hidden != bpf::kProposalHidden) return BPF_E_INVALID;
  }
  h->prop = p;
  return BPF_OK;
}

int bpf_state_ptrs(bpf_handle* h, void** x, double** lw, int** as, int* ld) {
  if (!h) return BPF_E_INVALID;
  if (x) *x = h->x[h->cur];
  if (lw) *lw = h->lw;
  if (as) *as = h->as;
  if (ld) *ld = h->ld;
  return BPF_OK;
}

int bpf_init(bpf_handle* h) {
  if (!h) return BPF_E_INVALID;
  h->cur = 0;
  h->step = 0;
  // the last-block tickets and grid-barrier words start from zero (a
  // cooperative resampling that timed out can leave a barrier counter set)
  // and the resampler's epoch moves on
  int rc = bpf::reset_scratch_words(h->rs, h->stream);
  if (rc) return rc;
  if (h->custom) {
    bpf_init_args a{};
    a.x = h->x[0];
    a.ld = h->ld;
    a.n = h->n;
    a.lw = h->lw;
    a.seed = h->cfg.seed;
    a.params = h->params.empty() ? nullptr : h->params.data();
    a.nparams = (int)h->params.size();
    rc = h->ops.init(&a, h->stream);
    if (!rc) rc = bpf::launch_stats_init(h->rs.stats, h->n, h->cfg.ess_rel, h->stream);
  } else {
    rc = bpf::launch_init(h->model, h->x[0], h->ld, h->n, h->lw, h->cfg.seed, h->rs.stats, h->cfg.ess_rel,
                          h->stream);
  }
  if (rc) return rc;
  h->pc_len = 0;
  h->pc_full = false;
  return path_record(h, false);
}

static void fill_out(const bpf::StepStats& s, bpf_step_out* out) {
  out->ess = s.ess;
  out->log_weight_sum = s.lW;
  out->log_increment = s.inc;
  out->log_likelihood = s.ll;
  out->resampled = s.resampled;
  out->status = s.status;
}

int bpf_step(bpf_handle* h, double t1, double t2, const void* y, bpf_step_out* out) {
  if (!h || !(t1 < t2)) return BPF_E_INVALID;
  const void* yd = nullptr;
  size_t yb = 0;
  if (y) {
    yb = (size_t)nobs(h) * h->esz;
    int rc = ensure_y(h, yb);
    if (rc) return rc;
    yd = h->y_dev;
  }
  int rc = enqueue_step(h, t1, t2, yd, ~0ull, y, yb);
  if (rc) return rc;
  if (out) {
    bpf::StepStats s;
    rc = read_stats(h, &s);
    if (rc) return rc;
    fill_out(s, out);
    return s.status;
  }
  return BPF_OK;
}

int bpf_step_sparse(bpf_handle* h, double t1, double t2, const void* y, const int* idx, int nidx, bpf_step_out* out) {
  if (!h || !(t1 < t2) || nidx < 0 || (nidx > 0 && (!y || !idx))) return BPF_E_INVALID;
  const int nob = nobs(h);
  if (nob > 64) return BPF_E_INVALID;
  uint64_t mask = 0;
  std::vector<unsigned char> dense((size_t)nob * h->esz, 0);
  for (int j = 0; j < nidx; ++j) {
    const int i = idx[j];
    if (i < 0 || i >= nob || ((mask >> i) & 1ull)) return BPF_E_INVALID;
    mask |= 1ull << i;
    std::memcpy(&dense[(size_t)i * h->esz], (const unsigned char*)y + (size_t)j * h->esz, h->esz);
  }
  const void* yd = nullptr;
  if (nidx > 0) {
    int rc = ensure_y(h, dense.size());
    if (rc) return rc;
    BPF_TRY(cudaMemcpyAsync(h->y_dev, dense.data(), dense.size(), cudaMemcpyHostToDevice, h->stream));
    BPF_TRY(cudaStreamSynchronize(h->stream));  // dense is a temporary
    yd = h->y_dev;
  }
  int rc = enqueue_step(h, t1, t2, yd, mask);
  if (rc) return rc;
  if (out) {
    bpf::StepStats s;
    rc = read_stats(h, &s);
    if (rc) return rc;
    fill_out(s, out);
    return s.status;
  }
  return BPF_OK;
}

int bpf_step_device(bpf_handle* h, double t1, double t2, const void* y_dev, bpf_step_out* out) {
  if (!h || !(t1 < t2)) return BPF_E_INVALID;
  int rc = enqueue_step(h, t1, t2, y_dev);
  if (rc) return rc;
  if (out) {
    bpf::StepStats s;
    rc = read_stats(h, &s);
    if (rc) return rc;
    fill_out(s, out);
    return s.status;
  }
  return BPF_OK;
}

// the T steps of bpf_filter (each step's last block records its entry in
// h->hist through the step statistics)
static int launch_filter_steps(bpf_handle* h, int T, double t0, double dt) {
  for (int k = 1; k <= T; ++k) {
    const double t1 = t0 + (k - 1) * dt, t2 = t0 + k * dt;
    int rc = enqueue_step(h, t1, t2, (const char*)h->y_dev + (size_t)(k - 1) * nobs(h) * h->esz);
    if (rc) return rc;
  }
  BPF_TRY(cudaGetLastError());
  return BPF_OK;
}

// Capture the steps into h->fgraph on the handle's capture stream (false:
// they would not capture; nothing was launched and the handle is as before)
static bool capture_filter_steps(bpf_handle* h, int T, double t0, double dt, const bpf_handle::FilterKey& key) {
  if (h->fgraph) {
    cudaGraphExecDestroy(h->fgraph);
    h->fgraph = nullptr;
  }
  if (!h->capture_stream && cudaStreamCreateWithFlags(&h->capture_stream, cudaStreamNonBlocking) != cudaSuccess) {
    h->capture_stream = nullptr;
    cudaGetLastError();
    return false;
  }
  const int cur0 = h->cur, step0 = h->step;
  if (cudaStreamBeginCapture(h->capture_stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  cudaStream_t launch_stream = h->stream;
  h->stream = h->capture_stream;
  const int rc = launch_filter_steps(h, T, t0, dt);
  h->stream = launch_stream;
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(h->capture_stream, &g);
  if (e == cudaSuccess && rc == BPF_OK && g) e = cudaGraphInstantiate(&h->fgraph, g, 0);
  if (g) cudaGraphDestroy(g);
  if (e != cudaSuccess || rc != BPF_OK || !h->fgraph) {
    if (h->fgraph) cudaGraphExecDestroy(h->fgraph);
    h->fgraph = nullptr;
    cudaGetLastError();
    h->cur = cur0;
    h->step = step0;
    return false;
  }
  h->fgraph_key = key;
  h->fgraph_cur = h->cur;
  return true;
}

// The steps of a filter run after bpf_init.  A caller that filters the same
// schedule again and again (a sampler's Filter::filter per proposal) gets
// them as one CUDA graph from the second call on: the launches of T steps
// then cost the host one graph launch.  Timing events, path recording,
// learned proposals and models compiled outside the library run the steps
// as separate launches.
static int enqueue_filter_steps(bpf_handle* h, int T, double t0, double dt) {
  bpf_handle::FilterKey key;
  key.T = T;
  key.t0 = t0;
  key.dt = dt;
  key.y = h->y_dev;
  key.hist = h->hist;
  key.fused = h->fused;
  key.wait_limit = bpf::barrier_limit();
  const bool graphable = !h->custom && !h->prop && !h->timing && !h->pc_on && h->cur == 0 && h->step == 0;
  if (graphable && h->fgraph && h->fgraph_key == key) {
    BPF_TRY(cudaGraphLaunch(h->fgraph, h->stream));
    h->cur = h->fgraph_cur;
    h->step = T;
    return BPF_OK;
  }
  const bool repeat = h->last_filter_set && h->last_filter == key;
  h->last_filter = key;
  h->last_filter_set = true;
  if (graphable && repeat && capture_filter_steps(h, T, t0, dt, key)) {
    BPF_TRY(cudaGraphLaunch(h->fgraph, h->stream));
    return BPF_OK;
  }
  return launch_filter_steps(h, T, t0, dt);
}

int bpf_filter(bpf_handle* h, int T, double t0, double dt, const void* y, double* log_increments, double* ess,
               double* log_likelihood) {
  if (!h || T <= 0 || !(dt > 0.0) || !y) return BPF_E_INVALID;
  int rc = bpf_init(h);
  if (rc) return rc;
  const size_t yb = (size_t)T * nobs(h) * h->esz;
  rc = ensure_y(h, yb);
  if (rc) return rc;
  BPF_TRY(cudaMemcpyAsync(h->y_dev, y, yb, cudaMemcpyHostToDevice, h->stream));
  if (T > h->hist_cap) {
    if (h->hist) cudaFree(h->hist);
    h->hist = nullptr;
    h->hist_cap = 0;
    if (cudaMalloc((void**)&h->hist, (size_t)3 * T * sizeof(double)) != cudaSuccess) return BPF_E_NOMEM;
    h->hist_cap = T;
  }
  k_set_hist<<<1, 1, 0, h->stream>>>(h->rs.stats, h->hist, T);
  rc = enqueue_filter_steps(h, T, t0, dt);
  k_set_hist<<<1, 1, 0, h->stream>>>(h->rs.stats, nullptr, 0);
  if (rc) return rc;
  // BootstrapPF::term: logLikelihood = logsumexp(lws) - log P
  // (share/src/bi/filter/BootstrapPF.hpp:192-196); keep the step statistics
  bpf::StepStats s;
  rc = read_stats(h, &s);
  if (rc) return rc;
  if (s.status != BPF_OK) return s.status;
  rc = bpf::launch_logsumexp(h->lw, h->n, h->rs, h->stream);
  if (rc) return rc;
  bpf::StepStats s2;
  rc = read_stats(h, &s2);
  if (rc) return rc;
  if (log_likelihood) *log_likelihood = s2.lW - std::log((double)h->n);
  // restore the step statistics the term reduction overwrote
  BPF_TRY(cudaMemcpyAsync(h->rs.stats, &s, sizeof(s), cudaMemcpyHostToDevice, h->stream));
  if (log_increments || ess) {
    double* tmp = new (std::nothrow) double[(size_t)3 * T];
    if (!tmp) return BPF_E_NOMEM;
    cudaError_t e = cudaMemcpyAsync(tmp, h->hist, (size_t)3 * T * sizeof(double), cudaMemcpyDeviceToHost,
                                    h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) { delete[] tmp; bpf_set_last_cuda_error(e); return BPF_E_CUDA; }
    for (int k = 0; k < T; ++k) {
      if (log_increments) log_increments[k] = tmp[3 * k];
      if (ess) ess[k] = tmp[3 * k + 1];
    }
    delete[] tmp;
  }
  BPF_TRY(cudaStreamSynchronize(h->stream));
  return BPF_OK;
}

int bpf_reduce(bpf_handle* h, double* lW, double* ess) {
  if (!h) return BPF_E_INVALID;
  bpf::StepStats keep;
  int rc = read_stats(h, &keep);
  if (rc) return rc;
  rc = bpf::launch_lw_reduce(h->lw, h->n, h->rs, h->stream);
  if (rc) return rc;
  bpf::StepStats s;
  rc = read_stats(h, &s);
  if (rc) return rc;
  if (lW) *lW = s.lW;
  if (ess) *ess = s.ess;
  // the reduction leaves mx/s1/s2/ess/lW of the current weights; keep the
  // filter's likelihood bookkeeping
  s.ll = keep.ll; s.inc = keep.inc; s.step = keep.step; s.resample = keep.resample;
  s.resampled = keep.resampled; s.ess_rel = keep.ess_rel; s.n = keep.n;
  BPF_TRY(cudaMemcpyAsync(h->rs.stats, &s, sizeof(s), cudaMemcpyHostToDevice, h->stream));
  BPF_TRY(cudaStreamSynchronize(h->stream));
  return BPF_OK;
}

int bpf_resample(bpf_handle* h, const double* uniforms, int* ancestors_out) {
  if (!h) return BPF_E_INVALID;
  // fresh max / reduction over the current log-weights
  bpf::StepStats keep;
  int rc = read_stats(h, &keep);
  if (rc) return rc;
  if (keep.status != BPF_OK) return keep.status;
  rc = bpf::launch_lw_reduce(h->lw, h->n, h->rs, h->stream);
  if (rc) return rc;
  bpf::ResampleArgs ra;
  ra.kind = h->cfg.resampler;
  ra.n = h->n;
  ra.B = h->cfg.metropolis_steps;
  ra.lw = h->lw;
  ra.uniforms = uniforms;
  ra.seed = h->cfg.seed;
  ra.step = h->step + 1;
  ra.permute = 1;
  ra.as = h->as;
  ra.Os_out = nullptr;
  ra.gate = nullptr;
  ra.max_known = true;
  rc = bpf::launch_resample(ra, h->rs, h->stream);
  if (rc) return rc;
  bpf::StepStats s;
  rc = read_stats(h, &s);
  if (rc) return rc;
  if (s.status != BPF_OK) return s.status;
  // gather (out of place into the other buffer) and reset log-weights to the
  // log-likelihood (Resampler.hpp:176-177)
  const void* X = h->x[h->cur];
  void* Y = h->x[h->cur ^ 1];
  rc = bpf::launch_gather(h->as, X, Y, h->n, h->dim, h->ld, h->esz, nullptr, h->stream);
  if (rc) return rc;
  h->cur ^= 1;
  k_reset_lw<<<(h->n + 255) / 256, 256, 0, h->stream>>>(h->lw, h->n, h->rs.stats);
  BPF_TRY(cudaGetLastError());
  if (ancestors_out) {
    BPF_TRY(cudaMemcpyAsync(ancestors_out, h->as, (size_t)h->n * sizeof(int), cudaMemcpyDeviceToDevice,
                            h->stream));
  }
  keep.resample = 0;
  keep.resampled = 1;
  BPF_TRY(cudaMemcpyAsync(h->rs.stats, &keep, sizeof(keep), cudaMemcpyHostToDevice, h->stream));
  BPF_TRY(cudaStreamSynchronize(h->stream));
  return BPF_OK;
}

int bpf_timing_enable(bpf_handle* h, int enable) {
  if (!h) return BPF_E_INVALID;
  h->timing = enable != 0;
  h->ev_steps = 0;
  return BPF_OK;
}

int bpf_timing_read(bpf_handle* h, int reset, double* resample_ms, double* transition_ms, int* steps) {
  if (!h) return BPF_E_INVALID;
  BPF_TRY(cudaStreamSynchronize(h->stream));
  double r = 0.0, t = 0.0;
  for (int s = 0; s < h->ev_steps; ++s) {
    float a = 0.f, b = 0.f;
    BPF_TRY(cudaEventElapsedTime(&a, h->ev[3 * s], h->ev[3 * s + 1]));
    BPF_TRY(cudaEventElapsedTime(&b, h->ev[3 * s + 1], h->ev[3 * s + 2]));
    r += a;
    t += b;
  }
  if (resample_ms) *resample_ms = r;
  if (transition_ms) *transition_ms = t;
  if (steps) *steps = h->ev_steps;
  if (reset) h->ev_steps = 0;
  return BPF_OK;
}

// ---- stand-alone resampler ------------------------------------------------

int bpf_resampler_create(int kind, int max_n, int metropolis_steps, void* stream, bpf_resampler** out) {
  if (!out) return BPF_E_INVALID;
  *out = nullptr;
  if (kind < BPF_RESAMPLER_SYSTEMATIC || kind > BPF_RESAMPLER_METROPOLIS || max_n <= 0 || metropolis_steps < 0)
    return BPF_E_INVALID;
  bpf_resampler* r = new (std::nothrow) bpf_resampler();
  if (!r) return BPF_E_NOMEM;
  r->kind = kind;
  r->B = metropolis_steps;
  r->stream = (cudaStream_t)stream;
  int rc = bpf::scratch_alloc(r->rs, max_n);
  if (rc) { delete r; return rc; }
  *out = r;
  return BPF_OK;
}

int bpf_resampler_destroy(bpf_resampler* r) {
  if (!r) return BPF_OK;
  if (r->stream) cudaStreamSynchronize(r->stream); else cudaDeviceSynchronize();
  for (cudaEvent_t e : r->ev)
    if (e) cudaEventDestroy(e);
  bpf::scratch_free(r->rs);
  delete r;
  return BPF_OK;
}

static int reset_status(bpf_resampler* r) {
  k_set_status_ok<<<1, 1, 0, r->stream>>>(r->rs.stats, r->rs.counters);
  BPF_TRY(cudaGetLastError());
  return BPF_OK;
}

static int timing_begin(bpf_resampler* r) {
  if (r->timing) BPF_TRY(cudaEventRecord(r->ev[0], r->stream));
  return BPF_OK;
}

static int timing_end(bpf_resampler* r) {
  if (r->timing) BPF_TRY(cudaEventRecord(r->ev[1], r->stream));
  return BPF_OK;
}

// called after the stream has been synchronised
static int timing_collect(bpf_resampler* r) {
  if (!r->timing) return BPF_OK;
  float ms = 0.0f;
  BPF_TRY(cudaEventElapsedTime(&ms, r->ev[0], r->ev[1]));
  r->timed_ms += ms;
  r->timed_calls += 1;
  return BPF_OK;
}

static int read_rs_stats(bpf_resampler* r, bpf::StepStats* s) {
  BPF_TRY(cudaMemcpyAsync(s, r->rs.stats, sizeof(*s), cudaMemcpyDeviceToHost, r->stream));
  BPF_TRY(cudaStreamSynchronize(r->stream));
  return timing_collect(r);
}

int bpf_resampler_timing_enable(bpf_resampler* r, int enable) {
  if (!r) return BPF_E_INVALID;
  if (enable) {
    for (cudaEvent_t& e : r->ev)
      if (!e) BPF_TRY(cudaEventCreate(&e));
  }
  r->timing = enable != 0;
  return BPF_OK;
}

int bpf_resampler_timing_read(bpf_resampler* r, int reset, double* ms, int* calls) {
  if (!r) return BPF_E_INVALID;
  if (ms) *ms = r->timed_ms;
  if (calls) *calls = r->timed_calls;
  if (reset) { r->timed_ms = 0.0; r->timed_calls = 0; }
  return BPF_OK;
}

int bpf_autotune_resampler(int n, void* stream, bpf_tune_result* out) {
  if (n <= 0) return BPF_E_INVALID;
  int best = -1;
  double us[BPF_RESAMPLE_SHAPES];
  const int rc = bpf::autotune_systematic(n, (cudaStream_t)stream, &best, us);
  if (out) {
    out->shape = best;
    for (int k = 0; k < BPF_RESAMPLE_SHAPES; ++k) out->us[k] = us[k];
  }
  return rc;
}

int bpf_resampler_set_shape(bpf_resampler* r, int shape) {
  if (!r || shape < -1 || shape >= BPF_RESAMPLE_SHAPES) return BPF_E_INVALID;
  r->shape = shape;
  return BPF_OK;
}

int bpf_ess_reduce(bpf_resampler* r, const double* lw, int n, double* lW, double* ess) {
  if (!r || !lw || n <= 0 || n > r->rs.max_n) return BPF_E_INVALID;
  int rc = reset_status(r);
  if (rc) return rc;
  if ((rc = timing_begin(r))) return rc;
  rc = bpf::launch_lw_reduce(lw, n, r->rs, r->stream);
  if (rc) return rc;
  if ((rc = timing_end(r))) return rc;
  bpf::StepStats s;
  rc = read_rs_stats(r, &s);
  if (rc) return rc;
  if (lW) *lW = s.lW;
  if (ess) *ess = s.ess;
  return BPF_OK;
}

int bpf_logsumexp_reduce(bpf_resampler* r, const double* lw, int n, double* out) {
  if (!r || !lw || n <= 0 || n > r->rs.max_n) return BPF_E_INVALID;
  int rc = reset_status(r);
  if (rc) return rc;
  if ((rc = timing_begin(r))) return rc;
  rc = bpf::launch_logsumexp(lw, n, r->rs, r->stream);
  if (rc) return rc;
  if ((rc = timing_end(r))) return rc;
  bpf::StepStats s;
  rc = read_rs_stats(r, &s);
  if (rc) return rc;
  if (out) *out = s.lW;
  return BPF_OK;
}

int bpf_resampler_ancestors(bpf_resampler* r, const double* lw, int n, const double* uniforms, int permute,
                            int* as, int* Os) {
  if (!r || !lw || !as || n <= 0 || n > r->rs.max_n) return BPF_E_INVALID;
  int rc = reset_status(r);
  if (rc) return rc;
  bpf::ResampleArgs ra;
  ra.kind = r->kind;
  ra.n = n;
  ra.B = r->B;
  ra.lw = lw;
  ra.uniforms = uniforms;
  ra.seed = 0;
  ra.step = 0;
  ra.permute = permute;
  ra.as = as;
  ra.Os_out = Os;
  ra.gate = nullptr;
  ra.max_known = false;
  ra.shape = r->shape;
  if ((rc = timing_begin(r))) return rc;
  rc = bpf::launch_resample(ra, r->rs, r->stream);
  if (rc) return rc;
  if ((rc = timing_end(r))) return rc;
  bpf::StepStats s;
  rc = read_rs_stats(r, &s);
  if (rc) return rc;
  return s.status;
}

int bpf_debug_set_wait_limit(long long cycles) { return bpf::set_barrier_limit(cycles); }

int bpf_gather_rows(const int* as, const void* X, void* Y, int n, int d, int ld, int elem_size, void* stream) {
  if (!as || !X || !Y || X == Y) return BPF_E_INVALID;
  return bpf::launch_gather(as, X, Y, n, d, ld, elem_size, nullptr, (cudaStream_t)stream);
}

// ---- checkpoint ------------------------------------------------------------

struct SnapHeader {
  uint64_t magic;
  int n, ld, dim, esz, step, pad;
  bpf::StepStats stats;
};

static const uint64_t kSnapMagic = 0x3130304250464253ull;  // "SBFPB001"

int bpf_snapshot_size(bpf_handle* h, uint64_t* bytes) {
  if (!h || !bytes) return BPF_E_INVALID;
  *bytes = sizeof(SnapHeader) + (uint64_t)h->ld * h->dim * h->esz + (uint64_t)h->n * (sizeof(double) + sizeof(int));
  return BPF_OK;
}

int bpf_snapshot(bpf_handle* h, void* buf, uint64_t bytes) {
  uint64_t need;
  if (bpf_snapshot_size(h, &need) || !buf || bytes < need) return BPF_E_INVALID;
  SnapHeader hd;
  std::memset(&hd, 0, sizeof(hd));
  hd.magic = kSnapMagic;
  hd.n = h->n; hd.ld = h->ld; hd.dim = h->dim; hd.esz = h->esz; hd.step = h->step;
  int rc = read_stats(h, &hd.stats);
  if (rc) return rc;
  char* p = (char*)buf;
  std::memcpy(p, &hd, sizeof(hd));
  p += sizeof(hd);
  const size_t xb = (size_t)h->ld * h->dim * h->esz;
  BPF_TRY(cudaMemcpyAsync(p, h->x[h->cur], xb, cudaMemcpyDeviceToHost, h->stream));
  p += xb;
  BPF_TRY(cudaMemcpyAsync(p, h->lw, (size_t)h->n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  p += (size_t)h->n * sizeof(double);
  BPF_TRY(cudaMemcpyAsync(p, h->as, (size_t)h->n * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  BPF_TRY(cudaStreamSynchronize(h->stream));
  return BPF_OK;
}

int bpf_restore(bpf_handle* h, const void* buf, uint64_t bytes) {
  uint64_t need;
  if (bpf_snapshot_size(h, &need) || !buf || bytes < need) return BPF_E_INVALID;
  SnapHeader hd;
  std::memcpy(&hd, buf, sizeof(hd));
  if (hd.magic != kSnapMagic || hd.n != h->n || hd.ld != h->ld || hd.dim != h->dim || hd.esz != h->esz)
    return BPF_E_INVALID;
  const char* p = (const char*)buf + sizeof(hd);
  const size_t xb = (size_t)h->ld * h->dim * h->esz;
  h->cur = 0;
  BPF_TRY(cudaMemcpyAsync(h->x[0], p, xb, cudaMemcpyHostToDevice, h->stream));
  p += xb;
  BPF_TRY(cudaMemcpyAsync(h->lw, p, (size_t)h->n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  p += (size_t)h->n * sizeof(double);
  BPF_TRY(cudaMemcpyAsync(h->as, p, (size_t)h->n * sizeof(int), cudaMemcpyHostToDevice, h->stream));
  // no whole-filter run is in progress after a restore (the saved record
  // pointer may name a buffer freed since)
  hd.stats.hist = nullptr;
  hd.stats.hist_n = 0;
  BPF_TRY(cudaMemcpyAsync(h->rs.stats, &hd.stats, sizeof(hd.stats), cudaMemcpyHostToDevice, h->stream));
  {
    const int rc = bpf::reset_scratch_words(h->rs, h->stream);
    if (rc) return rc;
  }
  BPF_TRY(cudaStreamSynchronize(h->stream));
  h->step = hd.step;
  return BPF_OK;
}

}  // extern "C"
