/*
 * libbi_b200 — B200-native bootstrap particle-filter step, C ABI.
 *
 * This is the drop-in boundary for LibBi's bootstrap particle filter hot
 * path.  Each entry point names the reference interface it replaces
 * (paths are relative to the LibBi source tree).  All functions are
 * extern "C", take plain pointers and sizes, and return an int status
 * (BPF_OK or one of the BPF_E_* codes).  Pointers documented as "device"
 * are CUDA device pointers on the current device; "host" pointers are
 * ordinary host memory.  Work is enqueued on the stream given at creation
 * (or the legacy default stream when that is NULL); functions that return
 * scalars to the host synchronise that stream.
 *
 * Threading: one handle per host thread.  Handles never share buffers.
 */
#ifndef LIBBI_B200_H
#define LIBBI_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
enum {
  BPF_OK = 0,
  /* all weights zero or not finite when a resample was due; the reference
   * throws ParticleFilterDegeneratedException here
   * (share/src/bi/resampler/SystematicResampler.hpp:127-129,
   *  share/src/bi/misc/exception.hpp:47) */
  BPF_E_DEGENERATE = 1,
  BPF_E_INVALID = 2,   /* bad argument (size, kind, null pointer) */
  BPF_E_CUDA = 3,      /* a CUDA runtime call failed */
  BPF_E_TIMEOUT = 4,   /* a bounded device-side wait gave up */
  BPF_E_NOMEM = 5,     /* device allocation failed */
  BPF_E_TOO_LARGE = 6  /* n exceeds BPF_STATIC_MAX_PARTICLES (bpf_systematic_ancestors_static) */
};

/* ---- model description ------------------------------------------------ */
/* The two models of the hot path.  LibBi compiles each .bi model into a
 * Model<Name> class (share/tt/cpp/model.hpp.tt:95-510); here the model's
 * transition and observation blocks are built into the library and chosen
 * by kind, with the .bi model's constants passed in theta. */
enum {
  /* Lorenz '96, d components (docs/src/users.tex:354-358):
   *   transition(delta) { eta[i] ~ gaussian(0, sigma_eta);
   *                       ode(alg='RK4', h) { dx[i]/dt = (x[i+1]-x[i-2])*x[i-1] - x[i] + F }
   *                       x[i] <- x[i] + eta[i] }
   *   observation       { y[i] ~ gaussian(x[i], sigma_y) }
   *   initial           { x[i] ~ gaussian(x0_mean, x0_std) }
   * theta = { F, sigma_eta, sigma_y, x0_mean, x0_std } */
  BPF_MODEL_L96 = 1,
  /* Phytoplankton-zooplankton (docs/src/users.tex:40-84):
   *   transition(delta) { alpha ~ log_normal(mu, sigma);
   *                       ode(alg='RK4(3)', h, atoler, rtoler) {
   *                         dP/dt = alpha*P - c*P*Z
   *                         dZ/dt = e*c*P*Z - m*Z - q*Z*Z } }
   *   observation       { y ~ gaussian(log(P), sigma_y) }
   *   initial           { P ~ log_normal(p0_mu, p0_sigma); Z ~ log_normal(z0_mu, z0_sigma) }
   * theta = { c, e, m, q, mu, sigma, sigma_y, p0_mu, p0_sigma, z0_mu, z0_sigma } */
  BPF_MODEL_PZ = 2
};

enum { BPF_ODE_RK4 = 0, BPF_ODE_RK43 = 1 };
enum { BPF_F32 = 0, BPF_F64 = 1 };

#define BPF_MAX_THETA 16

typedef struct {
  int kind;        /* BPF_MODEL_* */
  int dim;         /* state components: d for L96 (4, 8, 16, 32 or 40), 2 for PZ */
  int precision;   /* BPF_F32 or BPF_F64: state, ODE and log-density arithmetic
                      (L96: either; PZ: BPF_F64) */
  int integrator;  /* BPF_ODE_RK4 or BPF_ODE_RK43 (ode block 'alg') */
  double h;        /* ode block 'h' (RK4 step / RK4(3) initial step) */
  double atoler;   /* ode block 'atoler' (RK4(3) only) */
  double rtoler;   /* ode block 'rtoler' (RK4(3) only) */
  double theta[BPF_MAX_THETA];
} bpf_model_desc;

/* ---- filter configuration --------------------------------------------- */
/* Resampler kinds: share/src/bi/resampler/ResamplerFactory.cpp:8-39 */
enum {
  BPF_RESAMPLER_SYSTEMATIC = 0,
  BPF_RESAMPLER_MULTINOMIAL = 1,
  BPF_RESAMPLER_METROPOLIS = 2
};

typedef struct {
  int nparticles;        /* N (--nparticles) */
  int resampler;         /* BPF_RESAMPLER_* (--resampler) */
  int metropolis_steps;  /* B (--C), Metropolis only */
  double ess_rel;        /* resample when ESS < ess_rel*N (--ess-rel) */
  uint64_t seed;         /* --seed */
  void* stream;          /* cudaStream_t, or NULL for the default stream */
} bpf_config;

/* Output of one filter step: the fields of BootstrapPFState / FilterState
 * that BootstrapPF::correct updates (share/src/bi/filter/BootstrapPF.hpp:171-181). */
typedef struct {
  double ess;             /* s.ess */
  double log_weight_sum;  /* lW = max + log sum exp(lw - max) - log N */
  double log_increment;   /* s.logIncrements(k) = lW - previous logLikelihood */
  double log_likelihood;  /* s.logLikelihood */
  int resampled;          /* Resampler::resample returned true before this step's predict */
  int status;             /* device-side status (BPF_OK, BPF_E_DEGENERATE, BPF_E_TIMEOUT) */
} bpf_step_out;

typedef struct bpf_handle bpf_handle;

/* Create a filter: State + BootstrapPFState + Resampler + RNG for one model.
 * Replaces the construction in the generated filter client
 * (share/tt/cpp/client/filter_cpu.cpp.tt:105-184): BootstrapPFState(N),
 * ResamplerFactory::create*, Random(seed), BootstrapPF(m, in, obs, resam). */
int bpf_create(const bpf_model_desc* model, const bpf_config* config, bpf_handle** out);

/* Release all device memory of the handle. */
int bpf_destroy(bpf_handle* h);

/* The form of a step (no counterpart in the reference, whose step is a
 * sequence of host calls).  By default a step is two launches: the
 * resampler, then the transition as its programmatic dependent.  For the
 * built-in Lorenz-96 model with the systematic resampler, when the GPU
 * holds all of the step's blocks at once, bpf_set_step_form(h, 1) selects
 * the fused form instead: one launch per step, the resampling (when due) as
 * the transition kernel's prologue over the transition's blocks.  Both
 * forms compute the same ancestors, states and weights bit for bit.  On a
 * B200 at N = 65536 (d = 40, FP32) the fused form measured 0.065 ms per
 * step against 0.048 ms: its hand-overs run across 512 blocks of 128
 * threads, the resampler's across 64 blocks of 1024.
 * bpf_set_step_form(h, 0) selects the two-launch form; (h, 1) the fused
 * one (BPF_E_INVALID where it is not available). */
int bpf_set_step_form(bpf_handle* h, int fused);
int bpf_step_form(bpf_handle* h, int* fused);

/* ---- models compiled outside the library ------------------------------- */
/* LibBi generates a Model class per .bi file and instantiates the filter
 * templates on it (share/tt/cpp/model.hpp.tt:95-510; the block updaters of
 * share/tt/cpp/block/ode.hpp.tt:39-54 and pdf_.hpp.tt:46-75, which call
 * RK4Integrator<B,S>::update, RK43Integrator<B,S>::update,
 * StaticSampler<B,S>::samples and SparseStaticLogDensity<B,S>::logDensities).
 * A model class of that shape, compiled by the caller with nvcc against
 * include/bpf_model.cuh, yields this table of launchers (bpf::model_ops<B>),
 * and the library's filter drives it exactly as it drives its built-in
 * models: resampling, the log-weight reduction, steps, checkpoints and path
 * output are the library's.  The launchers enqueue on `stream` and return
 * BPF_OK, BPF_E_INVALID or BPF_E_CUDA. */
typedef struct {
  const void* x_in;   /* state before the step: dim columns, SoA, leading dimension ld */
  void* x_out;        /* state after the step */
  int ld, n;
  int* ancestors;     /* read (gather) and rewritten when the step resamples */
  double* lw;         /* FP64 log-weights, updated in place */
  const void* y;      /* device observation (nobs values) or NULL (unobserved step) */
  uint64_t obs_mask;  /* bit j: observed element j (every bit set for a full observation) */
  double t1, t2;
  uint64_t seed;
  int step;           /* schedule index of the observation (random stream address) */
  const double* params;  /* host, nparams values: the model's parameters */
  int nparams;
  void* stats;        /* the step statistics the kernel's last block finalises (bpf_device.cuh) */
  void* partials;     /* one bpf::LwPartial per block */
  int max_partials;   /* capacity of partials */
  unsigned* counter;  /* last-block ticket, zero on entry and on exit */
} bpf_transition_args;

typedef struct {
  void* x;            /* state to draw: dim columns, SoA, leading dimension ld */
  int ld, n;
  double* lw;         /* set to zero */
  uint64_t seed;
  const double* params;
  int nparams;
} bpf_init_args;

typedef struct {
  int dim;            /* state columns per particle (D_VAR then DX_VAR elements) */
  int nobs;           /* observed elements per observation, at most 64 */
  int nparams;        /* parameters (P_VAR elements) */
  int precision;      /* BPF_F32 or BPF_F64: the state and observation type */
  int (*init)(const bpf_init_args* a, void* stream);
  int (*transition)(const bpf_transition_args* a, void* stream);
} bpf_model_ops;

/* bpf_create for a model compiled outside the library: ops from
 * bpf::model_ops<Model>() (include/bpf_model.cuh), params the model's
 * nparams parameter values (host; copied).  The handle supports every
 * single-filter entry point except bpf_set_proposal.  Replaces the same
 * construction as bpf_create (share/tt/cpp/client/filter_cpu.cpp.tt:105-184)
 * for a model LibBi would generate. */
int bpf_create_model(const bpf_model_ops* ops, const double* params, const bpf_config* config, bpf_handle** out);

/* Device pointers of the particle store.  x: structure of arrays, component j
 * of particle p at x[j*ld + p] in the model precision (State Xdn, column-major,
 * share/src/bi/state/State.hpp:73-462); lw: N log-weights in FP64
 * (BootstrapPFState::logWeights); as: N ancestors (BootstrapPFState::ancestors).
 * The pointers stay valid until the next bpf_step / bpf_gather, which
 * alternate between two state buffers. */
int bpf_state_ptrs(bpf_handle* h, void** x, double** lw, int** as, int* ld);

/* Simulator::init for the filter: draw initial particles from the model's
 * initial block, clear log-weights, logLikelihood and ess
 * (share/src/bi/simulator/Simulator.hpp:255-332, Filter::filter
 * share/src/bi/filter/Filter.hpp:58-70). */
int bpf_init(bpf_handle* h);

/* One BootstrapPF::step from t1 to the observation at t2
 * (share/src/bi/filter/BootstrapPF.hpp:158-181): resample if the previous
 * schedule element was observed and ESS < ess_rel*N (Resampler::resample,
 * share/src/bi/resampler/Resampler.hpp:167-182), predict with
 * Model::transitionSamples (share/tt/cpp/model.hpp.tt:566-573), then correct
 * with Model::observationLogDensities (model.hpp.tt:757-765) and
 * Resampler::reduce.  y: host pointer to the step's observations in the
 * model precision (L96: dim values; PZ: 1 value), or NULL for an unobserved
 * step.  out may be NULL (no sync; y in pinned memory must then stay
 * unchanged until the stream has reached the step). */
int bpf_step(bpf_handle* h, double t1, double t2, const void* y, bpf_step_out* out);

/* bpf_step with only some components observed: the observation Mask of
 * Observer::getMask / SparseStaticLogDensity (share/src/bi/state/Mask.hpp:26-203,
 * share/src/bi/simulator/Observer.hpp:97-126).  y: host, nidx values in the
 * model precision for the components idx[0..nidx) (distinct, < 64); nidx = 0
 * is an unobserved step.  A filter with a learned proposal proposes from the
 * transition on such steps. */
int bpf_step_sparse(bpf_handle* h, double t1, double t2, const void* y, const int* idx, int nidx,
                    bpf_step_out* out);

/* bpf_step with the observation already in device memory (or NULL): no
 * host-to-device copy is enqueued. */
int bpf_step_device(bpf_handle* h, double t1, double t2, const void* y_device, bpf_step_out* out);

/* Filter<BootstrapPF>::filter over T observations at t0+dt, ..., t0+T*dt
 * (share/src/bi/filter/Filter.hpp:58-70 with BootstrapPF::term :192-196).
 * y: host, T observations (L96: dim values each; PZ: 1) in the model
 * precision, observation-major.
 * Outputs (host, may be NULL): log_increments[T], ess[T], and the final
 * log-likelihood.  Calls bpf_init first. */
int bpf_filter(bpf_handle* h, int T, double t0, double dt, const void* y,
               double* log_increments, double* ess, double* log_likelihood);

/* Resampler<R>::reduce over the handle's log-weights
 * (share/src/bi/resampler/Resampler.hpp:156-163 -> ess_reduce,
 *  share/src/bi/primitive/vector_primitive.hpp:960-974). */
int bpf_reduce(bpf_handle* h, double* lW, double* ess);

/* Force one resample of the handle's state now (the ancestors, gather and
 * log-weight reset of Resampler::resample, Resampler.hpp:170-177), whatever
 * the ESS.  uniforms: optional DEVICE pointer to the resampler's uniforms
 * (systematic: 1; multinomial: N in the reference's draw order; Metropolis:
 * 2*B*N, particle-major) to replace the handle's own draws.  ancestors_out:
 * optional device pointer receiving the N permuted ancestors. */
int bpf_resample(bpf_handle* h, const double* uniforms, int* ancestors_out);

/* Device timing of the steps (the reference's TicToc around Filter::filter,
 * share/src/bi/misc/TicToc.hpp:17-70, at kernel granularity): when enabled,
 * every step records CUDA events before its resample kernels, between them
 * and the fused transition, and after it.  bpf_timing_read synchronises the
 * stream and returns the summed milliseconds and the number of steps since
 * the last reset. */
int bpf_timing_enable(bpf_handle* h, int enable);
int bpf_timing_read(bpf_handle* h, int reset, double* resample_ms, double* transition_ms, int* steps);

/* Path output (BootstrapPFCache::writeState + AncestryCache,
 * share/src/bi/cache/BootstrapPFCache.hpp:182-210; BootstrapPF::samplePath,
 * share/src/bi/filter/BootstrapPF.hpp:148-154).  bpf_path_cache records up
 * to max_steps steps (0 stops recording) and starts the record from the
 * current state; every later step (and bpf_init, which restarts the record)
 * appends the new particles with their ancestors.  The record is pruned as
 * AncestryCache prunes it (share/src/bi/cuda/cache/AncestryCacheKernel.cuh:
 * 29-48): only particles with a line to the current generation keep their
 * node, so device memory follows the particles' genealogy (about N nodes
 * plus the distinct ancestors of each past generation), not steps x N.  A
 * recording step synchronises the stream once. */
int bpf_path_cache(bpf_handle* h, int max_steps);
/* Nodes the path record holds and the capacity of its pool (AncestryCache::
 * report, share/src/bi/cache/AncestryCache.hpp:455-466); synchronises. */
int bpf_path_cache_nodes(bpf_handle* h, int* nodes, int* capacity);
/* samplePath: p ~ multinomial(exp(lw)) over the current log-weights
 * (RngHost::multinomial, share/src/bi/host/random/RngHost.hpp:120-139) from
 * one uniform (u: device pointer, or NULL for the handle's own draw), then
 * the state path of p back through the recorded ancestors
 * (AncestryCache::readPath, share/src/bi/cache/AncestryCache.hpp:294-311).
 * path: host, len x dim in the model precision, oldest first; particle and
 * len: host.  BPF_E_TOO_LARGE when more steps were taken than the cache
 * holds. */
int bpf_sample_path(bpf_handle* h, const double* u, void* path, int* particle, int* len);

/* ---- stand-alone primitives (the Resampler<R> and gather APIs) -------- */

typedef struct bpf_resampler bpf_resampler;

/* Resampler<R>(essRel) with scratch for up to max_n particles
 * (share/src/bi/resampler/Resampler.hpp:125-132; B as MetropolisResampler(B),
 *  share/src/bi/resampler/MetropolisResampler.hpp:201-204). */
int bpf_resampler_create(int kind, int max_n, int metropolis_steps, void* stream,
                         bpf_resampler** out);
int bpf_resampler_destroy(bpf_resampler* r);

/* ess_reduce (vector_primitive.hpp:960-974): device lw[n] (FP64);
 * returns ESS and lW = max + log sum exp(lw-max) - log n through host pointers. */
int bpf_ess_reduce(bpf_resampler* r, const double* lw, int n, double* lW, double* ess);

/* logsumexp_reduce (vector_primitive.hpp:933-943), used by BootstrapPF::term. */
int bpf_logsumexp_reduce(bpf_resampler* r, const double* lw, int n, double* out);

/* R::ancestors / R::ancestorsPermute on device lw[n]:
 *  systematic  SystematicResampler.hpp:132-148 (+ ScanResampler::precompute,
 *              ScanResampler.hpp:35-40; cumulativeOffspring :111-130);
 *              uniforms: 1 value, the offset a;
 *  multinomial MultinomialResamplerHost::ancestors (sorted, Bentley & Saxe),
 *              share/src/bi/host/resampler/MultinomialResamplerHost.hpp:29-65;
 *              uniforms: n values in the reference's draw order;
 *  metropolis  MetropolisResamplerHost::ancestors,
 *              share/src/bi/host/resampler/MetropolisResamplerHost.hpp:32-62;
 *              uniforms: 2*B*n values, particle-major.
 * uniforms and as are DEVICE pointers.  permute = 0 gives R::ancestors,
 * permute = 1 gives the permuted form: every particle with offspring is its
 * own first offspring (as[i] == i) and the remaining copies, ordered by
 * ancestor, fill the childless slots in ascending order — the rule of
 * ResamplerHost::cumulativeOffspringToAncestorsPermute
 * (share/src/bi/host/resampler/ResamplerHost.hpp:134-168).
 * Os (optional, device, n ints) receives the cumulative offspring counts.
 * Returns BPF_E_DEGENERATE when the weights sum to zero or are not finite. */
int bpf_resampler_ancestors(bpf_resampler* r, const double* lw, int n,
                            const double* uniforms, int permute, int* as, int* Os);

/* Device timing of a resampler's compute kernels, the counterpart of
 * bpf_timing_enable for the stand-alone primitives: when enabled, every
 * bpf_ess_reduce, bpf_logsumexp_reduce and bpf_resampler_ancestors call
 * records CUDA events around its kernels (not around the status reset or the
 * read-back of the results), and bpf_resampler_timing_read returns the summed
 * milliseconds and the number of timed calls since the last reset. */
int bpf_resampler_timing_enable(bpf_resampler* r, int enable);
int bpf_resampler_timing_read(bpf_resampler* r, int reset, double* ms, int* calls);

/* Autotuner of the one-launch systematic resampler (no counterpart in the
 * reference): tile shapes of threads per block x particles per thread
 * (0: 256 x 2, 1: 128 x 4, 2: 512 x 1, 3: 512 x 2, 4: 256 x 4,
 * 5: 1024 x 1), all computing the same ancestors.  bpf_autotune_resampler
 * times every shape that fits the GPU in one wave on seeded synthetic
 * log-weights of n particles (on `stream`, which it synchronises; not
 * while the stream is being captured) and keeps the fastest for n's size
 * class (the next power of two) on the current device for the rest of the
 * process; bpf_create runs it for its N.  out (may be NULL) receives the
 * chosen shape and each shape's median microseconds (0: does not fit). */
#define BPF_RESAMPLE_SHAPES 6
typedef struct {
  int shape;
  double us[BPF_RESAMPLE_SHAPES];
} bpf_tune_result;
int bpf_autotune_resampler(int n, void* stream, bpf_tune_result* out);
/* Pin the shape a stand-alone resampler uses (-1: the autotuned shape, else
 * shape 0); a shape that does not fit in one wave falls back to one that
 * does. */
int bpf_resampler_set_shape(bpf_resampler* r, int shape);

/* Diagnostic hook, no counterpart in the reference (its resamplers have no
 * device-side waits).  Every wait of the cooperative systematic resampler
 * for the other blocks (a grid-wide barrier, or the poll of the other
 * blocks' published words) lasts at most `cycles` SM clock cycles on the
 * current device (BPF_WAIT_LIMIT_DEFAULT, about 2 s, unless changed); a
 * block that gives up records BPF_E_TIMEOUT and its kernel returns.  A
 * negative value makes a block give up at the first wait that finds the
 * others not yet there (a barrier still closed; and every poll, whatever it
 * finds), so that a test can take the timeout path without a kernel that
 * never arrives.  The next status reset (each stand-alone resampler call,
 * bpf_init, bpf_restore) clears the barrier state the abandoned launch left
 * and moves the resampler's epoch on, so that nothing the abandoned launch
 * published is taken for a later launch's. */
#define BPF_WAIT_LIMIT_DEFAULT 4000000000LL
int bpf_debug_set_wait_limit(long long cycles);

/* gather_rows (share/src/bi/primitive/matrix_primitive.hpp:630-638,
 * share/src/bi/cuda/primitive/matrix_primitive_kernel.cuh:50-57), out of
 * place on device SoA buffers: Y[j*ld + i] = X[j*ld + as[i]], j < d, i < n.
 * elem_size is 4 or 8. */
int bpf_gather_rows(const int* as, const void* X, void* Y, int n, int d, int ld,
                    int elem_size, void* stream);

/* Systematic resampling that allocates nothing.  No counterpart in the
 * reference: this entry point exists for callers that cannot let the library
 * allocate device memory, such as an application that has reserved the GPU's
 * memory up front for its own allocator, or a real-time loop in which a
 * cudaMalloc (which may synchronise the device) is not allowed.  It computes
 * exactly what bpf_resampler_ancestors computes for a systematic resampler
 * (same arguments: device lw[n], optional device offset a, permute, device
 * as[n], optional device Os[n]; work on `stream`), but its scratch is one
 * fixed-size __device__ array inside the library (under 1 MiB, held on every
 * GPU that loads the library until the process exits), so n may be at most
 * BPF_STATIC_MAX_PARTICLES; larger n returns BPF_E_TOO_LARGE.  The first call
 * on each device looks up that array's address; make it before any stream
 * capture.  The address is kept for the life of the process: after a
 * cudaDeviceReset the array may move, so this entry point must not be used
 * again in that process.  All calls share the array, so calls that overlap
 * on the GPU race and must be ordered by the caller.  Synchronises `stream`
 * and returns
 * BPF_E_DEGENERATE when the weights sum to zero or are not finite. */
#define BPF_STATIC_MAX_PARTICLES 65536
int bpf_systematic_ancestors_static(const double* lw, int n, const double* a, int permute, int* as, int* Os,
                                    void* stream);

/* ---- batched filters --------------------------------------------------- */
/* Many independent filters of one model advanced together: one launch per
 * phase (resample, transition) for the whole batch, and bpf_filter_batch runs
 * init + T steps as one captured CUDA graph.  The reference runs such filters
 * one Filter<BootstrapPF>::filter at a time, e.g. per iteration of
 * MarginalMH (share/src/bi/sampler/MarginalMH.hpp:230-271) or per parameter
 * particle of MarginalSIR (share/src/bi/sampler/MarginalSIR.hpp:283-420).
 * Filter f of a batch draws exactly what a single filter (bpf_create) with
 * the same particle count, resampler, seed and theta draws, so it reproduces
 * that filter's log-likelihood increments. */
#define BPF_BATCH_MAX_PARTICLES 32768

typedef struct {
  int nparticles;        /* N of this filter, 1 .. BPF_BATCH_MAX_PARTICLES */
  int resampler;         /* BPF_RESAMPLER_* */
  int metropolis_steps;  /* B, Metropolis only */
  uint64_t seed;
  double theta[BPF_MAX_THETA];  /* this filter's model constants (bpf_model_desc.theta) */
} bpf_batch_filter;

typedef struct bpf_batch bpf_batch;

/* model gives kind, dim, precision, integrator and h/atoler/rtoler shared by
 * every filter; filters[nfilters] the per-filter settings; ess_rel as in
 * bpf_config.  stream: cudaStream_t, or NULL for a library-owned blocking
 * stream.  Draws the initial particles (bpf_batch_init). */
int bpf_batch_create(const bpf_model_desc* model, int nfilters, const bpf_batch_filter* filters, double ess_rel,
                     void* stream, bpf_batch** out);
int bpf_batch_destroy(bpf_batch* b);
/* Simulator::init for every filter of the batch (see bpf_init). */
int bpf_batch_init(bpf_batch* b);
/* Replace every filter's theta (host, nfilters x BPF_MAX_THETA), e.g. a PMMH
 * proposal; takes effect from the next step or filter run. */
int bpf_batch_set_theta(bpf_batch* b, const double* theta);
/* Replace every filter's seed (host, nfilters), e.g. fresh randomness for
 * each filter run of a PMMH iteration; takes effect from the next init. */
int bpf_batch_set_seeds(bpf_batch* b, const uint64_t* seeds);
/* Threads per filter CTA of the batched resampler (256, 512 or 1024; no
 * counterpart in the reference).  bpf_batch_create autotunes it: the three
 * counts are timed on synthetic log-weights laid out as the batch's filters
 * and the fastest is kept; every count computes the same ancestors.
 * threads != 0 pins a count (a captured filter run is recaptured); current
 * and tuned_us[3] (the tuning medians for 256, 512, 1024; may be NULL)
 * report the state. */
int bpf_batch_resample_threads(bpf_batch* b, int threads, int* current, double* tuned_us);
/* One BootstrapPF::step of every filter (see bpf_step); y_device: device
 * observations, nfilters x (dim for L96, 1 for PZ), filter-major, in the
 * model precision, or NULL for an unobserved step.  Does not synchronise. */
int bpf_batch_step_device(bpf_batch* b, double t1, double t2, const void* y_device);
/* Host copies of every filter's logLikelihood (-inf after a degenerate
 * resample), ESS and status; returns the first non-OK status, if any. */
int bpf_batch_stats(bpf_batch* b, double* log_likelihoods, double* ess, int* status);
/* Device pointers of the shared buffers: filter f's particle p, component j
 * at x[j*ld + offsets[f] + p]; log-weights lw[offsets[f] + p]; ancestors
 * (filter-local indices) as[offsets[f] + p].  offsets: host, nfilters. */
int bpf_batch_state_ptrs(bpf_batch* b, void** x, double** lw, int** as, int* ld, int* offsets);
/* Filter<BootstrapPF>::filter for every filter over T observations at
 * t0+dt, ..., t0+T*dt: bpf_batch_init and T steps.  y: host, T x nfilters x
 * (dim or 1) in the model precision, step-major then filter-major.  Outputs
 * (host, may be NULL): log_likelihoods[nfilters] (BootstrapPF::term),
 * log_increments[T*nfilters] and ess[T*nfilters] (step-major),
 * status[nfilters].  The init and steps run as one CUDA graph, captured on
 * the first call and replayed while T, t0 and dt stay the same.  Returns the
 * first non-OK filter status, if any (the other filters' outputs are valid). */
int bpf_filter_batch(bpf_batch* b, int T, double t0, double dt, const void* y, double* log_likelihoods,
                     double* log_increments, double* ess, int* status);

/* Device timing of a batch: when enabled, bpf_batch_step_device times its
 * kernels and bpf_filter_batch its graph launch (init + T steps; not the
 * observation upload or the read-back) with CUDA events; these calls then
 * wait for the timed work.  bpf_batch_timing_read returns the summed
 * milliseconds and steps since the last reset. */
int bpf_batch_timing_enable(bpf_batch* b, int enable);
int bpf_batch_timing_read(bpf_batch* b, int reset, double* ms, int* steps);

/* ---- particle-marginal Metropolis-Hastings over many chains ------------ */
/* MarginalMH (share/src/bi/sampler/MarginalMH.hpp:190-271) for C chains at
 * once: every iteration proposes a Gaussian random-walk move of the sampled
 * entries of theta for each chain, filters all C proposals as one batch
 * (bpf_filter_batch) and accepts or rejects each chain with
 * min(1, exp(loglr + logpr)).  Proposals outside the prior's support are
 * rejected without a filter run for them; a degenerate filter gives
 * logLikelihood -inf (MarginalMH::propose). */
enum { BPF_PRIOR_UNIFORM = 0, BPF_PRIOR_LOG_NORMAL = 1, BPF_PRIOR_GAUSSIAN = 2 };

typedef struct {
  int index;    /* the entry of theta this parameter is */
  int prior;    /* BPF_PRIOR_UNIFORM (a, b = bounds), _LOG_NORMAL or _GAUSSIAN (a, b = mu, sigma) */
  double a, b;
  double step;  /* standard deviation of the random-walk proposal */
} bpf_pmmh_param;

typedef struct {
  int nchains;
  int nparticles;        /* per filter, at most BPF_BATCH_MAX_PARTICLES */
  int resampler;         /* BPF_RESAMPLER_* */
  int metropolis_steps;
  double ess_rel;
  uint64_t seed;         /* proposals, acceptance and filter seeds derive from it */
  int nparams;
  bpf_pmmh_param params[BPF_MAX_THETA];
  const int* chain_nparticles;  /* optional (host, nchains values, each 1 .. BPF_BATCH_MAX_PARTICLES):
                                   each chain's filter size; NULL: nparticles for every chain */
} bpf_pmmh_config;

typedef struct bpf_pmmh bpf_pmmh;

/* y: host, T observations (dim values for L96, 1 for PZ) at t0+dt, ...,
 * t0+T*dt, the same for every chain.  theta0: host, nchains x nparams
 * initial values, or NULL to draw them from the priors; the other entries of
 * theta come from model->theta.  Runs the initial filter of every chain
 * (MarginalMH::init). */
int bpf_pmmh_create(const bpf_model_desc* model, const bpf_pmmh_config* cfg, int T, double t0, double dt,
                    const void* y, const double* theta0, void* stream, bpf_pmmh** out);
int bpf_pmmh_destroy(bpf_pmmh* s);
/* Run `iterations` MH iterations of every chain.  Outputs (host, may be
 * NULL), per iteration i and chain c: samples[(i*C + c)*nparams + j] (the
 * chain's state after the iteration), log_likelihoods[i*C + c],
 * log_priors[i*C + c], proposal_log_likelihoods[i*C + c] (the proposal's
 * filter estimate, -inf when not filtered); accepted[c]: accepted moves so
 * far, counting the initial state as MarginalMH does. */
int bpf_pmmh_run(bpf_pmmh* s, int iterations, double* samples, double* log_likelihoods, double* log_priors,
                 double* proposal_log_likelihoods, int* accepted);
/* Current state: theta[c*nparams + j], logLikelihood and logPrior per chain,
 * and the number of filter runs so far (the next run index). */
int bpf_pmmh_state(bpf_pmmh* s, double* theta, double* log_likelihoods, double* log_priors, int* runs);
typedef struct bpf_proposal bpf_proposal;
/* Run every later filter of the chains as a guided filter with the learned
 * proposal p (NULL: back to the bootstrap filter); the proposal is owned by
 * the caller and must outlive its use.  No counterpart in the reference,
 * whose MarginalMH filters with the bootstrap filter. */
int bpf_pmmh_set_proposal(bpf_pmmh* s, bpf_proposal* p);

/* ---- SMC^2 over the batched filter -------------------------------------- */
/* MarginalSIR (share/src/bi/sampler/MarginalSIR.hpp:283-480): ntheta
 * parameter particles from the priors, each with a filter of nparticles; at
 * every observation the filters step together and each parameter particle's
 * log-weight grows by its filter's log-likelihood increment; when the
 * weights' ESS falls below theta_ess_rel * ntheta they are resampled
 * (systematic) and each makes `moves` PMMH moves (a random-walk proposal
 * filtered over the observations so far, MarginalMH's accept/reject).
 * After a resample-move round the filters replay the observations so far
 * from their (parameters, seed) pairs, which reproduces every
 * log-likelihood exactly.  Seeds: see libbi_b200/csrc/smc2.cu. */
typedef struct {
  int ntheta;             /* parameter particles */
  int nparticles;         /* per filter, at most BPF_BATCH_MAX_PARTICLES */
  int resampler;          /* the filters' BPF_RESAMPLER_* */
  int metropolis_steps;
  double ess_rel;         /* the filters' essRel */
  double theta_ess_rel;   /* resample the parameter particles when ESS < theta_ess_rel * ntheta */
  int moves;              /* PMMH moves per parameter particle after a resample */
  uint64_t seed;
  int nparams;
  bpf_pmmh_param params[BPF_MAX_THETA];  /* priors and random-walk steps */
} bpf_smc2_config;

/* y: host, T observations (dim values for L96, 1 for PZ) at t0+dt, ...,
 * t0+T*dt.  Outputs (host, may be NULL): theta_out[ntheta*nparams] and
 * log_weights[ntheta] after the last observation,
 * log_evidence_increments[T] (the marginal likelihood's log increments),
 * resample_steps (parameter resamples), acceptance (of the PMMH moves). */
int bpf_smc2_run(const bpf_model_desc* model, const bpf_smc2_config* cfg, int T, double t0, double dt,
                 const void* y, void* stream, double* theta_out, double* log_weights,
                 double* log_evidence_increments, int* resample_steps, double* acceptance);

/* ---- tensor-core dense layer (the learned proposal's arithmetic) ------- */
/* No counterpart in the reference.  D[m, n] = act(sum_k A(m,k) B(n,k) +
 * bias[n]) for m < M, n < N <= 256, on the sm_100a tensor cores (tcgen05,
 * BF16 operands, FP32 accumulation in tensor memory).  A(m,k) =
 * A[m*a_rs + k*a_cs] and B(n,k) = B[n*b_rs + k*b_cs] (device, BF16), so
 * transposed operands need no copy; bias: device, N floats, or NULL; relu:
 * 0 or 1; Df (FP32, row stride df_rs) and/or Dh (BF16, row stride dh_rs)
 * receive D; err: device int set to 1 if a bounded wait gave up.  Enqueued
 * on `stream`; does not synchronise. */
int bpf_dense_bf16(const void* A, long long a_rs, long long a_cs, const void* B, long long b_rs, long long b_cs,
                   int M, int N, int K, const float* bias, int relu, float* Df, long long df_rs, void* Dh,
                   long long dh_rs, int* err, void* stream);

/* ---- learned proposal (Lorenz-96, d = 40, FP32) ------------------------ */
/* No counterpart in the reference, whose bootstrap filter proposes from the
 * transition.  A small network proposes
 *   x_{t+1} ~ N(m(x_t) + delta, diag(exp(2 s))),  (delta, s) = MLP([x_t, y_{t+1} - m(x_t)]),
 * m the model's deterministic RK4 step over dt (the observation enters
 * through its innovation); input standardised with the training data's
 * statistics, two hidden layers of 128 ReLU units, BF16
 * weights and activations on the tensor cores (bpf_dense_bf16), FP32
 * accumulation, FP32 master weights trained by Adam on the Gaussian negative
 * log-likelihood of x_{t+1}.  A filter with a proposal attached
 * (bpf_set_proposal) weights each particle by p(y|x') p(x'|x) / q(x'|x, y),
 * so its likelihood estimate stays unbiased. */
/* bpf_proposal: declared with the PMMH entry points above */

/* model: L96, dim 40, BPF_F32 (F = theta[0], sigma_eta = theta[1], h), or
 * PZ, BPF_F64, RK4(3) (a proposal over the log-noise: bpf_proposal_set_states);
 * dt: the observation interval; max_batch: the largest training batch
 * (>= 128).  The untrained proposal is close to the transition itself. */
int bpf_proposal_create(const bpf_model_desc* model, double dt, int max_batch, uint64_t seed, void* stream,
                        bpf_proposal** out);
int bpf_proposal_destroy(bpf_proposal* p);
/* Training triples (device, n x 40 each, row-major, kept by the caller while
 * training): x_t, x_{t+1} simulated from x_t by the model, y_{t+1} observed
 * from x_{t+1}.  Computes the RK4 means and the input standardisation. */
int bpf_proposal_set_data(bpf_proposal* p, const float* x_t, const float* x_t1, const float* y_t1, int n);
/* The plankton model's proposal (model: PZ, FP64, RK4(3)): the network
 * proposes each particle's log-noise, log alpha ~ N(mu + delta, exp(2 s))
 * with (delta, s) = MLP([log P, log Z, y_{t+1} - log P]) (3 inputs, two
 * hidden layers of 128, 2 outputs; the untrained proposal is the prior
 * N(mu, sigma)).  Training rows are simulated from the states x_t (device,
 * n x 2 row-major FP64, e.g. particles of a run): for each row the
 * transition's log-noise from its prior, the ODE over dt and an observation
 * (tag BPF_RNG_DATA of the proposal's seed); the network learns the
 * log-noise from the state and the observation (bpf_proposal_train).  A
 * proposal for PZ attaches to batches (bpf_batch_set_proposal,
 * bpf_pmmh_set_proposal); their guided step weights each particle by
 * p(y | x') p(log alpha) / q(log alpha). */
int bpf_proposal_set_states(bpf_proposal* p, const double* x_t, int n);
/* `steps` Adam steps on minibatches of `batch` rows drawn with replacement
 * (counter-based stream of the seed), learning rate lr after a linear
 * warm-up over 5% of the steps and decaying by a cosine to lr/10;
 * loss_trace (host, may be NULL) gets each step's mean loss. */
int bpf_proposal_train(bpf_proposal* p, int steps, int batch, double lr, float* loss_trace);
/* Loss and gradient (device, nparams floats, the parameter layout of
 * bpf_proposal_params) on one given minibatch: U (device BF16, batch x 80,
 * standardised [x_t, y - m(x_t)]) and r0 (device FP32, batch x 40,
 * x_{t+1} - m(x_t)). */
int bpf_proposal_loss_grad(bpf_proposal* p, const void* U, const float* r0, int batch, double* loss, float* grads);
/* Host copies of the FP32 parameters W1 [128 x 80], b1, W2 [128 x 128], b2,
 * W3 [80 x 128], b3 and of the input shift and scale (80 each); any pointer
 * may be NULL.  bpf_proposal_set_params loads them. */
int bpf_proposal_params(bpf_proposal* p, float* params, float* shift, float* scale, int* nparams);
int bpf_proposal_set_params(bpf_proposal* p, const float* params, const float* shift, const float* scale);
/* Attach a proposal to a filter (L96, dim 40, FP32) or detach it (p = NULL).
 * Observed steps of exactly the proposal's dt then propose from it and weight
 * by p(y|x') p(x'|x) / q(x'|x, y); unobserved steps use the transition.  The
 * proposal must outlive its use by the handle. */
int bpf_set_proposal(bpf_handle* h, bpf_proposal* p);
/* The same for every filter of a batch (L96, dim 40, FP32; no counterpart in
 * the reference): observed steps of the proposal's dt run the guided step
 * for all filters in one launch, each filter with its own seed and theta,
 * bit for bit a single filter's guided step with that seed and theta.  A
 * captured filter run is recaptured after a change. */
int bpf_batch_set_proposal(bpf_batch* b, bpf_proposal* p);

/* ---- checkpoint (BootstrapPFState save/load,
 *      share/src/bi/state/BootstrapPFState.hpp:216-231) ------------------- */

/* Bytes needed by bpf_snapshot for this handle. */
int bpf_snapshot_size(bpf_handle* h, uint64_t* bytes);
/* Copy state, log-weights, ancestors, scalars and the RNG step counter into
 * host memory buf (bpf_snapshot_size bytes); bpf_restore reads it back. */
int bpf_snapshot(bpf_handle* h, void* buf, uint64_t bytes);
int bpf_restore(bpf_handle* h, const void* buf, uint64_t bytes);

/* Library version string. */
const char* bpf_version(void);
/* Human-readable message for a status code. */
const char* bpf_status_string(int status);

#ifdef __cplusplus
}
#endif

#endif
