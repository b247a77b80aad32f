// Oracle test infrastructure (never shipped, never timed as the product).
//
// Thin extern "C" driver around the reference's OWN host resampler code,
// compiled from the reference sources where they lie (see oracle/Makefile).
// Every draw the reference makes is served from a caller-filled tape of
// uniforms (oracle/shim/boost/random/tape.hpp), so that the reference's
// ancestors can be compared bit for bit with the CUDA path on the same
// log-weights and uniforms.  Instantiated with real = double.
#include "bi/math/loc_temp_vector.hpp"
#include "bi/traits/resampler_traits.hpp"
#include "bi/resampler/Resampler.hpp"
#include "bi/resampler/SystematicResampler.hpp"
#include "bi/resampler/MultinomialResampler.hpp"
#include "bi/resampler/MetropolisResampler.hpp"
#include "bi/host/resampler/ResamplerHost.hpp"
#include "bi/primitive/vector_primitive.hpp"
#include "bi/primitive/matrix_primitive.hpp"
#include "bi/math/vector.hpp"
#include "bi/math/matrix.hpp"
#include "bi/random/Random.hpp"

#include <stdexcept>

namespace {
typedef bi::host_vector<double> dvec;
typedef bi::host_vector<int> ivec;

/* one host thread, so the reference consumes the tape in loop order */
void ensure_init() {
  static bool init = false;
  if (!init) { bi_omp_init(1); init = true; }
}

bi::Random& rng() {
  ensure_init();
  static bi::Random r(0);
  return r;
}

void load(dvec& v, const double* x, int n) { for (int i = 0; i < n; ++i) v(i) = x[i]; }
void store(const ivec& v, int* x, int n) { for (int i = 0; i < n; ++i) x[i] = v(i); }
}

extern "C" {

/* bi::ess_reduce, share/src/bi/primitive/vector_primitive.hpp:960-974 */
double ref_ess_reduce(const double* lw, int n, double* lW) {
  ensure_init();
  dvec v(n); load(v, lw, n);
  return bi::ess_reduce(v, lW);
}

/* bi::logsumexp_reduce, share/src/bi/primitive/vector_primitive.hpp:933-943 */
double ref_logsumexp_reduce(const double* lw, int n) {
  ensure_init();
  dvec v(n); load(v, lw, n);
  return bi::logsumexp_reduce(v);
}

/* ScanResampler::precompute + SystematicResampler::cumulativeOffspring +
 * ResamplerHost::cumulativeOffspringToAncestors[Permute]
 * (share/src/bi/resampler/SystematicResampler.hpp:111-148,
 *  share/src/bi/host/resampler/ResamplerHost.hpp:110-168).
 * Returns 0, or 1 when the reference throws ParticleFilterDegeneratedException. */
int ref_systematic(const double* lw, int n, double a, int permute,
    double* Ws_out, int* Os_out, int* as_out) {
  ensure_init();
  bi::SystematicResampler R;
  dvec v(n); load(v, lw, n);
  bi::ScanResamplerPrecompute<bi::ON_HOST> pre;
  ivec Os(n), as(n);
  boost::random_tape::set(&a, 1);
  try {
    R.precompute(v, pre);
    R.cumulativeOffspring(rng(), v, n, Os, pre);
  } catch (bi::ParticleFilterDegeneratedException&) {
    return 1;
  }
  if (permute) bi::ResamplerHost::cumulativeOffspringToAncestorsPermute(Os, as);
  else bi::ResamplerHost::cumulativeOffspringToAncestors(Os, as);
  if (Ws_out) for (int i = 0; i < n; ++i) Ws_out[i] = pre.Ws(i);
  if (Os_out) store(Os, Os_out, n);
  if (as_out) store(as, as_out, n);
  return 0;
}

/* ScanResampler::precompute + MultinomialResamplerHost::ancestors
 * (Bentley & Saxe sorted draws, share/src/bi/host/resampler/MultinomialResamplerHost.hpp:29-65),
 * then ResamplerHost::permute (:171-190) when permute != 0.  u: n uniforms. */
int ref_multinomial(const double* lw, int n, const double* u, int permute, int* as_out) {
  ensure_init();
  bi::MultinomialResampler R;
  dvec v(n); load(v, lw, n);
  bi::ScanResamplerPrecompute<bi::ON_HOST> pre;
  ivec as(n);
  boost::random_tape::set(u, n);
  try {
    R.precompute(v, pre);
    if (permute) R.ancestorsPermute(rng(), v, as, pre);
    else R.ancestors(rng(), v, as, pre);
  } catch (bi::ParticleFilterDegeneratedException&) {
    return 1;
  }
  store(as, as_out, n);
  return 0;
}

/* MetropolisResamplerHost::ancestors[Permute]
 * (share/src/bi/host/resampler/MetropolisResamplerHost.hpp:32-62).
 * u: 2*B*n uniforms, particle-major: for p, for k<B: (index draw, accept draw). */
int ref_metropolis(const double* lw, int n, int B, const double* u, int permute, int* as_out) {
  ensure_init();
  bi::MetropolisResampler R(B);
  dvec v(n); load(v, lw, n);
  bi::ResamplerPrecompute<bi::ON_HOST> pre;
  ivec as(n);
  boost::random_tape::set(u, (size_t)2*B*n);
  if (permute) R.ancestorsPermute(rng(), v, as, pre);
  else R.ancestors(rng(), v, as, pre);
  store(as, as_out, n);
  return 0;
}

/* ResamplerHost::permute, share/src/bi/host/resampler/ResamplerHost.hpp:171-190 */
void ref_permute(int* as, int n) {
  ensure_init();
  ivec v(n);
  for (int i = 0; i < n; ++i) v(i) = as[i];
  bi::ResamplerHost::permute(v);
  store(v, as, n);
}

/* bi::gather_rows, share/src/bi/host/primitive/matrix_primitive.hpp:66-75:
 * X(i,:) = X(as(i),:) in place on a column-major n x d matrix. */
void ref_gather_rows(const int* as, double* X, int n, int d) {
  ensure_init();
  bi::host_matrix<double> M(n, d);
  ivec a(n);
  for (int i = 0; i < n; ++i) a(i) = as[i];
  for (int j = 0; j < d; ++j) for (int i = 0; i < n; ++i) M(i, j) = X[(size_t)j*n + i];
  bi::gather_rows(a, M, M);
  for (int j = 0; j < d; ++j) for (int i = 0; i < n; ++i) X[(size_t)j*n + i] = M(i, j);
}

}
