// A filter client over the C++ interface (include/libbi_b200.hpp), shaped
// like LibBi's generated filter client (share/tt/cpp/client/filter_cpu.cpp.tt:
// model, observer, schedule, resampler, state, Filter<BootstrapPF>::filter).
//
//   filter_client <l96|pz> <N> <seed> <essRel> <obs file> [path]
//
// The observation file holds one "time component value" line per entry.  It
// prints the log-likelihood, then one "increment ess" line per observation
// (17 significant digits), or "degenerate" when the filter throws
// ParticleFilterDegeneratedException; with "path", also a sampled path.
#include "libbi_b200.hpp"

#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <string>
#include <vector>

using namespace bi_b200;

template <class M>
int run(M& model, int N, uint64_t seed, double essRel, const Observer& obs, double delta, bool path) {
  Schedule sched(0.0, delta, &obs);
  Resampler<SystematicResampler> resam(essRel);
  Filter<BootstrapPF<M, const Observer, Resampler<SystematicResampler>>> filter(model, obs, resam);
  BootstrapPFState<M> s(model, N);
  Random rng(seed);
  try {
    if (path) {
      filter.init(rng, s);
      filter.recordPath(s, sched.size());
    }
    filter.filter(rng, sched.begin(), sched.end(), s);
  } catch (const ParticleFilterDegeneratedException&) {
    std::printf("degenerate\n");
    return 0;
  }
  std::printf("%.17g\n", s.logLikelihood);
  for (size_t k = 0; k < s.logIncrements.size(); ++k) std::printf("%.17g\n", s.logIncrements[k]);
  if (path) {
    std::vector<typename M::real> p;
    int particle = -1;
    const int len = filter.samplePath(rng, s, p, &particle);
    std::printf("path %d %d\n", particle, len);
  }
  return 0;
}

int main(int argc, char** argv) {
  if (argc < 6) {
    std::fprintf(stderr, "usage: %s <l96|pz> <N> <seed> <essRel> <obs file> [path]\n", argv[0]);
    return 2;
  }
  const std::string kind = argv[1];
  const int N = std::atoi(argv[2]);
  const uint64_t seed = std::strtoull(argv[3], nullptr, 10);
  const double essRel = std::atof(argv[4]);
  const bool path = argc > 6 && std::string(argv[6]) == "path";
  std::vector<double> t, v;
  std::vector<int> c;
  std::ifstream in(argv[5]);
  double tt, vv;
  int cc;
  while (in >> tt >> cc >> vv) {
    t.push_back(tt);
    c.push_back(cc);
    v.push_back(vv);
  }
  if (!in.eof()) {
    std::fprintf(stderr, "error: unreadable observation file %s\n", argv[5]);
    return 1;
  }
  const Observer obs(t, c, v);
  try {
    if (kind == "l96") {
      ModelL96 m;
      m.dim = 8;
      return run(m, N, seed, essRel, obs, 0.05, path);
    }
    ModelPZ m;
    return run(m, N, seed, essRel, obs, 1.0, path);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
}
