// A filter client for a model compiled outside the library: LibBi's
// generated filter client (share/tt/cpp/client/filter_cpu.cpp.tt:105-192:
// model, observer, schedule, resampler, state, Filter<BootstrapPF>::filter)
// over the C++ interface (include/libbi_b200.hpp) with the reference's
// Test.bi model in the generated form (model_test_ar1.cuh), compiled here by
// nvcc against include/bpf_model.cuh.
//
//   model_client <N> <seed> <essRel> <obs file>
//
// The observation file holds one "time component value" line per entry.
// It prints the log-likelihood, then one log-likelihood increment per
// observation (17 significant digits).
#include "bpf_model.cuh"
#include "model_test_ar1.cuh"
#include "libbi_b200.hpp"

#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <vector>

using namespace bi_b200;
typedef DeviceModel<test_ar1::ModelTest> Model;

int main(int argc, char** argv) {
  if (argc < 5) {
    std::fprintf(stderr, "usage: model_client <N> <seed> <essRel> <obs file>\n");
    return 2;
  }
  const int N = std::atoi(argv[1]);
  const uint64_t seed = std::strtoull(argv[2], nullptr, 10);
  const double essRel = std::atof(argv[3]);
  std::vector<double> t, v;
  std::vector<int> c;
  std::ifstream in(argv[4]);
  double a, x;
  int b;
  while (in >> a >> b >> x) {
    t.push_back(a);
    c.push_back(b);
    v.push_back(x);
  }
  Model model({0.9, 0.25});  // theta, sigma2
  Observer obs(t, c, v);
  Schedule sched(0.0, 1.0, &obs);
  Resampler<SystematicResampler> resam(essRel);
  Filter<BootstrapPF<Model, const Observer, Resampler<SystematicResampler>>> filter(model, obs, resam);
  BootstrapPFState<Model> s(model, N);
  Random rng(seed);
  try {
    filter.filter(rng, sched.begin(), sched.end(), s);
  } catch (const ParticleFilterDegeneratedException&) {
    std::printf("degenerate\n");
    return 0;
  } catch (const BpfError& e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 1;
  }
  std::printf("%.17g\n", s.logLikelihood);
  for (double inc : s.logIncrements) std::printf("%.17g\n", inc);
  return 0;
}
