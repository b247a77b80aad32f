// Systematic resampling without any device allocation.
//
// Some callers cannot let a library allocate device memory: a host
// application that has reserved the GPU's memory up front for its own
// allocator, or a real-time loop in which a cudaMalloc (which may
// synchronise the whole device) is not allowed.  For them
// bpf_systematic_ancestors_static runs the same systematic resampling
// kernels as bpf_resampler_ancestors, but its scratch lives in one
// file-scope __device__ array of fixed size that the library carries on
// every GPU that loads it, for as long as the process runs.
//
// The first call on each device looks up the array's device address with
// cudaGetSymbolAddress (with that device current) and caches it; make that
// first call before any stream capture.  Every call shares the one array:
// calls whose work overlaps on the GPU (two streams, or two host threads on
// the same device) race on it and must be ordered by the caller.
#include "internal.cuh"

#include <mutex>

namespace bpf {
namespace {

constexpr int kStaticMaxN = BPF_STATIC_MAX_PARTICLES;
constexpr int kStaticTiles = (kStaticMaxN + kTile - 1) / kTile;
constexpr int kStaticPartials = (kStaticMaxN + 63) / 64 + 1;

constexpr size_t align256(size_t b) { return (b + 255) / 256 * 256; }

// carve-up of the scratch array (byte offsets, each 256-byte aligned)
constexpr size_t kOffTileSum = 0;
constexpr size_t kOffTilePrefix = kOffTileSum + align256((kStaticTiles + 1) * sizeof(u128));
constexpr size_t kOffZcount = kOffTilePrefix + align256((kStaticTiles + 1) * sizeof(u128));
constexpr size_t kOffZprefix = kOffZcount + align256((kStaticTiles + 1) * sizeof(int));
constexpr size_t kOffOs = kOffZprefix + align256((kStaticTiles + 1) * sizeof(int));
constexpr size_t kOffE = kOffOs + align256(kStaticMaxN * sizeof(int));
constexpr size_t kOffSlot = kOffE + align256(kStaticMaxN * sizeof(int));
constexpr size_t kOffEtile = kOffSlot + align256(kStaticMaxN * sizeof(int));
constexpr size_t kOffCounters = kOffEtile + align256((kStaticMaxN / 16 + 2) * sizeof(int));
constexpr size_t kOffStats = kOffCounters + align256(16 * sizeof(unsigned));
constexpr size_t kOffPartials = kOffStats + align256(sizeof(StepStats));
constexpr size_t kOffPub = kOffPartials + align256(kStaticPartials * sizeof(LwPartial));
constexpr int kStaticPubEntries = kStaticMaxN / 128 + 2;
constexpr size_t kPubBytes = (size_t)kStaticPubEntries * kPubWords * sizeof(unsigned long long);
constexpr size_t kScratchBytes = kOffPub + align256(kPubBytes);

// the scratch itself: zero at module load, about 1 MiB per device
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
unsigned char* g_base[kMaxDevices] = {nullptr};

// device address of g_scratch on the current device, looked up once
int scratch_base(unsigned char** base) {
  int dev = 0;
  BPF_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return BPF_E_INVALID;
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_base[dev]) {
    void* p = nullptr;
    BPF_TRY(cudaGetSymbolAddress(&p, g_scratch));
    g_base[dev] = static_cast<unsigned char*>(p);
  }
  *base = g_base[dev];
  return BPF_OK;
}

}  // namespace
}  // namespace bpf

extern "C" int bpf_systematic_ancestors_static(const double* lw, int n, const double* a, int permute, int* as,
                                               int* Os, void* stream) {
  using namespace bpf;
  if (!lw || !as || n <= 0) return BPF_E_INVALID;
  if (n > kStaticMaxN) return BPF_E_TOO_LARGE;
  unsigned char* base = nullptr;
  int rc = scratch_base(&base);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  ResampleScratch s;
  s.max_n = kStaticMaxN;
  s.max_tiles = kStaticTiles;
  s.tile_sum = reinterpret_cast<u128*>(base + kOffTileSum);
  s.tile_prefix = reinterpret_cast<u128*>(base + kOffTilePrefix);
  s.zcount = reinterpret_cast<int*>(base + kOffZcount);
  s.zprefix = reinterpret_cast<int*>(base + kOffZprefix);
  s.Os = reinterpret_cast<int*>(base + kOffOs);
  s.E = reinterpret_cast<int*>(base + kOffE);
  s.slot = reinterpret_cast<int*>(base + kOffSlot);
  s.etile = reinterpret_cast<int*>(base + kOffEtile);
  s.counters = reinterpret_cast<unsigned*>(base + kOffCounters);
  s.stats = reinterpret_cast<StepStats*>(base + kOffStats);
  s.partials = reinterpret_cast<LwPartial*>(base + kOffPartials);
  s.max_partials = kStaticPartials;
  s.pub = reinterpret_cast<unsigned long long*>(base + kOffPub);
  s.pub_entries = kStaticPubEntries;
  // the array keeps the previous call's contents: clear the last-block
  // counters (the one-launch kernel's epoch among them) and the statistics
  // (status = BPF_OK) before this call's kernels, and give the published
  // words tags no epoch of this call carries
  BPF_TRY(cudaMemsetAsync(s.counters, 0, 16 * sizeof(unsigned), st));
  BPF_TRY(cudaMemsetAsync(s.stats, 0, sizeof(StepStats), st));
  BPF_TRY(cudaMemsetAsync(s.pub, 0xFF, kPubBytes, st));
  ResampleArgs ra;
  ra.kind = BPF_RESAMPLER_SYSTEMATIC;
  ra.n = n;
  ra.B = 0;
  ra.lw = lw;
  ra.uniforms = a;
  ra.seed = 0;
  ra.step = 0;
  ra.permute = permute;
  ra.as = as;
  ra.Os_out = Os;
  ra.gate = nullptr;
  ra.max_known = false;
  rc = launch_resample(ra, s, st);
  if (rc) return rc;
  int status = BPF_OK;
  BPF_TRY(cudaMemcpyAsync(&status, &s.stats->status, sizeof(int), cudaMemcpyDeviceToHost, st));
  BPF_TRY(cudaStreamSynchronize(st));
  return status;
}
