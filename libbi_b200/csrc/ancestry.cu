// Path output with pruned ancestry: the node pool behind bpf_path_cache and
// bpf_sample_path.
//
// LibBi's AncestryCache (share/src/bi/cache/AncestryCache.hpp:294-470) keeps
// one node per recorded particle: its state, the node of its ancestor and a
// count of its recorded children.  Each write (BootstrapPFCache::writeState,
// share/src/bi/cache/BootstrapPFCache.hpp:182-210) counts the offspring of
// the current leaves from the new ancestors, prunes every leaf left without
// offspring and, up its line, every ancestor whose last child went
// (kernelAncestryCachePrune, share/src/bi/cuda/cache/AncestryCacheKernel.cuh:
// 29-48), then inserts the new generation into free nodes.  Only lines that
// reach the current particles are kept, so the store holds the particles'
// genealogy (about N nodes plus the distinct ancestors of each past
// generation, which coalesce) instead of every state of every step.
//
// Here the pool is structure-of-arrays (state element i of node v at
// x[i * cap + v]); free nodes are a stack with a device counter.  A write is
// three kernels: offspring counts (one atomic add per new particle on its
// parent leaf), the prune (one thread per old leaf walks up while it removes
// the last child: each freed node is freed by exactly one thread, whose
// decrement took its count to zero), and the insert (new nodes popped from
// the stack, parent = the leaf of the particle's ancestor, the state copied
// in).  Between prune and insert the host reads the free count and grows
// the pool when fewer than N nodes are free, so a write synchronises the
// stream once.
#include "internal.cuh"

#include <vector>

namespace bpf {
namespace {

__global__ void k_anc_init_stack(int* stack, int* top, int cap) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < cap) stack[i] = cap - 1 - i;  // node 0 on top
  if (i == 0) *top = cap;
}

// offspring of the old leaves: the parent leaf of every new particle
__global__ void k_anc_count(const int* __restrict__ as, const StepStats* st, const int* __restrict__ leaf,
                            int* __restrict__ ref, int n) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const int a = st->resampled ? as[j] : j;
  atomicAdd(&ref[leaf[a]], 1);
}

// free every old leaf without offspring and, up its line, every node whose
// last recorded child was freed
__global__ void k_anc_prune(const int* __restrict__ leaf, int* __restrict__ ref, const int* __restrict__ par,
                            int* __restrict__ stack, int* top, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int v = leaf[i];
  if (ref[v] != 0) return;
  while (true) {
    stack[atomicAdd(top, 1)] = v;
    const int q = par[v];
    if (q < 0) break;
    if (atomicSub(&ref[q], 1) != 1) break;  // q keeps other children
    v = q;
  }
}

// the new generation into free nodes stack[base .. base + n): parent = the
// leaf of the particle's ancestor (none for the first generation)
template <class T>
__global__ void k_anc_insert(const T* __restrict__ x, int ld, int dim, const int* __restrict__ as,
                             const StepStats* st, const int* __restrict__ leaf_old, int* __restrict__ leaf_new,
                             int* __restrict__ par, int* __restrict__ ref, T* __restrict__ nx, int cap,
                             const int* __restrict__ stack, int base, int* top, int n, int first) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j == 0) *top = base;
  if (j >= n) return;
  const int v = stack[base + j];
  par[v] = first ? -1 : leaf_old[st->resampled ? as[j] : j];
  ref[v] = 0;
  for (int i = 0; i < dim; ++i) nx[(size_t)i * cap + v] = x[(size_t)i * ld + j];
  leaf_new[j] = v;
}

// AncestryCache::readPath (AncestryCache.hpp:294-311): from the leaf of
// particle *p back to the first generation
template <class T>
__global__ void k_anc_trace(const T* __restrict__ nx, int cap, const int* __restrict__ par,
                            const int* __restrict__ leaf, int len, int dim, const int* p_in, T* path) {
  int v = leaf[*p_in];
  for (int t = len - 1; t >= 0 && v >= 0; --t) {
    for (int i = threadIdx.x; i < dim; i += blockDim.x) path[(size_t)t * dim + i] = nx[(size_t)i * cap + v];
    v = par[v];
  }
}

int blocks_for(int n) { return (n + 255) / 256; }

int read_top(AncestryPool& a, cudaStream_t st, int* top) {
  BPF_TRY(cudaMemcpyAsync(a.host_top, a.top, sizeof(int), cudaMemcpyDeviceToHost, st));
  BPF_TRY(cudaStreamSynchronize(st));
  *top = *a.host_top;
  return BPF_OK;
}

// a larger pool: the nodes kept where they are, the new ones free
int grow(AncestryPool& a, int top, int need, cudaStream_t st) {
  const int cap2 = a.cap + (a.cap > need ? a.cap : need);
  void* x2 = nullptr;
  int *par2 = nullptr, *ref2 = nullptr, *stack2 = nullptr;
  if (cudaMalloc(&x2, (size_t)a.dim * cap2 * a.esz) != cudaSuccess ||
      cudaMalloc((void**)&par2, (size_t)cap2 * sizeof(int)) != cudaSuccess ||
      cudaMalloc((void**)&ref2, (size_t)cap2 * sizeof(int)) != cudaSuccess ||
      cudaMalloc((void**)&stack2, (size_t)cap2 * sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    if (x2) cudaFree(x2);
    if (par2) cudaFree(par2);
    if (ref2) cudaFree(ref2);
    return BPF_E_NOMEM;
  }
  BPF_TRY(cudaMemcpy2DAsync(x2, (size_t)cap2 * a.esz, a.x, (size_t)a.cap * a.esz, (size_t)a.cap * a.esz, a.dim,
                            cudaMemcpyDeviceToDevice, st));
  BPF_TRY(cudaMemcpyAsync(par2, a.par, (size_t)a.cap * sizeof(int), cudaMemcpyDeviceToDevice, st));
  BPF_TRY(cudaMemcpyAsync(ref2, a.ref, (size_t)a.cap * sizeof(int), cudaMemcpyDeviceToDevice, st));
  // free ids: the old stack, then the new nodes
  BPF_TRY(cudaMemcpyAsync(stack2, a.stack, (size_t)top * sizeof(int), cudaMemcpyDeviceToDevice, st));
  {
    std::vector<int> ids(cap2 - a.cap);
    for (int i = 0; i < cap2 - a.cap; ++i) ids[i] = cap2 - 1 - i;
    BPF_TRY(cudaMemcpyAsync(stack2 + top, ids.data(), ids.size() * sizeof(int), cudaMemcpyHostToDevice, st));
    const int top2 = top + (cap2 - a.cap);
    BPF_TRY(cudaMemcpyAsync(a.top, &top2, sizeof(int), cudaMemcpyHostToDevice, st));
    BPF_TRY(cudaStreamSynchronize(st));  // ids and top2 live on this stack frame
  }
  cudaFree(a.x);
  cudaFree(a.par);
  cudaFree(a.ref);
  cudaFree(a.stack);
  a.x = x2;
  a.par = par2;
  a.ref = ref2;
  a.stack = stack2;
  a.cap = cap2;
  return BPF_OK;
}

int insert(AncestryPool& a, const void* x, int ld, const int* as, const StepStats* st, int base, int first,
           cudaStream_t s) {
  int* leaf_old = a.leaf[a.cur];
  int* leaf_new = a.leaf[a.cur ^ 1];
  if (a.esz == 4)
    k_anc_insert<float><<<blocks_for(a.n), 256, 0, s>>>((const float*)x, ld, a.dim, as, st, leaf_old, leaf_new,
                                                        a.par, a.ref, (float*)a.x, a.cap, a.stack, base, a.top, a.n,
                                                        first);
  else
    k_anc_insert<double><<<blocks_for(a.n), 256, 0, s>>>((const double*)x, ld, a.dim, as, st, leaf_old, leaf_new,
                                                         a.par, a.ref, (double*)a.x, a.cap, a.stack, base, a.top,
                                                         a.n, first);
  BPF_TRY(cudaGetLastError());
  a.cur ^= 1;
  return BPF_OK;
}

}  // namespace

void ancestry_free(AncestryPool& a) {
  void* p[] = {a.x, a.par, a.ref, a.stack, a.top, a.leaf[0], a.leaf[1]};
  for (void* q : p)
    if (q) cudaFree(q);
  if (a.host_top) cudaFreeHost(a.host_top);
  a = AncestryPool();
}

int ancestry_reset(AncestryPool& a, int n, int dim, int esz, const void* x, int ld, cudaStream_t st) {
  if (a.n != n || a.dim != dim || a.esz != esz || !a.x) {
    ancestry_free(a);
    a.n = n;
    a.dim = dim;
    a.esz = esz;
    a.cap = 4 * n;
    if (cudaMalloc(&a.x, (size_t)dim * a.cap * esz) != cudaSuccess ||
        cudaMalloc((void**)&a.par, (size_t)a.cap * sizeof(int)) != cudaSuccess ||
        cudaMalloc((void**)&a.ref, (size_t)a.cap * sizeof(int)) != cudaSuccess ||
        cudaMalloc((void**)&a.stack, (size_t)a.cap * sizeof(int)) != cudaSuccess ||
        cudaMalloc((void**)&a.top, sizeof(int)) != cudaSuccess ||
        cudaMalloc((void**)&a.leaf[0], (size_t)n * sizeof(int)) != cudaSuccess ||
        cudaMalloc((void**)&a.leaf[1], (size_t)n * sizeof(int)) != cudaSuccess ||
        cudaMallocHost((void**)&a.host_top, sizeof(int)) != cudaSuccess) {
      cudaGetLastError();
      ancestry_free(a);
      return BPF_E_NOMEM;
    }
  }
  k_anc_init_stack<<<blocks_for(a.cap), 256, 0, st>>>(a.stack, a.top, a.cap);
  BPF_TRY(cudaGetLastError());
  a.cur = 0;
  return insert(a, x, ld, nullptr, nullptr, a.cap - n, 1, st);
}

int ancestry_append(AncestryPool& a, const void* x, int ld, const int* as, const StepStats* st, cudaStream_t s) {
  k_anc_count<<<blocks_for(a.n), 256, 0, s>>>(as, st, a.leaf[a.cur], a.ref, a.n);
  k_anc_prune<<<blocks_for(a.n), 256, 0, s>>>(a.leaf[a.cur], a.ref, a.par, a.stack, a.top, a.n);
  BPF_TRY(cudaGetLastError());
  int top = 0;
  int rc = read_top(a, s, &top);
  if (rc) return rc;
  if (top < a.n) {
    if ((rc = grow(a, top, a.n, s))) return rc;
    if ((rc = read_top(a, s, &top))) return rc;
  }
  return insert(a, x, ld, as, st, top - a.n, 0, s);
}

int ancestry_trace(const AncestryPool& a, int len, const int* p_dev, void* path_dev, cudaStream_t st) {
  if (a.esz == 4)
    k_anc_trace<float><<<1, 64, 0, st>>>((const float*)a.x, a.cap, a.par, a.leaf[a.cur], len, a.dim, p_dev,
                                         (float*)path_dev);
  else
    k_anc_trace<double><<<1, 64, 0, st>>>((const double*)a.x, a.cap, a.par, a.leaf[a.cur], len, a.dim, p_dev,
                                          (double*)path_dev);
  BPF_TRY(cudaGetLastError());
  return BPF_OK;
}

int ancestry_nodes(AncestryPool& a, cudaStream_t st, int* nodes, int* capacity) {
  int top = 0;
  int rc = read_top(a, st, &top);
  if (rc) return rc;
  if (nodes) *nodes = a.cap - top;
  if (capacity) *capacity = a.cap;
  return BPF_OK;
}

}  // namespace bpf
