// Host launcher and instantiations of the DMMA GEMM.
#include <cstdlib>
#include <map>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "gemm.cuh"

namespace dmrg2 {

std::atomic<long long>& launch_counter() {
  static std::atomic<long long> c{0};
  return c;
}

namespace {
// the calling thread's private stream for pool calls on the current device
cudaStream_t pool_stream(int& device) {
  constexpr int kMaxDev = 64;
  // the thread's private streams, destroyed when the thread ends
  struct Streams {
    cudaStream_t s[kMaxDev] = {};
    ~Streams() {
      for (cudaStream_t x : s)
        if (x) (void)cudaStreamDestroy(x);
    }
  };
  thread_local Streams own;
  cudaStream_t* streams = own.s;
  static std::atomic<unsigned long long> pool_ready[kMaxDev];
  DMRG2_CUDA(cudaGetDevice(&device));
  if (device < 0 || device >= kMaxDev) throw std::runtime_error("dev_alloc: device index out of range");
  if (!pool_ready[device].load()) {
    // keep freed blocks in the pool instead of returning them at each synchronisation
    cudaMemPool_t pool;
    DMRG2_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
    unsigned long long keep = ~0ull;
    DMRG2_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    pool_ready[device].store(1);
  }
  if (!streams[device]) DMRG2_CUDA(cudaStreamCreateWithFlags(&streams[device], cudaStreamNonBlocking));
  return streams[device];
}
}  // namespace

void* dev_alloc(size_t bytes) {
  int dev = 0;
  cudaStream_t s = pool_stream(dev);
  void* p = nullptr;
  DMRG2_CUDA(cudaMallocAsync(&p, bytes ? bytes : 16, s));
  DMRG2_CUDA(cudaStreamSynchronize(s));  // usable from any stream from here on
  return p;
}

void dev_free(void* p) {
  if (!p) return;
  int dev = 0;
  cudaStream_t s = pool_stream(dev);
  cudaFreeAsync(p, s);
}

namespace {
struct PinnedCache {
  std::mutex mu;
  std::map<size_t, std::vector<void*>> free_blocks;  // size class -> idle blocks
  std::unordered_map<void*, size_t> cls;             // block -> its size class
};
PinnedCache& pinned_cache() {
  static PinnedCache* c = new PinnedCache();  // lives to process exit (blocks may outlive statics)
  return *c;
}
}  // namespace

void* host_pinned(size_t bytes) {
  size_t c = 64;
  while (c < bytes) c <<= 1;
  PinnedCache& pc = pinned_cache();
  {
    std::lock_guard<std::mutex> lk(pc.mu);
    auto& v = pc.free_blocks[c];
    if (!v.empty()) {
      void* p = v.back();
      v.pop_back();
      return p;
    }
  }
  void* p = nullptr;
  DMRG2_CUDA(cudaMallocHost(&p, c));
  std::lock_guard<std::mutex> lk(pc.mu);
  pc.cls[p] = c;
  return p;
}

void host_unpin(void* p) {
  if (!p) return;
  PinnedCache& pc = pinned_cache();
  std::lock_guard<std::mutex> lk(pc.mu);
  auto it = pc.cls.find(p);
  if (it == pc.cls.end()) return;  // not from this cache
  pc.free_blocks[it->second].push_back(p);
}

bool test_unsignalled_waits() {
  static const bool on = [] {
    const char* e = std::getenv("DMRG2_TEST_UNSIGNALLED_WAITS");
    return e && e[0] == '1';
  }();
  return on;
}

template <typename T>
__global__ void splitk_reduce_kernel(const T* __restrict__ ws, int ns, int M, int N, double ar,
                                     double ai, double br, double bi, T* __restrict__ C, ll ldc,
                                     const int* skip) {
  if (skip && *((volatile const int*)skip)) return;
  const ll tot = (ll)M * N;
  const T alpha = ST<T>::make(ar, ai), beta = ST<T>::make(br, bi);
  const bool use_beta = (br != 0.0 || bi != 0.0);
  for (ll t = (ll)blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += (ll)gridDim.x * blockDim.x) {
    T acc = ws[t];
    for (int z = 1; z < ns; ++z) acc = acc + ws[(ll)z * tot + t];
    const ll m = t / N, n = t % N;
    T* c = C + m * ldc + n;
    T v = ST<T>::mul(alpha, acc);
    if (use_beta) v = v + ST<T>::mul(beta, *c);
    *c = v;
  }
}

template <typename T>
static void splitk_reduce(const T* ws, int ns, int M, int N, T alpha, T beta, T* C, ll ldc,
                          const int* skip, cudaStream_t st) {
  ll tot = (ll)M * N;
  ll g = (tot + 255) / 256;
  if (g > 148 * 8) g = 148 * 8;
  splitk_reduce_kernel<T><<<(int)(g < 1 ? 1 : g), 256, 0, st>>>(ws, ns, M, N, ST<T>::re(alpha), ST<T>::im(alpha),
                                                          ST<T>::re(beta), ST<T>::im(beta), C, ldc, skip);
  DMRG2_CHECK_LAUNCH();
}

template <typename T, bool TA, bool TB, bool CA>
static void launch_impl(const Gemm<T>& d, cudaStream_t st) {
  using G = GemmTile<T>;
  using S = GemmSmem<T, TA, TB>;
  static std::atomic<unsigned long long> attr{0};  // per instantiation, per device
  set_smem_attr_once(attr, (const void*)gemm_kernel<T, TA, TB, CA>, (int)S::BYTES);
  GemmArgs a;
  a.M = d.M; a.N = d.N; a.K = d.K;
  a.A = d.A; a.lda = d.lda; a.sA1 = d.sA1; a.sA2 = d.sA2;
  a.B = d.B; a.ldb = d.ldb; a.sB1 = d.sB1; a.sB2 = d.sB2;
  a.C = d.C; a.ldc = d.ldc; a.sC1 = d.sC1; a.sC2 = d.sC2;
  a.nb2 = d.nb2;
  a.alpha_re = ST<T>::re(d.alpha); a.alpha_im = ST<T>::im(d.alpha);
  a.beta_re = ST<T>::re(d.beta); a.beta_im = ST<T>::im(d.beta);
  a.skip = d.skip;
  a.kchunk = 0;
  a.kcluster = 0;
  if (d.splitk > 1) {
    const int chunk = ceil_div(ceil_div(d.K, d.splitk), G::BK) * G::BK;
    const int nsplit = ceil_div(d.K, chunk);
    a.kchunk = chunk;
    a.sA1 = a.sA2 = a.sB1 = a.sB2 = a.sC1 = a.sC2 = 0;
    a.nb2 = 1;
    if (nsplit > 1 && nsplit <= 8) {
      // the slices of a tile form one cluster and are summed in it: no workspace, no
      // second launch, the same summation order as the reduction kernel
      a.kcluster = nsplit;
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(ceil_div(d.N, G::BN), ceil_div(d.M, G::BM), nsplit);
      cfg.blockDim = dim3(G::THREADS);
      cfg.dynamicSmemBytes = S::BYTES;
      cfg.stream = st;
      cudaLaunchAttribute at[1];
      at[0].id = cudaLaunchAttributeClusterDimension;
      at[0].val.clusterDim.x = 1;
      at[0].val.clusterDim.y = 1;
      at[0].val.clusterDim.z = nsplit;
      cfg.attrs = at;
      cfg.numAttrs = 1;
      DMRG2_CUDA(cudaLaunchKernelEx(&cfg, gemm_kernel<T, TA, TB, CA>, a));
      DMRG2_CHECK_LAUNCH();
      return;
    }
    // more slices than a portable cluster: partial products per K slice into ws[z]
    // (M x N, ld N), then one reduction
    a.C = d.ws; a.ldc = d.N; a.sC1 = (ll)d.M * d.N; a.sC2 = 0;
    a.sA1 = a.sA2 = a.sB1 = a.sB2 = 0;
    a.nb2 = 1;
    a.alpha_re = 1.0; a.alpha_im = 0.0; a.beta_re = 0.0; a.beta_im = 0.0;
    dim3 grid(ceil_div(d.N, G::BN), ceil_div(d.M, G::BM), nsplit);
    gemm_kernel<T, TA, TB, CA><<<grid, G::THREADS, S::BYTES, st>>>(a);
    DMRG2_CHECK_LAUNCH();
    splitk_reduce<T>(d.ws, nsplit, d.M, d.N, d.alpha, d.beta, d.C, d.ldc, d.skip, st);
    return;
  }
  dim3 grid(ceil_div(d.N, G::BN), ceil_div(d.M, G::BM), d.nb1 * d.nb2);
  gemm_kernel<T, TA, TB, CA><<<grid, G::THREADS, S::BYTES, st>>>(a);
  DMRG2_CHECK_LAUNCH();
}

template <typename T>
void launch_gemm(const Gemm<T>& d, cudaStream_t st) {
  if (d.M <= 0 || d.N <= 0 || d.nb1 * d.nb2 <= 0) return;
  if (d.nb1 * d.nb2 > 65535) throw std::runtime_error("gemm: batch count exceeds 65535");
  if (d.splitk > 1 && (d.nb1 * d.nb2 != 1 || !d.ws))
    throw std::runtime_error("gemm: split-K needs a single GEMM and a workspace");
  if (ceil_div(d.M, GemmTile<T>::BM) > 65535) throw std::runtime_error("gemm: M too large");
  const bool ca = ST<T>::cplx && d.ca;
  if (!d.ta && !d.tb && !ca) return launch_impl<T, false, false, false>(d, st);
  if (!d.ta && d.tb && !ca) return launch_impl<T, false, true, false>(d, st);
  if (d.ta && !d.tb && !ca) return launch_impl<T, true, false, false>(d, st);
  if (d.ta && d.tb && !ca) return launch_impl<T, true, true, false>(d, st);
  if constexpr (ST<T>::cplx) {
    if (!d.ta && !d.tb) return launch_impl<T, false, false, true>(d, st);
    if (!d.ta && d.tb) return launch_impl<T, false, true, true>(d, st);
    if (d.ta && !d.tb) return launch_impl<T, true, false, true>(d, st);
    return launch_impl<T, true, true, true>(d, st);
  }
}

template void launch_gemm<double>(const Gemm<double>&, cudaStream_t);
template void launch_gemm<zc>(const Gemm<zc>&, cudaStream_t);

}  // namespace dmrg2
