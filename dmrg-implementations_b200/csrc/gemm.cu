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

long long& thread_launches() {
  thread_local long long c = 0;
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

template <typename T, typename G, bool TA, bool TB, bool CA>
static void launch_impl(const Gemm<T>& d, int splitk, cudaStream_t st) {
  using S = GemmSmem<T, G, TA, TB>;
  static std::atomic<unsigned long long> attr{0};  // per instantiation, per device
  set_smem_attr_once(attr, (const void*)gemm_kernel<T, G, TA, TB, CA>, (int)S::BYTES);
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
  if (splitk > 1) {
    const int chunk = ceil_div(ceil_div(d.K, splitk), G::BK) * G::BK;
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
      DMRG2_CUDA(cudaLaunchKernelEx(&cfg, gemm_kernel<T, G, TA, TB, CA>, a));
      DMRG2_CHECK_LAUNCH();
      return;
    }
    if (nsplit > 8) {
      // more slices than a portable cluster: partial products per K slice into ws[z]
      // (M x N, ld N), then one reduction
      if (!d.ws) throw std::runtime_error("gemm: more than 8 K slices need a workspace");
      a.C = d.ws; a.ldc = d.N; a.sC1 = (ll)d.M * d.N; a.sC2 = 0;
      a.alpha_re = 1.0; a.alpha_im = 0.0; a.beta_re = 0.0; a.beta_im = 0.0;
      dim3 grid(ceil_div(d.N, G::BN), ceil_div(d.M, G::BM), nsplit);
      gemm_kernel<T, G, TA, TB, CA><<<grid, G::THREADS, S::BYTES, st>>>(a);
      DMRG2_CHECK_LAUNCH();
      splitk_reduce<T>(d.ws, nsplit, d.M, d.N, d.alpha, d.beta, d.C, d.ldc, d.skip, st);
      return;
    }
    a.kchunk = 0;  // one slice
  }
  dim3 grid(ceil_div(d.N, G::BN), ceil_div(d.M, G::BM), d.nb1 * d.nb2);
  gemm_kernel<T, G, TA, TB, CA><<<grid, G::THREADS, S::BYTES, st>>>(a);
  DMRG2_CHECK_LAUNCH();
}

template <typename T, typename G>
static void dispatch(const Gemm<T>& d, int splitk, cudaStream_t st) {
  const bool ca = ST<T>::cplx && d.ca;
  if (!d.ta && !d.tb && !ca) return launch_impl<T, G, false, false, false>(d, splitk, st);
  if (!d.ta && d.tb && !ca) return launch_impl<T, G, false, true, false>(d, splitk, st);
  if (d.ta && !d.tb && !ca) return launch_impl<T, G, true, false, false>(d, splitk, st);
  if (d.ta && d.tb && !ca) return launch_impl<T, G, true, true, false>(d, splitk, st);
  if constexpr (ST<T>::cplx) {
    if (!d.ta && !d.tb) return launch_impl<T, G, false, false, true>(d, splitk, st);
    if (!d.ta && d.tb) return launch_impl<T, G, false, true, true>(d, splitk, st);
    if (d.ta && !d.tb) return launch_impl<T, G, true, false, true>(d, splitk, st);
    return launch_impl<T, G, true, true, true>(d, splitk, st);
  }
}

// ---------------------------------------------------------------- autotuner
// A single real GEMM of at least TUNE_MIN_FLOP is run in each configuration (64 x 64
// tiles with 1, 2, 4 or 8 K slices reduced in a cluster; 32 x 32 tiles with 1, 2 or 4)
// the first time its shape (transposes, M, N, K) occurs in the process, on the caller's
// stream and operands, writing into a scratch output (never the caller's C, no skip
// flag); the fastest by CUDA events serves every later GEMM of that shape. Smaller GEMMs
// are latency-bound and keep the default (64 x 64 tiles, the caller's K split): their
// many distinct shapes (chain ends, bond-dimension ramps) would cost more to time than
// a configuration can save. The tuning is off unless DMRG2_GEMM_TUNE=1: measured on the
// L=100, chi=256 sweep it gains 2% on steady sweeps but loses 10% on a run that starts
// from a fresh engine (the choices timed in isolation, on L2-resident operands, do not
// carry over to the sweep's own cache state), and off, results do not depend on timing.
namespace {
struct TuneKey {
  int ta, tb, M, N, K, dev;
  bool operator==(const TuneKey& o) const {
    return ta == o.ta && tb == o.tb && M == o.M && N == o.N && K == o.K && dev == o.dev;
  }
};
struct TuneKeyHash {
  size_t operator()(const TuneKey& k) const {
    size_t h = (size_t)k.M * 1000003u ^ (size_t)k.N * 9176u ^ (size_t)k.K * 31u;
    return h ^ (size_t)(k.ta * 2 + k.tb) ^ ((size_t)k.dev << 40);
  }
};
struct TuneChoice {
  int tile;   // 0: TileD64, 1: TileD32
  int splitk;
};
constexpr double TUNE_MIN_FLOP = 1e8;
std::mutex& tune_mutex() {
  static std::mutex m;
  return m;
}
std::unordered_map<TuneKey, TuneChoice, TuneKeyHash>& tune_cache() {
  static auto* c = new std::unordered_map<TuneKey, TuneChoice, TuneKeyHash>();
  return *c;
}
}  // namespace

bool tune_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("DMRG2_GEMM_TUNE");
    return e && e[0] == '1';
  }();
  return on;
}

namespace {
TuneChoice tuned(const Gemm<double>& d, cudaStream_t st) {
  int dev = 0;
  DMRG2_CUDA(cudaGetDevice(&dev));
  const TuneKey key{d.ta ? 1 : 0, d.tb ? 1 : 0, d.M, d.N, d.K, dev};
  std::lock_guard<std::mutex> lk(tune_mutex());
  auto it = tune_cache().find(key);
  if (it != tune_cache().end()) return it->second;
  Gemm<double> t = d;
  t.skip = nullptr;
  t.ldc = d.N;
  t.sC1 = t.sC2 = 0;
  t.C = (double*)dev_alloc(sizeof(double) * (size_t)d.M * d.N);
  cudaEvent_t e0, e1;
  DMRG2_CUDA(cudaEventCreate(&e0));
  DMRG2_CUDA(cudaEventCreate(&e1));
  TuneChoice best{0, 1};
  float best_ms = 1e30f;
  for (int tile = 0; tile < 2; ++tile)
    for (int sk = 1; sk <= (tile == 0 ? 8 : 4); sk *= 2) {
      if (sk > 1 && d.K < 32 * sk) continue;  // at least two k-tiles per slice
      auto run = [&]() {
        if (tile == 0) dispatch<double, TileD64>(t, sk, st);
        else dispatch<double, TileD32>(t, sk, st);
      };
      run();  // first launch: attributes, instruction cache
      DMRG2_CUDA(cudaEventRecord(e0, st));
      for (int r = 0; r < 2; ++r) run();
      DMRG2_CUDA(cudaEventRecord(e1, st));
      DMRG2_CUDA(cudaEventSynchronize(e1));
      float ms = 0.f;
      DMRG2_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      if (ms < best_ms) {
        best_ms = ms;
        best = {tile, sk};
      }
    }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  dev_free(t.C);  // the stream is idle after the last event
  tune_cache()[key] = best;
  return best;
}
}  // namespace

template <typename T>
void launch_gemm(const Gemm<T>& d, cudaStream_t st) {
  if (d.M <= 0 || d.N <= 0 || d.nb1 * d.nb2 <= 0) return;
  if (d.nb1 * d.nb2 > 65535) throw std::runtime_error("gemm: batch count exceeds 65535");
  if (d.splitk > 1 && d.nb1 * d.nb2 != 1) throw std::runtime_error("gemm: split-K needs a single GEMM");
  if (ceil_div(d.M, TileD32::BM) > 65535) throw std::runtime_error("gemm: M too large");
  if constexpr (!ST<T>::cplx) {
    if (d.nb1 * d.nb2 == 1 && 2.0 * d.M * d.N * d.K >= TUNE_MIN_FLOP && tune_enabled()) {
      const TuneChoice c = tuned(d, st);
      if (c.tile == 1) return dispatch<T, TileD32>(d, c.splitk, st);
      return dispatch<T, TileD64>(d, c.splitk, st);
    }
  }
  dispatch<T, GemmTile<T>>(d, d.splitk, st);
}

template void launch_gemm<double>(const Gemm<double>&, cudaStream_t);
template void launch_gemm<zc>(const Gemm<zc>&, cudaStream_t);

}  // namespace dmrg2
