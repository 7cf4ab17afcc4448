// Shared scalar types, error handling and small device helpers.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>

namespace dmrg2 {

typedef long long ll;

struct __align__(16) zc {
  double re, im;
};

__host__ __device__ inline zc mkz(double r, double i) { zc z; z.re = r; z.im = i; return z; }
__host__ __device__ inline zc operator+(zc a, zc b) { return mkz(a.re + b.re, a.im + b.im); }
__host__ __device__ inline zc operator-(zc a, zc b) { return mkz(a.re - b.re, a.im - b.im); }
__host__ __device__ inline zc operator*(zc a, zc b) {
  return mkz(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
__host__ __device__ inline zc operator*(double s, zc a) { return mkz(s * a.re, s * a.im); }

// Scalar traits: real double or complex double (interleaved re, im).
template <typename T> struct ST;
template <> struct ST<double> {
  static constexpr bool cplx = false;
  __host__ __device__ static double zero() { return 0.0; }
  __host__ __device__ static double one() { return 1.0; }
  __host__ __device__ static double conj(double a) { return a; }
  __host__ __device__ static double re(double a) { return a; }
  __host__ __device__ static double im(double) { return 0.0; }
  __host__ __device__ static double abs2(double a) { return a * a; }
  __host__ __device__ static double make(double r, double) { return r; }
  __host__ __device__ static double mul(double a, double b) { return a * b; }
  __host__ __device__ static double add(double a, double b) { return a + b; }
  __host__ __device__ static double scale(double s, double a) { return s * a; }
  // conj(a) * b
  __host__ __device__ static double cmul(double a, double b) { return a * b; }
};
template <> struct ST<zc> {
  static constexpr bool cplx = true;
  __host__ __device__ static zc zero() { return mkz(0, 0); }
  __host__ __device__ static zc one() { return mkz(1, 0); }
  __host__ __device__ static zc conj(zc a) { return mkz(a.re, -a.im); }
  __host__ __device__ static double re(zc a) { return a.re; }
  __host__ __device__ static double im(zc a) { return a.im; }
  __host__ __device__ static double abs2(zc a) { return a.re * a.re + a.im * a.im; }
  __host__ __device__ static zc make(double r, double i) { return mkz(r, i); }
  __host__ __device__ static zc mul(zc a, zc b) { return a * b; }
  __host__ __device__ static zc add(zc a, zc b) { return a + b; }
  __host__ __device__ static zc scale(double s, zc a) { return mkz(s * a.re, s * a.im); }
  __host__ __device__ static zc cmul(zc a, zc b) {
    return mkz(a.re * b.re + a.im * b.im, a.re * b.im - a.im * b.re);
  }
};

struct CudaError : public std::runtime_error {
  explicit CudaError(const std::string& s) : std::runtime_error(s) {}
};

// A numerical method did not reach its accuracy (reported as DMRG2_ERR_NUMERIC).
struct NumericError : public std::runtime_error {
  explicit NumericError(const std::string& s) : std::runtime_error(s) {}
};

#define DMRG2_CUDA(call)                                                              \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess) {                                                          \
      throw ::dmrg2::CudaError(std::string("CUDA error ") + cudaGetErrorString(e_) +  \
                               " at " + __FILE__ + ":" + std::to_string(__LINE__) +   \
                               " (" #call ")");                                       \
    }                                                                                 \
  } while (0)

// Every kernel launch of the library goes through DMRG2_CHECK_LAUNCH, which
// also counts it (reported through dmrg2_get_launch_count).
std::atomic<long long>& launch_counter();  // kernels launched by this library (all threads)
long long& thread_launches();              // the same, by the calling thread
#define DMRG2_CHECK_LAUNCH()            \
  do {                                  \
    DMRG2_CUDA(cudaGetLastError());     \
    ++::dmrg2::launch_counter();        \
    ++::dmrg2::thread_launches();       \
  } while (0)

// GEMMs pick their tile shapes by timing candidates (DMRG2_GEMM_TUNE=1)
bool tune_enabled();

inline int ceil_div(ll a, ll b) { return (int)((a + b - 1) / b); }

// Test hook for the bounded device waits: with DMRG2_TEST_UNSIGNALLED_WAITS=1 in the
// environment, the kernels that wait on a completion (the tensor-core commit of the
// split GEMM, the grid barrier of the cooperative Jacobi SVD) wait on one that nothing
// signals, with a short poll limit, so a test can see the timeout reported as
// DMRG2_ERR_NUMERIC while the device stays usable.
bool test_unsignalled_waits();

// Device memory of the library, from the device's stream-ordered pool (cudaMallocAsync
// on a private stream of the calling thread, which the call then waits for). Unlike
// cudaMalloc / cudaFree, neither call synchronises the device, so an engine that is created
// or destroyed while others run (the served form) does not stall their streams; the pool
// keeps released memory for the next allocation. dev_free requires that no stream still
// uses the memory (owners synchronise their stream first).
void* dev_alloc(size_t bytes);
void dev_free(void* p);

// Page-locked host memory from a process-wide cache of blocks in power-of-two size
// classes: a block is page-locked once and reused, never handed back to the driver
// (cudaFreeHost synchronises the device, which would stall every other engine's stream).
void* host_pinned(size_t bytes);
void host_unpin(void* p);

// cudaFuncSetAttribute acts on the current device only; `done` records, one bit
// per device ordinal (mod 64), where the attribute was already set.
inline void func_attr_once(std::atomic<unsigned long long>& done, const void* func, cudaFuncAttribute attr,
                           int value) {
  int dev = 0;
  DMRG2_CUDA(cudaGetDevice(&dev));
  const unsigned long long bit = 1ull << (dev & 63);
  if (done.load(std::memory_order_acquire) & bit) return;
  DMRG2_CUDA(cudaFuncSetAttribute(func, attr, value));
  done.fetch_or(bit, std::memory_order_acq_rel);
}

inline void set_smem_attr_once(std::atomic<unsigned long long>& done, const void* func, int bytes) {
  func_attr_once(done, func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

}  // namespace dmrg2
