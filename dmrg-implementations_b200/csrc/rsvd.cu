// Device kernels of the randomised truncated split: the random sketch matrix and the
// real embedding of complex column blocks used by its CholeskyQR passes.
#include "rsvd.cuh"

namespace dmrg2 {

namespace {

// SplitMix64 (Steele, Lea and Flood, OOPSLA 2014): a counter-based generator, one
// independent 64-bit output per (seed, index)
__device__ inline unsigned long long splitmix64(unsigned long long x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
// uniform on [-1, 1) from the top 53 bits
__device__ inline double unit_sym(unsigned long long h) { return (double)(h >> 11) * 0x1.0p-52 - 1.0; }

template <typename T>
__global__ void rsvd_omega_kernel(T* __restrict__ om, ll n, unsigned long long seed) {
  const unsigned long long key = splitmix64(seed);
  for (ll t = (ll)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (ll)gridDim.x * blockDim.x) {
    if constexpr (ST<T>::cplx) {
      om[t] = mkz(unit_sym(splitmix64(key ^ (2ull * t))), unit_sym(splitmix64(key ^ (2ull * t + 1))));
    } else {
      om[t] = unit_sym(splitmix64(key ^ (unsigned long long)t));
    }
  }
}

// Y (len x r complex, row-major) -> YR (2 len x 2 r real): the column pair (2j, 2j+1) is
// the real image of (y_j, i y_j), row 2i holds real parts and row 2i+1 imaginary parts
__global__ void embed_pairs_kernel(const zc* __restrict__ Y, ll len, int r, double* __restrict__ YR) {
  const ll tot = len * r;
  for (ll t = (ll)blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += (ll)gridDim.x * blockDim.x) {
    const ll i = t / r;
    const int j = (int)(t % r);
    const zc y = Y[t];
    double* r0 = YR + (2 * i) * (2 * (ll)r) + 2 * j;
    double* r1 = r0 + 2 * (ll)r;
    r0[0] = y.re;
    r0[1] = -y.im;
    r1[0] = y.im;
    r1[1] = y.re;
  }
}

// Q (len x r complex) from the even columns of QR (2 len x 2 r real)
__global__ void extract_pairs_kernel(const double* __restrict__ QR, ll len, int r, zc* __restrict__ Q) {
  const ll tot = len * r;
  for (ll t = (ll)blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += (ll)gridDim.x * blockDim.x) {
    const ll i = t / r;
    const int j = (int)(t % r);
    Q[t] = mkz(QR[(2 * i) * (2 * (ll)r) + 2 * j], QR[(2 * i + 1) * (2 * (ll)r) + 2 * j]);
  }
}

int grid_for(ll tot) {
  ll g = (tot + 255) / 256;
  if (g > 148 * 8) g = 148 * 8;
  return (int)(g < 1 ? 1 : g);
}

}  // namespace

template <typename T>
void rsvd_omega(T* om, ll n, unsigned long long seed, cudaStream_t s) {
  if (n < 1) return;
  rsvd_omega_kernel<T><<<grid_for(n), 256, 0, s>>>(om, n, seed);
  DMRG2_CHECK_LAUNCH();
}
template void rsvd_omega<double>(double*, ll, unsigned long long, cudaStream_t);
template void rsvd_omega<zc>(zc*, ll, unsigned long long, cudaStream_t);

void embed_pairs(const zc* Y, ll len, int r, double* YR, cudaStream_t s) {
  if (len < 1 || r < 1) return;
  embed_pairs_kernel<<<grid_for(len * r), 256, 0, s>>>(Y, len, r, YR);
  DMRG2_CHECK_LAUNCH();
}

void extract_pairs(const double* QR, ll len, int r, zc* Q, cudaStream_t s) {
  if (len < 1 || r < 1) return;
  extract_pairs_kernel<<<grid_for(len * r), 256, 0, s>>>(QR, len, r, Q);
  DMRG2_CHECK_LAUNCH();
}

}  // namespace dmrg2
