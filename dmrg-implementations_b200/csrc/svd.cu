// Theta truncation: one-sided block Jacobi SVD with on-device sort, cutoff and
// gauge split.
//
// Replaces rocsolver gesvdj/gesvd + svd_truncate_kernel + extract_cols /
// scale_rows/cols kernels of the reference (gpu-rocm/dmrg2-gpu/src/dmrg2_gpu_impl.h:1167-1343,
// gpu-rocm/common/scalar_traits.h:164-188,497-547).
//
// Method (Hestenes one-sided Jacobi, block-cyclic): the matrix is held as
// `nvec` vectors of length `len` (contiguous). Vectors are grouped into blocks
// of B; each round of the round-robin tournament pairs all blocks, and each
// CTA of a cooperative grid orthogonalises one block pair: it forms the
// 2B x 2B Gram matrix, diagonalises it with cyclic two-sided Jacobi in shared
// memory, and applies the accumulated unitary to the vectors and to the
// accumulated right factor Q. Sweeps repeat until no pair rotates. The
// singular values are the final vector norms; no division by a singular
// value is ever needed because both factors of the split come either from
// the rotated vectors (which carry S) or from Q (which is unitary).
#include "kernels.cuh"

#include <cooperative_groups.h>

namespace dmrg2 {

template <typename T>
struct JacobiCfg;
template <>
struct JacobiCfg<double> {
  static constexpr int B = 16, CH = 64;
};
template <>
struct JacobiCfg<zc> {
  static constexpr int B = 8, CH = 32;
};

static constexpr int JT = 256;  // threads per Jacobi CTA

// grid barrier; `arrivals` is the block count (one more under the unsignalled-wait
// test hook, so nothing completes it), `spin_max` the polls before it gives up
__device__ bool jacobi_grid_sync(JacobiCtl* c, unsigned nblocks, long long spin_max) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned* genp = &c->bar_gen;
    unsigned g = *genp;
    __threadfence();
    unsigned arrived = atomicAdd(&c->bar_count, 1u) + 1u;
    ok = 1;
    if (arrived == nblocks) {
      atomicExch(&c->bar_count, 0u);
      __threadfence();
      atomicAdd(&c->bar_gen, 1u);
    } else {
      long long spins = 0;
      while (*genp == g) {
        if (*((volatile int*)&c->err)) { ok = 0; break; }
        if (++spins > spin_max) { atomicExch(&c->err, 2); ok = 0; break; }
        __nanosleep(64);
      }
    }
    __threadfence();
  }
  __syncthreads();
  return ok != 0;
}

// position-k player of the circle method with m = nb-1 rotating players
__device__ inline int rr_player(int k, int r, int m) { return 1 + ((k + r) % m); }

template <typename T>
struct Rot {
  double r00, r01;
  T r10, r11;
  int a, b;
};

template <typename T>
__device__ inline T conjT(T v) { return ST<T>::conj(v); }

template <typename T>
__global__ void __launch_bounds__(JT)
    jacobi_kernel(T* __restrict__ X, T* __restrict__ Q, int nvec, ll len, int nb, JacobiCtl* ctl,
                  int max_sweeps, double tol, const double* fro2_dev, int unsignalled) {
  constexpr int B = JacobiCfg<T>::B, P = 2 * B, CH = JacobiCfg<T>::CH;
  __shared__ T G[P][P + 1];
  __shared__ T J[P][P + 1];
  __shared__ T tile[P][CH + 1];
  __shared__ Rot<T> rot[B];
  __shared__ int vid[P];
  __shared__ int any_s, skip_s;
  const int tid = threadIdx.x;
  const double fro2 = fro2_dev ? *fro2_dev : 1.0;
  const double thr = 1e-30 * fro2;  // squared-norm floor below which a vector is treated as zero
  const int m = nb - 1;
  int sweep = 0;
  bool alive = true;
  for (sweep = 0; sweep < max_sweeps && alive; ++sweep) {
    for (int r = 0; r < m && alive; ++r) {
      for (int p = blockIdx.x; p < nb / 2; p += gridDim.x) {
        int bi, bj;
        if (p == 0) { bi = 0; bj = rr_player(0, r, m); }
        else { bi = rr_player(p, r, m); bj = rr_player(m - p, r, m); }
        if (tid < P) {
          int blk = (tid < B) ? bi : bj;
          int v = blk * B + (tid % B);
          vid[tid] = (v < nvec) ? v : -1;
        }
        __syncthreads();
        // ---- Gram matrix of the pair
        T acc[(P * P + JT - 1) / JT];
#pragma unroll
        for (int e = 0; e < (P * P + JT - 1) / JT; ++e) acc[e] = ST<T>::zero();
        for (ll c0 = 0; c0 < len; c0 += CH) {
          for (int e = tid; e < P * CH; e += JT) {
            int u = e / CH, l = e % CH;
            int v = vid[u];
            tile[u][l] = (v >= 0 && c0 + l < len) ? X[(ll)v * len + c0 + l] : ST<T>::zero();
          }
          __syncthreads();
#pragma unroll
          for (int e = 0; e < (P * P + JT - 1) / JT; ++e) {
            int idx = tid + e * JT;
            if (idx < P * P) {
              int pp = idx / P, qq = idx % P;
              T s = ST<T>::zero();
#pragma unroll 8
              for (int l = 0; l < CH; ++l) s = s + ST<T>::cmul(tile[pp][l], tile[qq][l]);
              acc[e] = acc[e] + s;
            }
          }
          __syncthreads();
        }
#pragma unroll
        for (int e = 0; e < (P * P + JT - 1) / JT; ++e) {
          int idx = tid + e * JT;
          if (idx < P * P) G[idx / P][idx % P] = acc[e];
        }
        for (int idx = tid; idx < P * P; idx += JT) J[idx / P][idx % P] = (idx / P == idx % P) ? ST<T>::one() : ST<T>::zero();
        if (tid == 0) skip_s = 1;
        __syncthreads();
        // ---- quick test: is any pair of this block pair non-orthogonal?
        for (int idx = tid; idx < P * P; idx += JT) {
          int a = idx / P, b = idx % P;
          if (a < b) {
            double gaa = ST<T>::re(G[a][a]), gbb = ST<T>::re(G[b][b]);
            if (gaa > thr && gbb > thr && sqrt(ST<T>::abs2(G[a][b])) > tol * sqrt(gaa * gbb)) skip_s = 0;
          }
        }
        __syncthreads();
        if (skip_s) continue;
        // ---- inner cyclic Jacobi on the Gram matrix, accumulating J
        for (int isw = 0; isw < 20; ++isw) {
          if (tid == 0) any_s = 0;
          __syncthreads();
          for (int ir = 0; ir < P - 1; ++ir) {
            if (tid < B) {
              int k = tid, a, b;
              const int mm = P - 1;
              if (k == 0) { a = 0; b = 1 + (ir % mm); }
              else { a = 1 + ((k + ir) % mm); b = 1 + ((mm - k + ir) % mm); }
              Rot<T> R;
              R.a = a; R.b = b;
              R.r00 = 1.0; R.r01 = 0.0; R.r10 = ST<T>::zero(); R.r11 = ST<T>::one();
              double gaa = ST<T>::re(G[a][a]), gbb = ST<T>::re(G[b][b]);
              T gab = G[a][b];
              double ab = sqrt(ST<T>::abs2(gab));
              if (gaa > thr && gbb > thr && ab > tol * sqrt(gaa * gbb)) {
                double zeta = (gbb - gaa) / (2.0 * ab);
                double t = (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
                double cs = 1.0 / sqrt(1.0 + t * t), sn = cs * t;
                // e^{-i phi} = conj(gab)/|gab|
                T ph = ST<T>::scale(1.0 / ab, ST<T>::conj(gab));
                R.r00 = cs;
                R.r01 = sn;
                R.r10 = ST<T>::scale(-sn, ph);
                R.r11 = ST<T>::scale(cs, ph);
                any_s = 1;
              }
              rot[k] = R;
            }
            __syncthreads();
            // rows: G <- R^H G
            for (int idx = tid; idx < B * P; idx += JT) {
              int k = idx / P, c = idx % P;
              const Rot<T>& R = rot[k];
              T g1 = G[R.a][c], g2 = G[R.b][c];
              G[R.a][c] = ST<T>::scale(R.r00, g1) + ST<T>::mul(conjT(R.r10), g2);
              G[R.b][c] = ST<T>::scale(R.r01, g1) + ST<T>::mul(conjT(R.r11), g2);
            }
            __syncthreads();
            // columns: G <- G R, J <- J R
            for (int idx = tid; idx < B * P; idx += JT) {
              int k = idx / P, rr = idx % P;
              const Rot<T>& R = rot[k];
              T g1 = G[rr][R.a], g2 = G[rr][R.b];
              G[rr][R.a] = ST<T>::scale(R.r00, g1) + ST<T>::mul(g2, R.r10);
              G[rr][R.b] = ST<T>::scale(R.r01, g1) + ST<T>::mul(g2, R.r11);
              T j1 = J[rr][R.a], j2 = J[rr][R.b];
              J[rr][R.a] = ST<T>::scale(R.r00, j1) + ST<T>::mul(j2, R.r10);
              J[rr][R.b] = ST<T>::scale(R.r01, j1) + ST<T>::mul(j2, R.r11);
            }
            __syncthreads();
          }
          int cont = any_s;
          __syncthreads();
          if (!cont) break;
        }
        // ---- apply J to the vectors and to Q
        for (int pass = 0; pass < 2; ++pass) {
          T* base = (pass == 0) ? X : Q;
          const ll L = (pass == 0) ? len : (ll)nvec;
          for (ll c0 = 0; c0 < L; c0 += CH) {
            for (int e = tid; e < P * CH; e += JT) {
              int u = e / CH, l = e % CH;
              int v = vid[u];
              tile[u][l] = (v >= 0 && c0 + l < L) ? base[(ll)v * L + c0 + l] : ST<T>::zero();
            }
            __syncthreads();
            for (int e = tid; e < P * CH; e += JT) {
              int vv = e / CH, l = e % CH;
              int v = vid[vv];
              if (v >= 0 && c0 + l < L) {
                T s = ST<T>::zero();
#pragma unroll 8
                for (int u = 0; u < P; ++u) s = s + ST<T>::mul(tile[u][l], J[u][vv]);
                base[(ll)v * L + c0 + l] = s;
              }
            }
            __syncthreads();
          }
        }
        if (tid == 0) ctl->rotated[sweep] = 1;
        __syncthreads();
      }
      alive = unsignalled ? jacobi_grid_sync(ctl, gridDim.x + 1, 1LL << 14)
                          : jacobi_grid_sync(ctl, gridDim.x, 1LL << 25);
    }
    if (!alive) break;
    if (!*((volatile int*)&ctl->rotated[sweep])) { ++sweep; break; }
  }
  if (blockIdx.x == 0 && tid == 0) ctl->sweeps = sweep;
}

template <typename T>
void svd_jacobi(T* X, T* Q, int nvec, ll len, JacobiCtl* ctl, int max_sweeps, double tol,
                const double* fro2_dev, cudaStream_t s) {
  constexpr int B = JacobiCfg<T>::B;
  if (max_sweeps > 64) max_sweeps = 64;
  int nb = (nvec + B - 1) / B;
  if (nb < 2) nb = 2;
  if (nb & 1) ++nb;
  DMRG2_CUDA(cudaMemsetAsync(ctl, 0, sizeof(JacobiCtl), s));
  int max_coresident = 0;
  {
    int dev = 0, nsm = 0, per = 0;
    DMRG2_CUDA(cudaGetDevice(&dev));
    DMRG2_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    DMRG2_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, jacobi_kernel<T>, JT, 0));
    max_coresident = nsm * (per > 0 ? per : 1);
  }
  int grid = nb / 2;
  if (grid > max_coresident) grid = max_coresident;
  int unsignalled = test_unsignalled_waits() ? 1 : 0;
  void* args[] = {&X, &Q, &nvec, &len, &nb, &ctl, &max_sweeps, &tol, (void*)&fro2_dev, &unsignalled};
  DMRG2_CUDA(cudaLaunchCooperativeKernel((const void*)jacobi_kernel<T>, dim3(grid), dim3(JT), args,
                                         0, s));
  DMRG2_CHECK_LAUNCH();
}

// ----------------------------------------------------------------------------
template <typename T>
__global__ void vec_norms_kernel(const T* __restrict__ X, int nvec, ll len, double* sigma) {
  int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (w >= nvec) return;
  double s = 0.0;
  for (ll l = lane; l < len; l += 32) s += ST<T>::abs2(X[(ll)w * len + l]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) sigma[w] = sqrt(s);
}

__global__ void sort_truncate_kernel(const double* sigma, int nvec, ll len, int* perm, SvdOut* out,
                                     int chi_max, double cutoff, int relative, const JacobiCtl* ctl) {
  for (int v = threadIdx.x; v < nvec; v += blockDim.x) {
    double sv = sigma[v];
    int r = 0;
    for (int u = 0; u < nvec; ++u) {
      double su = sigma[u];
      r += (su > sv) || (su == sv && u < v);
    }
    perm[r] = v;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double smax = sigma[perm[0]];
    int kmax = nvec < len ? nvec : (int)len;
    int k = chi_max < kmax ? chi_max : kmax;
    double thr = relative ? cutoff * smax : cutoff;
    int nz = 0;
    for (int r = 0; r < kmax; ++r) if (sigma[perm[r]] > 0.0) ++nz;
    if (cutoff > 0.0) {
      for (int r = 0; r < k; ++r) {
        if (sigma[perm[r]] < thr) { k = r; break; }
      }
    }
    if (k < 1) k = 1;
    double te = 0.0, f2 = 0.0;
    for (int r = 0; r < nvec; ++r) {
      double s2 = sigma[perm[r]] * sigma[perm[r]];
      f2 += s2;
      if (r >= k) te += s2;
    }
    out->k = k;
    out->nonzero = nz;
    out->trunc_err = te;
    out->sigma_max = smax;
    out->sigma_max2 = smax * smax;
    out->fro2 = f2;
    out->jacobi_sweeps = ctl ? ctl->sweeps : 0;
    out->jacobi_err = ctl ? ctl->err : 0;
  }
}

template <typename T>
void svd_sort_truncate(const T* X, int nvec, ll len, double* sigma, int* perm, SvdOut* out,
                       int chi_max, double cutoff, bool relative_cutoff, const JacobiCtl* ctl,
                       cudaStream_t s) {
  int threads = 256;
  int blocks = (nvec * 32 + threads - 1) / threads;
  vec_norms_kernel<T><<<blocks, threads, 0, s>>>(X, nvec, len, sigma);
  DMRG2_CHECK_LAUNCH();
  sort_truncate_kernel<<<1, 1024, 0, s>>>(sigma, nvec, len, perm, out, chi_max, cutoff,
                                          relative_cutoff ? 1 : 0, ctl);
  DMRG2_CHECK_LAUNCH();
}

template <typename T>
__global__ void gather_kernel(const T* __restrict__ X, const T* __restrict__ Q,
                              const int* __restrict__ perm, int nvec, ll len, int k, int mode,
                              T* __restrict__ left, T* __restrict__ right) {
  // left: rows x k, right: k x cols; rows = (mode 0 ? nvec : len), cols = (mode 0 ? len : nvec)
  const ll rows = mode == 0 ? nvec : len;
  const ll cols = mode == 0 ? len : nvec;
  const ll nl = rows * k, nr = (ll)k * cols;
  for (ll i = (ll)blockIdx.x * blockDim.x + threadIdx.x; i < nl + nr;
       i += (ll)gridDim.x * blockDim.x) {
    if (i < nl) {
      ll r = i / k;
      int j = (int)(i % k);
      int v = perm[j];
      left[i] = (mode == 0) ? ST<T>::conj(Q[(ll)v * nvec + r]) : X[(ll)v * len + r];
    } else {
      ll t = i - nl;
      int j = (int)(t / cols);
      ll c = t % cols;
      int v = perm[j];
      right[t] = (mode == 0) ? X[(ll)v * len + c] : ST<T>::conj(Q[(ll)v * nvec + c]);
    }
  }
}

template <typename T>
void svd_gather(const T* X, const T* Q, const int* perm, int nvec, ll len, int k, int mode,
                T* left, T* right, cudaStream_t s) {
  ll tot = ((mode == 0 ? (ll)nvec : len) + (mode == 0 ? len : (ll)nvec)) * k;
  ll g = (tot + 255) / 256;
  if (g > 148 * 8) g = 148 * 8;
  if (g < 1) g = 1;
  gather_kernel<T><<<(int)g, 256, 0, s>>>(X, Q, perm, nvec, len, k, mode, left, right);
  DMRG2_CHECK_LAUNCH();
}

// ----------------------------------------------------------------------------
template <typename T>
__global__ void transpose_kernel(const T* __restrict__ in, T* __restrict__ out, ll rows, ll cols) {
  __shared__ T t[32][33];
  ll c0 = (ll)blockIdx.x * 32, r0 = (ll)blockIdx.y * 32;
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    ll r = r0 + i, c = c0 + threadIdx.x;
    if (r < rows && c < cols) t[i][threadIdx.x] = in[r * cols + c];
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    ll c = c0 + i, r = r0 + threadIdx.x;
    if (r < rows && c < cols) out[c * rows + r] = t[threadIdx.x][i];
  }
}

template <typename T>
void transpose(const T* in, T* out, ll rows, ll cols, cudaStream_t s) {
  dim3 grid(ceil_div(cols, 32), ceil_div(rows, 32));
  if (grid.y > 65535) throw std::runtime_error("transpose: too many rows");
  transpose_kernel<T><<<grid, dim3(32, 8), 0, s>>>(in, out, rows, cols);
  DMRG2_CHECK_LAUNCH();
}

template <typename T>
__global__ void identity_kernel(T* Q, int n) {
  ll tot = (ll)n * n;
  for (ll i = (ll)blockIdx.x * blockDim.x + threadIdx.x; i < tot; i += (ll)gridDim.x * blockDim.x)
    Q[i] = (i / n == i % n) ? ST<T>::one() : ST<T>::zero();
}

template <typename T>
void set_identity(T* Q, int n, cudaStream_t s) {
  ll tot = (ll)n * n;
  ll g = (tot + 255) / 256;
  if (g > 148 * 8) g = 148 * 8;
  if (g < 1) g = 1;
  identity_kernel<T><<<(int)g, 256, 0, s>>>(Q, n);
  DMRG2_CHECK_LAUNCH();
}

// flag[0] = 1 when max |P - 1| <= tol for the n x n matrix P (one block)
template <typename T>
__global__ void identity_check_kernel(const T* __restrict__ P, int n, double tol, int* __restrict__ flag) {
  __shared__ double red[256];
  double m = 0.0;
  const ll tot = (ll)n * n;
  for (ll e = threadIdx.x; e < tot; e += blockDim.x) {
    const ll i = e / n, j = e % n;
    const T v = P[e];
    const double re = ST<T>::re(v) - (i == j ? 1.0 : 0.0), im = ST<T>::im(v);
    m = fmax(m, fabs(re) + fabs(im));
  }
  red[threadIdx.x] = m;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0) *flag = (red[0] <= tol) ? 1 : 0;
}

template <typename T>
void identity_check(const T* P, int n, double tol, int* flag, cudaStream_t s) {
  identity_check_kernel<T><<<1, 256, 0, s>>>(P, n, tol, flag);
  DMRG2_CHECK_LAUNCH();
}

template <typename T>
__global__ void trace_kernel(const T* M, int n, ll ld, double* out_re, double* out_im) {
  __shared__ double sr[256], si[256];
  double a = 0.0, b = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    T v = M[(ll)i * ld + i];
    a += ST<T>::re(v);
    b += ST<T>::im(v);
  }
  sr[threadIdx.x] = a;
  si[threadIdx.x] = b;
  __syncthreads();
  if (threadIdx.x == 0) {
    double ta = 0.0, tb = 0.0;
    for (int i = 0; i < (int)blockDim.x; ++i) { ta += sr[i]; tb += si[i]; }
    *out_re = ta;
    *out_im = tb;
  }
}

template <typename T>
void trace_real(const T* M, int n, ll ld, double* out_re, double* out_im, cudaStream_t s) {
  trace_kernel<T><<<1, 256, 0, s>>>(M, n, ld, out_re, out_im);
  DMRG2_CHECK_LAUNCH();
}

// ---------------------------------------------------------------- boundary-merge helpers
// out[j] = sigma[perm[j]], j < k: the kept singular values in sorted order
__global__ void gather_sigma_kernel(const double* __restrict__ sigma, const int* __restrict__ perm, int k,
                                    double* __restrict__ out) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < k; j += gridDim.x * blockDim.x) out[j] = sigma[perm[j]];
}
void gather_sigma(const double* sigma, const int* perm, int k, double* out, cudaStream_t s) {
  if (k < 1) return;
  gather_sigma_kernel<<<(k + 255) / 256, 256, 0, s>>>(sigma, perm, k, out);
  DMRG2_CHECK_LAUNCH();
}
// v[j] <- 1 / max(v[j], floor)
__global__ void inv_clip_kernel(double* __restrict__ v, int k, double floor) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < k; j += gridDim.x * blockDim.x) v[j] = 1.0 / fmax(v[j], floor);
}
void inv_clip(double* v, int k, double floor, cudaStream_t s) {
  if (k < 1) return;
  inv_clip_kernel<<<(k + 255) / 256, 256, 0, s>>>(v, k, floor);
  DMRG2_CHECK_LAUNCH();
}
// out[r][c] = in[r][c] * v[r] (or / v[r] when invert), rows x cols row-major
template <typename T>
__global__ void row_scale_kernel(const T* __restrict__ in, const double* __restrict__ v, int rows, ll cols,
                                 T* __restrict__ out, int invert) {
  const ll tot = (ll)rows * cols;
  for (ll t = (ll)blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += (ll)gridDim.x * blockDim.x) {
    const double f = invert ? 1.0 / v[t / cols] : v[t / cols];
    if constexpr (ST<T>::cplx) out[t] = mkz(f * in[t].re, f * in[t].im);
    else out[t] = f * in[t];
  }
}
template <typename T>
void row_scale(const T* in, const double* v, int rows, ll cols, T* out, bool invert, cudaStream_t s) {
  const ll tot = (ll)rows * cols;
  if (tot < 1) return;
  ll g = (tot + 255) / 256;
  if (g > 148 * 8) g = 148 * 8;
  row_scale_kernel<T><<<(int)g, 256, 0, s>>>(in, v, rows, cols, out, invert ? 1 : 0);
  DMRG2_CHECK_LAUNCH();
}

#define INST(T)                                                                                 \
  template void svd_jacobi<T>(T*, T*, int, ll, JacobiCtl*, int, double, const double*,        \
                              cudaStream_t);   \
  template void svd_sort_truncate<T>(const T*, int, ll, double*, int*, SvdOut*, int, double,     \
                                     bool, const JacobiCtl*, cudaStream_t);                                        \
  template void svd_gather<T>(const T*, const T*, const int*, int, ll, int, int, T*, T*,         \
                              cudaStream_t);                                                     \
  template void transpose<T>(const T*, T*, ll, ll, cudaStream_t);                                \
  template void set_identity<T>(T*, int, cudaStream_t);                                          \
  template void trace_real<T>(const T*, int, ll, double*, double*, cudaStream_t);                \
  template void identity_check<T>(const T*, int, double, int*, cudaStream_t);                   \
  template void row_scale<T>(const T*, const double*, int, ll, T*, bool, cudaStream_t);
INST(double)
INST(zc)
#undef INST

}  // namespace dmrg2
