// Device-resident Lanczos with full reorthogonalisation.
//
// Replaces the reference's Lanczos loop (gpu-rocm/dmrg2-gpu/src/dmrg2_gpu_impl.h:971-1160):
// the BLAS-1/2 calls (dot, axpy, two reorthogonalisation GEMVs, nrm2, scal) and
// the per-iteration scalar kernels become three fused streaming kernels per
// iteration that read every Krylov vector with coalesced loads, reduce with
// warp shuffles, and finalise in the last block to arrive (no host sync). The
// last block of the third kernel also solves the tridiagonal eigenproblem for
// its lowest eigenvalue (Sturm-sequence multisection), applies the |dE| stop
// rule and, once done, computes the Ritz coefficients by inverse iteration, so
// the host never copies alpha/beta back.
#include "kernels.cuh"

namespace dmrg2 {

static constexpr int MAX_CHUNK = 2048;

int vec_blocks(ll n) {
  ll nb = (n + VEC_THREADS - 1) / VEC_THREADS;
  if (nb > 592) nb = 592;
  if (nb < 1) nb = 1;
  ll ch = (n + nb - 1) / nb;
  if (ch > MAX_CHUNK) nb = (n + MAX_CHUNK - 1) / MAX_CHUNK;
  return (int)nb;
}

__device__ inline double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ inline double block_sum(double v, double* sh) {
  v = warp_sum(v);
  int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x < 32) {
    r = (threadIdx.x < (blockDim.x >> 5)) ? sh[threadIdx.x] : 0.0;
    r = warp_sum(r);
  }
  __syncthreads();
  if (threadIdx.x == 0) sh[0] = r;
  __syncthreads();
  r = sh[0];
  __syncthreads();
  return r;
}

__device__ inline bool arrive_last(unsigned* counter, unsigned nblk) {
  __shared__ int am_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) am_last = (atomicAdd(counter, 1u) == nblk - 1) ? 1 : 0;
  __syncthreads();
  if (am_last) __threadfence();
  return am_last != 0;
}

// ----------------------------------------------------------------------------
// tridiagonal helpers (block-wide / single thread)
// ----------------------------------------------------------------------------
// 1/a from the hardware estimate and two Newton-Raphson steps y <- y + y (1 - a y)
__device__ inline double rcp_refined(double a) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(a));
  double r = fma(-a, y, 1.0);
  y = fma(y, r, y);
  r = fma(-a, y, 1.0);
  return fma(y, r, y);
}

__device__ inline int sturm_count(const double* a, const double* b, int k, double x, double pivmin) {
  double q = a[0] - x;
  int c = 0;
  if (fabs(q) < pivmin) q = -pivmin;
  if (q < 0) ++c;
  for (int i = 1; i < k; ++i) {
    q = (a[i] - x) - b[i - 1] * b[i - 1] * rcp_refined(q);
    if (fabs(q) < pivmin) q = -pivmin;
    if (q < 0) ++c;
  }
  return c;
}

// Lowest eigenvalue of the symmetric tridiagonal (a, b) of order k. All threads
// of the block must call; the result is returned to every thread. When hint is
// finite, the bracket starts at [hint - 2|b_{k-2}| - tiny, hint]: by Cauchy
// interlacing the lowest eigenvalue of T_k is at most that of T_{k-1} (hint),
// and by Weyl's bound it is at least hint - |b_{k-2}| - |a_{k-1} - ...| which the
// Gershgorin check below still guards.
__device__ double tridiag_lowest(const double* a, const double* b, int k, double hint) {
  __shared__ double lo_s, hi_s, piv_s;
  __shared__ int tmin;
  const int NT = blockDim.x;
  if (threadIdx.x == 0) {
    double lo = 1e300, hi = -1e300, bm = 0.0;
    for (int i = 0; i < k; ++i) {
      double r = (i > 0 ? fabs(b[i - 1]) : 0.0) + (i < k - 1 ? fabs(b[i]) : 0.0);
      lo = fmin(lo, a[i] - r);
      hi = fmax(hi, a[i] + r);
      if (i < k - 1) bm = fmax(bm, b[i] * b[i]);
    }
    double w = fmax(hi - lo, 1e-300);
    lo_s = lo - 1e-14 * w;
    hi_s = hi + 1e-14 * w;
    piv_s = 1e-300 * fmax(1.0, bm);
    if (k >= 2 && isfinite(hint) && hint < 1e299) {
      // tight bracket: [hint - 2 |b_{k-2}| - slack, hint + slack], verified by counts below
      double slack = 1e-12 * fmax(fabs(hint), 1e-300) + 1e-300;
      double tlo = hint - 2.0 * fabs(b[k - 2]) - slack, thi = hint + slack;
      int clo = sturm_count(a, b, k, tlo, piv_s), chi = sturm_count(a, b, k, thi, piv_s);
      if (clo == 0 && chi >= 1) {
        lo_s = tlo;
        hi_s = thi;
      }
    }
  }
  __syncthreads();
  for (int round = 0; round < 12; ++round) {
    double lo = lo_s, hi = hi_s;
    double x = lo + (hi - lo) * (double)(threadIdx.x + 1) / (double)(NT + 1);
    int c = sturm_count(a, b, k, x, piv_s);
    if (threadIdx.x == 0) tmin = NT;
    __syncthreads();
    if (c >= 1) atomicMin(&tmin, (int)threadIdx.x);
    __syncthreads();
    if (threadIdx.x == 0) {
      int t = tmin;
      double step = (hi - lo) / (double)(NT + 1);
      if (t == NT) {
        lo_s = lo + step * NT;
      } else {
        hi_s = lo + step * (t + 1);
        lo_s = lo + step * t;
      }
    }
    __syncthreads();
    double l2 = lo_s, h2 = hi_s;
    if (h2 - l2 <= 4e-16 * fmax(fabs(l2), fabs(h2)) + 1e-300) break;
  }
  double r = 0.5 * (lo_s + hi_s);
  __syncthreads();
  return r;
}

// Eigenvector of the tridiagonal (a, b) for eigenvalue lam by inverse iteration
// with partial pivoting (single thread; k <= KRYLOV_CAP).
__device__ void tridiag_vector(const double* a, const double* b, int k, double lam, double* y,
                               double* work) {
  double* u0 = work;
  double* u1 = work + KRYLOV_CAP;
  double* u2 = work + 2 * KRYLOV_CAP;
  double* l = work + 3 * KRYLOV_CAP;
  double* sw = work + 4 * KRYLOV_CAP;
  double scale = 0.0;
  for (int i = 0; i < k; ++i) scale = fmax(scale, fabs(a[i]) + (i < k - 1 ? fabs(b[i]) : 0.0));
  const double tiny = 1e-15 * fmax(scale, 1e-300);
  for (int i = 0; i < k; ++i) {
    u0[i] = a[i] - lam;
    u1[i] = (i < k - 1) ? b[i] : 0.0;
    u2[i] = 0.0;
  }
  for (int i = 0; i < k - 1; ++i) {
    double s = b[i];
    if (fabs(u0[i]) >= fabs(s)) {
      if (u0[i] == 0.0) u0[i] = tiny;
      double m = s / u0[i];
      u0[i + 1] -= m * u1[i];
      l[i] = m;
      sw[i] = 0.0;
    } else {
      double m = u0[i] / s;
      double old_u1i = u1[i];
      u0[i] = s;
      u1[i] = u0[i + 1];
      u2[i] = u1[i + 1];
      u0[i + 1] = old_u1i - m * u1[i];
      u1[i + 1] = -m * u2[i];
      l[i] = m;
      sw[i] = 1.0;
    }
  }
  if (u0[k - 1] == 0.0) u0[k - 1] = tiny;
  for (int i = 0; i < k; ++i) y[i] = 1.0;
  for (int it = 0; it < 3; ++it) {
    for (int i = 0; i < k - 1; ++i) {
      if (sw[i] != 0.0) { double t = y[i]; y[i] = y[i + 1]; y[i + 1] = t; }
      y[i + 1] -= l[i] * y[i];
    }
    for (int i = k - 1; i >= 0; --i) {
      double v = y[i];
      if (i + 1 < k) v -= u1[i] * y[i + 1];
      if (i + 2 < k) v -= u2[i] * y[i + 2];
      double d = u0[i];
      if (fabs(d) < tiny) d = (d < 0 ? -tiny : tiny);
      y[i] = v / d;
    }
    double nrm = 0.0;
    for (int i = 0; i < k; ++i) nrm += y[i] * y[i];
    nrm = sqrt(nrm);
    if (!(nrm > 0.0) || !isfinite(nrm)) {
      for (int i = 0; i < k; ++i) y[i] = (i == 0) ? 1.0 : 0.0;
      break;
    }
    for (int i = 0; i < k; ++i) y[i] /= nrm;
  }
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// ----------------------------------------------------------------------------
// the fused streaming kernel
//   PHASE 0: coef_i = <v_i, w>              (i < nv), nrm2 = |w|^2; alpha_j = Re coef_j
//   PHASE 1: w -= sum coef_i v_i; coef_i = <v_i, w>; alpha_j += Re coef_j
//   PHASE 2: w -= sum coef_i v_i; beta_j = |w|; convergence check
// nv < 0: the device-looped solve; nv = st->j + 1, and PHASE 0 (the first kernel after
// the matvec) adds the matvec's time since st->t_mark to st->mv_ns
// ----------------------------------------------------------------------------
template <typename T, int PHASE>
__global__ void __launch_bounds__(VEC_THREADS)
    lz_pass_kernel(const T* __restrict__ V, int nv, ll n, T* __restrict__ w, LanczosDev* st,
                   double* part, unsigned* counter, int kmax) {
  if (*((volatile int*)&st->done)) return;
  if (nv < 0) {
    if (PHASE == 0 && blockIdx.x == 0 && threadIdx.x == 0) st->mv_ns += global_ns() - st->t_mark;
    nv = st->j + 1;
  }
  constexpr bool CPLX = ST<T>::cplx;
  constexpr int NW = VEC_THREADS / 32;
  __shared__ T ws[MAX_CHUNK];
  __shared__ double csh[2 * (KRYLOV_CAP + 1)];
  __shared__ double red[32];
  const int nblk = gridDim.x;
  const ll ch = (n + nblk - 1) / nblk;
  const ll x0 = (ll)blockIdx.x * ch;
  const ll x1 = (x0 + ch < n) ? x0 + ch : n;
  const int len = (x1 > x0) ? (int)(x1 - x0) : 0;
  const int ncoef = (PHASE == 2) ? 0 : nv;

  if (PHASE >= 1) {
    for (int i = threadIdx.x; i < 2 * nv; i += blockDim.x) csh[i] = st->coef[i];
    __syncthreads();
  }
  double ww = 0.0;
  for (int x = threadIdx.x; x < len; x += blockDim.x) {
    T v = w[x0 + x];
    if (PHASE >= 1) {
      for (int i = 0; i < nv; ++i) {
        T c = ST<T>::make(csh[2 * i], csh[2 * i + 1]);
        v = v - ST<T>::mul(c, V[(ll)i * n + x0 + x]);
      }
      w[x0 + x] = v;
    }
    ws[x] = v;
    ww += ST<T>::abs2(v);
  }
  __syncthreads();
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int i = wid; i < ncoef; i += NW) {
    const T* vi = V + (ll)i * n + x0;
    double sr = 0.0, si = 0.0;
    for (int x = lane; x < len; x += 32) {
      T p = ST<T>::cmul(vi[x], ws[x]);
      sr += ST<T>::re(p);
      if (CPLX) si += ST<T>::im(p);
    }
    sr = warp_sum(sr);
    if (CPLX) si = warp_sum(si);
    if (lane == 0) {  // partials are coefficient-major: part[idx][block]
      part[(ll)(2 * i) * nblk + blockIdx.x] = sr;
      part[(ll)(2 * i + 1) * nblk + blockIdx.x] = si;
    }
  }
  ww = block_sum(ww, red);
  if (threadIdx.x == 0) part[(ll)(2 * nv) * nblk + blockIdx.x] = ww;

  if (!arrive_last(counter, nblk)) return;

  // ---- finalize (last block): deterministic fixed-order sums, one warp per coefficient
  //      (lane l adds blocks l, l+32, ... in order, then a fixed shuffle tree)
  for (int c = wid; c < 2 * ncoef + 1; c += NW) {
    const int idx = (c == 2 * ncoef) ? 2 * nv : c;
    const double* pc = part + (ll)idx * nblk;
    double s = 0.0;
    for (int b = lane; b < nblk; b += 32) s += pc[b];
    s = warp_sum(s);
    if (lane == 0) {
      if (c == 2 * ncoef) st->nrm2 = s;
      else st->coef[c] = s;
    }
  }
  __syncthreads();
  __threadfence_block();
  const int j = nv - 1;
  if (PHASE == 0) {
    if (threadIdx.x == 0) st->alpha[j] = st->coef[2 * j];
  } else if (PHASE == 1) {
    if (threadIdx.x == 0) st->alpha[j] += st->coef[2 * j];
  } else {
    __shared__ int done_s;
    __shared__ double tv_work[5 * KRYLOV_CAP];
    if (threadIdx.x == 0) {
      double b = sqrt(fmax(st->nrm2, 0.0));
      st->beta[j] = b;
    }
    __syncthreads();
    const int k = j + 1;
    double lam = tridiag_lowest(st->alpha, st->beta, k, st->e_prev);
    if (threadIdx.x == 0) {
      st->e_cur = lam;
      bool conv = (k >= 3) && (fabs(lam - st->e_prev) < st->tol);
      bool brk = st->beta[j] < 1e-14;
      bool full = (k >= kmax);
      st->e_prev = lam;
      done_s = (conv || brk || full) ? 1 : 0;
      if (done_s) {
        st->converged = (conv || brk) ? 1 : 0;
        st->n_iter = k;
        tridiag_vector(st->alpha, st->beta, k, lam, st->ritz, tv_work);
        __threadfence();
        st->done = 1;
      }
    }
  }
  if (threadIdx.x == 0) *counter = 0u;
}

template <typename T>
__global__ void lz_normalize_kernel(T* __restrict__ vnext, const T* __restrict__ w, ll n,
                                    LanczosDev* st) {
  if (*((volatile int*)&st->done)) return;
  double inv = 1.0 / sqrt(st->nrm2);
  for (ll x = (ll)blockIdx.x * blockDim.x + threadIdx.x; x < n; x += (ll)gridDim.x * blockDim.x)
    vnext[x] = ST<T>::scale(inv, w[x]);
}

// device-looped form: v_(j+1) = w / |w| into V[j + 1] and into cur, j = st->j
template <typename T>
__global__ void lz_normalize_dev_kernel(T* __restrict__ V, T* __restrict__ cur, const T* __restrict__ w,
                                        ll n, LanczosDev* st) {
  if (*((volatile int*)&st->done)) return;
  const int j1 = st->j + 1;
  if (j1 >= st->kmax) return;
  double inv = 1.0 / sqrt(st->nrm2);
  T* vnext = V + (ll)j1 * n;
  for (ll x = (ll)blockIdx.x * blockDim.x + threadIdx.x; x < n; x += (ll)gridDim.x * blockDim.x) {
    const T v = ST<T>::scale(inv, w[x]);
    vnext[x] = v;
    cur[x] = v;
  }
}

// last node of the device loop's body (one thread)
__global__ void lz_loop_next_kernel(LanczosDev* st, cudaGraphConditionalHandle h, int kmax) {
  const int g = st->guard + 1;
  st->guard = g;
  const int done = *((volatile int*)&st->done);
  if (!done) st->j += 1;
  st->t_mark = global_ns();
  cudaGraphSetConditional(h, (!done && g < kmax) ? 1u : 0u);
}

// |x|^2 into st->nrm2 (or out), last-block finalize
template <typename T>
__global__ void norm2_kernel(const T* __restrict__ x, ll n, double* out, double* part,
                             unsigned* counter) {
  __shared__ double red[32];
  double s = 0.0;
  for (ll i = (ll)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (ll)gridDim.x * blockDim.x)
    s += ST<T>::abs2(x[i]);
  s = block_sum(s, red);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
  if (!arrive_last(counter, gridDim.x)) return;
  if (threadIdx.x < 32) {  // fixed order: lane l adds blocks l, l+32, ..., then a shuffle tree
    double t = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += 32) t += part[b];
    t = warp_sum(t);
    if (threadIdx.x == 0) {
      *out = t;
      *counter = 0u;
    }
  }
}

__device__ inline double hash_uniform(unsigned long long x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  x ^= x >> 31;
  return (double)(x >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
}

// reset solver state; if |theta| is ~0, replace theta by a seeded random vector
template <typename T>
__global__ void lz_reset_kernel(T* theta, ll n, LanczosDev* st, unsigned seed, double tol, int kmax,
                                const unsigned* seed_dev) {
  if (seed_dev) seed = *seed_dev;
  const bool tiny = !(st->nrm2 >= 1e-28);
  if (tiny) {
    for (ll x = (ll)blockIdx.x * blockDim.x + threadIdx.x; x < n; x += (ll)gridDim.x * blockDim.x) {
      double r = hash_uniform(((unsigned long long)seed << 32) ^ (unsigned long long)(2 * x));
      double i = ST<T>::cplx ? hash_uniform(((unsigned long long)seed << 32) ^ (2 * x + 1)) : 0.0;
      theta[x] = ST<T>::make(r, i);
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->randomized = tiny ? 1 : 0;
    st->done = 0;
    st->converged = 0;
    st->n_iter = 0;
    st->e_prev = 1e300;
    st->e_cur = 0.0;
    st->tol = tol;
    st->kmax = kmax;
    st->j = 0;
    st->guard = 0;
    st->t_mark = 0ull;
    st->mv_ns = 0ull;
  }
}

template <typename T>
__global__ void lz_v0_kernel(const T* __restrict__ theta, T* __restrict__ v0, ll n, LanczosDev* st,
                             T* __restrict__ cur) {
  double inv = 1.0 / sqrt(st->nrm2);
  for (ll x = (ll)blockIdx.x * blockDim.x + threadIdx.x; x < n; x += (ll)gridDim.x * blockDim.x) {
    const T v = ST<T>::scale(inv, theta[x]);
    v0[x] = v;
    if (cur) cur[x] = v;
  }
  if (cur && blockIdx.x == 0 && threadIdx.x == 0) st->t_mark = global_ns();
}

template <typename T>
__global__ void lz_ritz_kernel(const T* __restrict__ V, ll n, T* __restrict__ out,
                               const LanczosDev* st) {
  __shared__ double r[KRYLOV_CAP];
  const int k = st->n_iter;
  for (int i = threadIdx.x; i < k; i += blockDim.x) r[i] = st->ritz[i];
  __syncthreads();
  for (ll x = (ll)blockIdx.x * blockDim.x + threadIdx.x; x < n; x += (ll)gridDim.x * blockDim.x) {
    T acc = ST<T>::zero();
    for (int i = 0; i < k; ++i) acc = acc + ST<T>::scale(r[i], V[(ll)i * n + x]);
    out[x] = acc;
  }
}

template <typename T>
__global__ void scale_by_inv_sqrt_kernel(T* x, ll n, const double* nrm2) {
  double s = *nrm2;
  double inv = (s > 0.0) ? 1.0 / sqrt(s) : 0.0;
  for (ll i = (ll)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (ll)gridDim.x * blockDim.x)
    x[i] = ST<T>::scale(inv, x[i]);
}

static int grid_for(ll n) {
  ll g = (n + VEC_THREADS - 1) / VEC_THREADS;
  if (g > 148 * 8) g = 148 * 8;
  if (g < 1) g = 1;
  return (int)g;
}

template <typename T>
void lz_dots(const T* V, int nv, ll n, const T* w, LanczosDev* st, RedScratch& r, cudaStream_t s) {
  lz_pass_kernel<T, 0><<<vec_blocks(n), VEC_THREADS, 0, s>>>(V, nv, n, const_cast<T*>(w), st,
                                                             r.part, r.counter, 0);
  DMRG2_CHECK_LAUNCH();
}
template <typename T>
void lz_update_dots(const T* V, int nv, ll n, T* w, LanczosDev* st, RedScratch& r, cudaStream_t s) {
  lz_pass_kernel<T, 1><<<vec_blocks(n), VEC_THREADS, 0, s>>>(V, nv, n, w, st, r.part, r.counter, 0);
  DMRG2_CHECK_LAUNCH();
}
template <typename T>
void lz_update_norm_check(const T* V, int nv, ll n, T* w, LanczosDev* st, RedScratch& r, int j,
                          int kmax, cudaStream_t s) {
  (void)j;
  lz_pass_kernel<T, 2><<<vec_blocks(n), VEC_THREADS, 0, s>>>(V, nv, n, w, st, r.part, r.counter,
                                                             kmax);
  DMRG2_CHECK_LAUNCH();
}
template <typename T>
void lz_normalize_next(T* vnext, const T* w, ll n, LanczosDev* st, cudaStream_t s) {
  lz_normalize_kernel<T><<<grid_for(n), VEC_THREADS, 0, s>>>(vnext, w, n, st);
  DMRG2_CHECK_LAUNCH();
}

template <typename T>
void norm2(const T* x, ll n, double* out_dev, RedScratch& r, cudaStream_t s) {
  int g = grid_for(n);
  if (g > r.nblk) g = r.nblk;
  norm2_kernel<T><<<g, VEC_THREADS, 0, s>>>(x, n, out_dev, r.part, r.counter);
  DMRG2_CHECK_LAUNCH();
}

template <typename T>
void lz_start(T* theta, T* v0, ll n, LanczosDev* st, RedScratch& r, unsigned seed, double tol,
              int kmax, cudaStream_t s, T* cur, const unsigned* seed_dev) {
  norm2<T>(theta, n, &st->nrm2, r, s);
  lz_reset_kernel<T><<<grid_for(n), VEC_THREADS, 0, s>>>(theta, n, st, seed, tol, kmax, seed_dev);
  DMRG2_CHECK_LAUNCH();
  norm2<T>(theta, n, &st->nrm2, r, s);
  lz_v0_kernel<T><<<grid_for(n), VEC_THREADS, 0, s>>>(theta, v0, n, st, cur);
  DMRG2_CHECK_LAUNCH();
}

template <typename T>
void lz_step_dev(const T* V, ll n, T* w, T* cur, LanczosDev* st, RedScratch& r, int kmax, cudaStream_t s) {
  lz_pass_kernel<T, 0><<<vec_blocks(n), VEC_THREADS, 0, s>>>(V, -1, n, w, st, r.part, r.counter, 0);
  DMRG2_CHECK_LAUNCH();
  lz_pass_kernel<T, 1><<<vec_blocks(n), VEC_THREADS, 0, s>>>(V, -1, n, w, st, r.part, r.counter, 0);
  DMRG2_CHECK_LAUNCH();
  lz_pass_kernel<T, 2><<<vec_blocks(n), VEC_THREADS, 0, s>>>(V, -1, n, w, st, r.part, r.counter, kmax);
  DMRG2_CHECK_LAUNCH();
  lz_normalize_dev_kernel<T><<<grid_for(n), VEC_THREADS, 0, s>>>(const_cast<T*>(V), cur, w, n, st);
  DMRG2_CHECK_LAUNCH();
}

void lz_loop_next(LanczosDev* st, cudaGraphConditionalHandle h, int kmax, cudaStream_t s) {
  lz_loop_next_kernel<<<1, 1, 0, s>>>(st, h, kmax);
  DMRG2_CHECK_LAUNCH();
}

template <typename T>
void lz_ritz(const T* V, ll n, T* out, LanczosDev* st, RedScratch& r, cudaStream_t s) {
  lz_ritz_kernel<T><<<grid_for(n), VEC_THREADS, 0, s>>>(V, n, out, st);
  DMRG2_CHECK_LAUNCH();
  norm2<T>(out, n, &st->nrm2, r, s);
  scale_by_inv_sqrt_kernel<T><<<grid_for(n), VEC_THREADS, 0, s>>>(out, n, &st->nrm2);
  DMRG2_CHECK_LAUNCH();
}

template <typename T>
void scale_inplace(T* x, ll n, const double* nrm2_dev, cudaStream_t s) {
  scale_by_inv_sqrt_kernel<T><<<grid_for(n), VEC_THREADS, 0, s>>>(x, n, nrm2_dev);
  DMRG2_CHECK_LAUNCH();
}

#define INST(T)                                                                                   \
  template void lz_dots<T>(const T*, int, ll, const T*, LanczosDev*, RedScratch&, cudaStream_t); \
  template void lz_update_dots<T>(const T*, int, ll, T*, LanczosDev*, RedScratch&, cudaStream_t);\
  template void lz_update_norm_check<T>(const T*, int, ll, T*, LanczosDev*, RedScratch&, int, int,\
                                        cudaStream_t);                                            \
  template void lz_normalize_next<T>(T*, const T*, ll, LanczosDev*, cudaStream_t);                \
  template void lz_start<T>(T*, T*, ll, LanczosDev*, RedScratch&, unsigned, double, int,      \
                            cudaStream_t, T*, const unsigned*);                                   \
  template void lz_step_dev<T>(const T*, ll, T*, T*, LanczosDev*, RedScratch&, int, cudaStream_t); \
  template void lz_ritz<T>(const T*, ll, T*, LanczosDev*, RedScratch&, cudaStream_t);             \
  template void norm2<T>(const T*, ll, double*, RedScratch&, cudaStream_t);                       \
  template void scale_inplace<T>(T*, ll, const double*, cudaStream_t);
INST(double)
INST(zc)
#undef INST

}  // namespace dmrg2
