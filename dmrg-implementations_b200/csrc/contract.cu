#include "contract.cuh"

#include <algorithm>
#include <cstring>
#include <stdexcept>

namespace dmrg2 {

// Y[a][o][e] = sum_k W[o][k] X[a][k][e] for Kin, Kout <= KM (the two-site MPO
// mixing of H_eff step 2 when D d^2 is small): one thread per (a, e), the Kin
// inputs in registers, W in shared memory. Bandwidth-bound: X read once, Y
// written once.
template <typename T, int KM>
__global__ void __launch_bounds__(128)
    mpo_mix_kernel(const T* __restrict__ X, const T* __restrict__ W, T* __restrict__ Y, int Kin,
                   int Kout, int cR, ll sX, ll sY, const int* skip) {
  if (skip && *((volatile const int*)skip)) return;
  __shared__ T Ws[KM * KM];
  for (int i = threadIdx.x; i < KM * KM; i += blockDim.x) {
    const int o = i / KM, k = i % KM;
    Ws[i] = (o < Kout && k < Kin) ? W[(ll)o * Kin + k] : ST<T>::zero();
  }
  __syncthreads();
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= cR) return;
  const ll a = blockIdx.y;
  const T* xa = X + a * sX + e;
  T* ya = Y + a * sY + e;
  T xin[KM];
#pragma unroll
  for (int k = 0; k < KM; ++k) xin[k] = (k < Kin) ? xa[(ll)k * cR] : ST<T>::zero();
  for (int o = 0; o < Kout; ++o) {
    T acc = ST<T>::zero();
#pragma unroll
    for (int k = 0; k < KM; ++k) acc = acc + ST<T>::mul(Ws[o * KM + k], xin[k]);
    ya[(ll)o * cR] = acc;
  }
}

// The same mixing with W in its nonzero form (row starts, ascending columns, values; Kin,
// Kout <= 32 and at most MIX_SPARSE_NNZ nonzeros): each output sums only its row's
// nonzeros, in the order of the dense loop above (whose other terms are exact zeros). A
// thread first loads its Kin inputs together (a static loop, as the dense kernel does)
// into its own column of shared memory, so the sums read shared memory, not L2.
constexpr int MIX_SPARSE_NNZ = 512;
constexpr int MIX_SPARSE_NT = 64;
template <typename T>
__global__ void __launch_bounds__(MIX_SPARSE_NT)
    mpo_mix_sparse_kernel(const T* __restrict__ X, const T* __restrict__ val, const int* __restrict__ rowp,
                          T* __restrict__ Y, int Kin, int Kout, int cR, ll sX, ll sY, const int* skip) {
  if (skip && *((volatile const int*)skip)) return;
  constexpr int KM = 32, NT = MIX_SPARSE_NT;
  __shared__ int rp[KM + 1];
  __shared__ int cs[MIX_SPARSE_NNZ];
  __shared__ T vs[MIX_SPARSE_NNZ];
  __shared__ T xs[KM * NT];  // xs[k][thread]
  const int tid = threadIdx.x;
  for (int i = tid; i <= Kout; i += NT) rp[i] = rowp[i];
  __syncthreads();
  const int nnz = min(rp[Kout], MIX_SPARSE_NNZ);
  const int* col = rowp + Kout + 1;
  for (int i = tid; i < nnz; i += NT) {
    cs[i] = col[i];
    vs[i] = val[i];
  }
  __syncthreads();
  const int e = blockIdx.x * NT + tid;
  if (e >= cR) return;
  const ll a = blockIdx.y;
  const T* xa = X + a * sX + e;
  T* ya = Y + a * sY + e;
#pragma unroll
  for (int k = 0; k < KM; ++k)
    if (k < Kin) xs[k * NT + tid] = xa[(ll)k * cR];
  for (int o = 0; o < Kout; ++o) {
    T acc = ST<T>::zero();
    const int j1 = min(rp[o + 1], nnz);
    for (int j = rp[o]; j < j1; ++j) acc = acc + ST<T>::mul(vs[j], xs[cs[j] * NT + tid]);
    ya[(ll)o * cR] = acc;
  }
}

template <typename T>
int wwt_sparse_block(std::vector<T>& w, int Kin, int Kout) {
  const ll kk = (ll)Kin * Kout;
  if ((ll)w.size() != kk) throw std::invalid_argument("wwt_sparse_block: dense matrix of the wrong size");
  std::vector<T> val((size_t)kk, ST<T>::zero());
  std::vector<int> ints((size_t)(Kout + 1 + kk), 0);
  int nnz = 0;
  for (int o = 0; o < Kout; ++o) {
    ints[(size_t)o] = nnz;
    for (int k = 0; k < Kin; ++k) {
      const T v = w[(size_t)o * Kin + k];
      if (ST<T>::abs2(v) != 0.0) {
        val[(size_t)nnz] = v;
        ints[(size_t)(Kout + 1 + nnz)] = k;
        ++nnz;
      }
    }
  }
  ints[(size_t)Kout] = nnz;
  const ll total = wwt_block_elems(Kin, Kout, sizeof(T));
  w.resize((size_t)total, ST<T>::zero());
  std::copy(val.begin(), val.end(), w.begin() + kk);
  std::memcpy(w.data() + 2 * kk, ints.data(), sizeof(int) * ints.size());
  return nnz;
}

// step 2 of the matvec: Y[a] = W X[a] for every a (MPO mixing, FP64); X[a] is Kin x cR,
// Y[a] is Kout x cR; wsp: W's nonzero form (wwt_sparse_block), or null
template <typename T>
static void mix_rows(const T* X, const T* W, T* Y, int cL, int cR, int Kin, int Kout, const int* skip,
                     cudaStream_t s, const T* wsp = nullptr) {
  if (wsp && Kin <= 32 && Kout <= 32 && 2 * Kin * Kout <= 2 * MIX_SPARSE_NNZ && cL <= 65535) {
    // (the engine uses the nonzero form only where nnz <= Kin Kout / 2 <= MIX_SPARSE_NNZ)
    const ll kk = (ll)Kin * Kout;
    dim3 grid(ceil_div(cR, MIX_SPARSE_NT), cL);
    mpo_mix_sparse_kernel<T><<<grid, MIX_SPARSE_NT, 0, s>>>(X, wsp, (const int*)(wsp + kk), Y, Kin, Kout, cR,
                                                            (ll)Kin * cR, (ll)Kout * cR, skip);
    DMRG2_CHECK_LAUNCH();
  } else if (Kin <= 32 && Kout <= 32 && cL <= 65535) {
    dim3 grid(ceil_div(cR, 128), cL);
    mpo_mix_kernel<T, 32><<<grid, 128, 0, s>>>(X, W, Y, Kin, Kout, cR, (ll)Kin * cR, (ll)Kout * cR, skip);
    DMRG2_CHECK_LAUNCH();
  } else {
    Gemm<T> g;
    g.M = Kout; g.N = cR; g.K = Kin;
    g.A = W; g.lda = Kin; g.sA1 = 0;
    g.B = X; g.ldb = cR; g.sB1 = (ll)Kin * cR;
    g.C = Y; g.ldc = cR; g.sC1 = (ll)Kout * cR;
    g.nb1 = cL; g.skip = skip;
    launch_gemm(g, s);
  }
}

template <typename T>
void heff_apply_split(const T* Lenv, const T* Renv, const T* WWt, const T* in, T* out, T* X, T* Y, int cL,
                      int cR, int d, int Dl, int Dr, SplitScratch& ws, const int* skip, cudaStream_t s) {
  const ll dd = (ll)d * d;
  const T one = ST<T>::one(), zero = ST<T>::zero();
  // step 1: X[a][w][.] = L[a][w][:] theta, Dl batches sharing theta
  gemm_bf16x3<T>(0, 0, cL, (int)(dd * cR), cL, one, Lenv, (ll)Dl * cL, cL, in, dd * cR, 0, zero, X,
                 (ll)Dl * dd * cR, dd * cR, Dl, ws, s, skip);
  mix_rows(X, WWt, Y, cL, cR, (int)(Dl * dd), (int)(dd * Dr), skip, s);
  // step 3: out[(a,p,q)][f] = sum_(n,e) Y[(a,p,q)][(n,e)] R[f][(n,e)]
  gemm_bf16x3<T>(0, 1, (int)(cL * dd), cR, Dr * cR, one, Y, (ll)Dr * cR, 0, Renv, (ll)Dr * cR, 0, zero, out, cR,
                 0, 1, ws, s, skip);
}

template <typename T>
void heff_apply(const T* Lenv, const T* Renv, const T* WWt, const T* in, T* out, T* X, T* Y, int cL,
                int cR, int d, int Dl, int Dr, const int* skip, cudaStream_t s, const T* wsp) {
  const ll dd = (ll)d * d;
  {
    Gemm<T> g;
    g.M = cL; g.N = (int)(dd * cR); g.K = cL;
    g.A = Lenv; g.lda = (ll)Dl * cL; g.sA1 = cL;
    g.B = in; g.ldb = dd * cR; g.sB1 = 0;
    g.C = X; g.ldc = (ll)Dl * dd * cR; g.sC1 = dd * cR;
    g.nb1 = Dl; g.skip = skip;
    launch_gemm(g, s);
  }
  mix_rows(X, WWt, Y, cL, cR, (int)(Dl * dd), (int)(dd * Dr), skip, s, wsp);
  {
    Gemm<T> g;
    g.tb = true;
    g.M = (int)(cL * dd); g.N = cR; g.K = Dr * cR;
    g.A = Y; g.lda = (ll)Dr * cR;
    g.B = Renv; g.ldb = (ll)Dr * cR;
    g.C = out; g.ldc = cR;
    g.skip = skip;
    // split K when the output tiles cannot fill the GPU; X is free again and
    // holds Dl * cL * d^2 * cR >= splitk * cL * d^2 * cR partial products
    const int tiles = ceil_div(g.M, GemmTile<T>::BM) * ceil_div(g.N, GemmTile<T>::BN);
    int sk = 1;
    while (sk < Dl && sk < 8 && tiles * sk < 2 * 148 && (ll)g.K / (sk * 2) >= 4 * GemmTile<T>::BK) sk *= 2;
    if (sk > Dl) sk = Dl;
    if (sk > 1) {
      g.splitk = sk;
      g.ws = X;
    }
    launch_gemm(g, s);
  }
}

template <typename T>
void heff1_apply(const T* Lenv, const T* Renv, const T* WmixL, const T* in, T* out, T* X, T* Y, int cL, int cR,
                 int d, int Dl, int Dr, const int* skip, cudaStream_t s) {
  {
    Gemm<T> g;  // X[a][w][(s,e)] = sum_c L[a][w][c] A[c][(s,e)]
    g.M = cL; g.N = d * cR; g.K = cL;
    g.A = Lenv; g.lda = (ll)Dl * cL; g.sA1 = cL;
    g.B = in; g.ldb = (ll)d * cR; g.sB1 = 0;
    g.C = X; g.ldc = (ll)Dl * d * cR; g.sC1 = (ll)d * cR;
    g.nb1 = Dl; g.skip = skip;
    launch_gemm(g, s);
  }
  mix_rows(X, WmixL, Y, cL, cR, Dl * d, d * Dr, skip, s);  // Y[a][(t,w')][e]
  {
    Gemm<T> g;  // out[(a,t)][f] = sum_(w',e) Y[(a,t)][(w',e)] R[f][(w',e)]
    g.tb = true;
    g.M = cL * d; g.N = cR; g.K = Dr * cR;
    g.A = Y; g.lda = (ll)Dr * cR;
    g.B = Renv; g.ldb = (ll)Dr * cR;
    g.C = out; g.ldc = cR;
    g.skip = skip;
    const int tiles = ceil_div(g.M, GemmTile<T>::BM) * ceil_div(g.N, GemmTile<T>::BN);
    int sk = 1;
    while (sk < Dl && sk < 8 && tiles * sk < 2 * 148 && (ll)g.K / (sk * 2) >= 4 * GemmTile<T>::BK) sk *= 2;
    if (sk > Dl) sk = Dl;
    if (sk > 1) {
      g.splitk = sk;
      g.ws = X;  // X holds Dl * cL * d * cR >= splitk * cL * d * cR partial products
    }
    launch_gemm(g, s);
  }
}

double heff1_flops(int cL, int cR, int d, int Dl, int Dr, bool cplx) {
  const double f = 2.0 * Dl * cL * ((double)d * cR) * cL + 2.0 * cL * ((double)d * Dr) * cR * ((double)Dl * d) +
                   2.0 * ((double)cL * d) * cR * ((double)Dr * cR);
  return cplx ? 4.0 * f : f;
}

double heff_flops(int cL, int cR, int d, int Dl, int Dr, bool cplx) {
  double dd = (double)d * d;
  double f = 2.0 * Dl * cL * (dd * cR) * cL + 2.0 * cL * (dd * Dr) * cR * (Dl * dd) +
             2.0 * (cL * dd) * cR * ((double)Dr * cR);
  return cplx ? 4.0 * f : f;
}

double env_flops(int ci, int co, int d, int Dl, int Dr, bool cplx) {
  double f = 2.0 * ((double)ci * Dl) * ((double)d * co) * ci + 2.0 * ci * ((double)d * Dr) * co * (Dl * d) +
             2.0 * co * ((double)Dr * co) * ((double)ci * d);
  return cplx ? 4.0 * f : f;
}

// split the K range of an environment GEMM over CTAs when its output tiles do not fill
// the GPU, with ws (room for ws_elems elements) as the partial-product workspace
template <typename T>
static void env_splitk(Gemm<T>& g, ll ws_elems, T* ws) {
  const int tiles = ceil_div(g.M, GemmTile<T>::BM) * ceil_div(g.N, GemmTile<T>::BN);
  int sk = 1;
  while (sk < 8 && tiles * sk < 148 && (ll)g.K / (2 * sk) >= 4 * GemmTile<T>::BK &&
         (ll)(2 * sk) * g.M * g.N <= ws_elems)
    sk *= 2;
  if (sk > 1) {
    g.splitk = sk;
    g.ws = ws;
  }
}

template <typename T>
void env_left(const T* Lenv, const T* A, const T* WmixL, T* Lnew, T* X, T* Y, int cL, int cO, int d,
              int Dl, int Dr, cudaStream_t s) {
  {
    Gemm<T> g;
    g.M = cL * Dl; g.N = d * cO; g.K = cL;
    g.A = Lenv; g.lda = cL;
    g.B = A; g.ldb = (ll)d * cO;
    g.C = X; g.ldc = (ll)d * cO;
    launch_gemm(g, s);
  }
  // Y[a] = WmixL X[a] for every a: the MPO mixing, a (d Dr) x (Dl d) matrix (a batched GEMM
  // of tiny matrices wastes most of each tensor-core tile: 13 us at chi = 256 against ~5)
  mix_rows(X, WmixL, Y, cL, cO, Dl * d, d * Dr, nullptr, s);
  {
    Gemm<T> g;
    g.ta = true; g.ca = true;
    g.M = cO; g.N = Dr * cO; g.K = cL * d;
    g.A = A; g.lda = cO;
    g.B = Y; g.ldb = (ll)Dr * cO;
    g.C = Lnew; g.ldc = (ll)Dr * cO;
    // K split when the output tiles cannot fill the GPU; X (free again) holds the
    // cL Dl d cO products of step 1
    env_splitk(g, (ll)cL * Dl * d * cO, X);
    launch_gemm(g, s);
  }
}

template <typename T>
void env_right(const T* Renv, const T* B, const T* WmixR, T* Rnew, T* X, T* Y, int cI, int cO,
               int d, int Dl, int Dr, cudaStream_t s) {
  {
    Gemm<T> g;
    g.tb = true;
    g.M = cI * Dr; g.N = cO; g.K = cI;
    g.A = Renv; g.lda = cI; g.sA1 = 0;
    g.B = B; g.ldb = (ll)d * cI; g.sB1 = cI;
    g.C = X; g.ldc = (ll)d * cO; g.sC1 = cO;
    g.nb1 = d;
    launch_gemm(g, s);
  }
  // Y[s][a] = WmixR[s] X[a] for every a and physical index s (MPO mixing, Dl x (Dr d))
  for (int sp = 0; sp < d; ++sp)
    mix_rows(X, WmixR + (ll)sp * Dl * Dr * d, Y + (ll)sp * cI * Dl * cO, cI, cO, Dr * d, Dl, nullptr, s);
  {
    Gemm<T> g;
    g.ca = true;
    g.M = cO; g.N = Dl * cO; g.K = d * cI;
    g.A = B; g.lda = (ll)d * cI;
    g.B = Y; g.ldb = (ll)Dl * cO;
    g.C = Rnew; g.ldc = (ll)Dl * cO;
    env_splitk(g, (ll)cI * Dr * d * cO, X);  // X holds the cI Dr d cO products of step 1
    launch_gemm(g, s);
  }
}

template <typename T>
void theta_form(const T* A, const T* B, T* theta, int cL, int cM, int cR, int d, cudaStream_t s, T* ws,
                ll ws_elems) {
  Gemm<T> g;
  g.M = cL * d; g.N = d * cR; g.K = cM;
  g.A = A; g.lda = cM;
  g.B = B; g.ldb = (ll)d * cR;
  g.C = theta; g.ldc = (ll)d * cR;
  if (ws) env_splitk(g, ws_elems, ws);
  launch_gemm(g, s);
}

template <typename T>
void build_wwt(const T* WL, const T* WR, int Dl, int Dm, int Dr, int d, std::vector<T>& out) {
  // WWt[(p,q,n)][(w,s,r)] = sum_m WL[w][m][s][p] WR[m][n][r][q]
  const int rows = d * d * Dr, cols = Dl * d * d;
  out.assign((size_t)rows * cols, ST<T>::zero());
  for (int p = 0; p < d; ++p)
    for (int q = 0; q < d; ++q)
      for (int n = 0; n < Dr; ++n)
        for (int w = 0; w < Dl; ++w)
          for (int s = 0; s < d; ++s)
            for (int r = 0; r < d; ++r) {
              T acc = ST<T>::zero();
              for (int m = 0; m < Dm; ++m) {
                T a = WL[(((size_t)w * Dm + m) * d + s) * d + p];
                T b = WR[(((size_t)m * Dr + n) * d + r) * d + q];
                acc = acc + ST<T>::mul(a, b);
              }
              size_t row = ((size_t)p * d + q) * Dr + n;
              size_t col = ((size_t)w * d + s) * d + r;
              out[row * cols + col] = acc;
            }
}

template <typename T>
void build_wmix_left(const T* W, int Dl, int Dr, int d, std::vector<T>& out) {
  // WmixL[(t,w')][(w,s)] = W[w][w'][s][t]
  const int rows = d * Dr, cols = Dl * d;
  out.assign((size_t)rows * cols, ST<T>::zero());
  for (int t = 0; t < d; ++t)
    for (int wp = 0; wp < Dr; ++wp)
      for (int w = 0; w < Dl; ++w)
        for (int s = 0; s < d; ++s)
          out[((size_t)t * Dr + wp) * cols + (size_t)w * d + s] = W[(((size_t)w * Dr + wp) * d + s) * d + t];
}

template <typename T>
void build_wmix_right(const T* W, int Dl, int Dr, int d, std::vector<T>& out) {
  // WmixR[t][w'][(w,s)] = W[w'][w][s][t]   (w' left index in Dl, w right index in Dr)
  const int cols = Dr * d;
  out.assign((size_t)d * Dl * cols, ST<T>::zero());
  for (int t = 0; t < d; ++t)
    for (int wp = 0; wp < Dl; ++wp)
      for (int w = 0; w < Dr; ++w)
        for (int s = 0; s < d; ++s)
          out[((size_t)t * Dl + wp) * cols + (size_t)w * d + s] = W[(((size_t)wp * Dr + w) * d + s) * d + t];
}

#define INST(T)                                                                                 \
  template void heff_apply<T>(const T*, const T*, const T*, const T*, T*, T*, T*, int, int, int, \
                              int, int, const int*, cudaStream_t, const T*);                     \
  template int wwt_sparse_block<T>(std::vector<T>&, int, int);                                  \
  template void heff1_apply<T>(const T*, const T*, const T*, const T*, T*, T*, T*, int, int, int,  \
                               int, int, const int*, cudaStream_t);                              \
  template void heff_apply_split<T>(const T*, const T*, const T*, const T*, T*, T*, T*, int, int,   \
                                    int, int, int, SplitScratch&, const int*, cudaStream_t);     \
  template void env_left<T>(const T*, const T*, const T*, T*, T*, T*, int, int, int, int, int,  \
                            cudaStream_t);                                                       \
  template void env_right<T>(const T*, const T*, const T*, T*, T*, T*, int, int, int, int, int, \
                             cudaStream_t);                                                      \
  template void theta_form<T>(const T*, const T*, T*, int, int, int, int, cudaStream_t, T*, ll); \
  template void build_wwt<T>(const T*, const T*, int, int, int, int, std::vector<T>&);          \
  template void build_wmix_left<T>(const T*, int, int, int, std::vector<T>&);                   \
  template void build_wmix_right<T>(const T*, int, int, int, std::vector<T>&);
INST(double)
INST(zc)
#undef INST

}  // namespace dmrg2
