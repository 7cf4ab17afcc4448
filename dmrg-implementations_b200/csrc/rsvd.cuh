// Randomised truncated split of a two-site tensor (optional truncation mode): the
// range finder of Halko, Martinsson and Tropp (SIAM Review 53, 2011) without power
// iterations, as the reference's svd_split uses it (gpu-rocm/dmrg2-gpu/src/
// dmrg2_gpu_impl.h:1178-1266: r = min(k + 10, full_k) sketch columns, a fresh random
// test matrix per call, used when full_k > k + 10 and the sketched side is longer
// than 2k).
//
// The sketch is taken on the side that receives the isometry, so that the small
// eigenproblem has order r in both directions:
//   'R': Y = theta Omega (m x r), Q = orth(Y), B = Q^H theta (r x nt);
//        the density-matrix split of B gives U_s (r x k) and right = U_s^H B;
//        left = Q U_s.
//   'L': Y = theta^H Omega (nt x r), Q = orth(Y), B = theta Q (m x r);
//        the split of B gives left = B V_s and V_s^H (k x r); right = V_s^H Q^H.
// orth is shifted CholeskyQR followed by two plain CholeskyQR passes (Fukaya,
// Kannan, Nakatsukasa, Yamamoto and Yanagisawa, SIAM J. Sci. Comput. 42, 2020), on
// unit columns, with the tiled Cholesky and the row solve: a random sketch carries the
// whole spread of theta's singular values, which one plain pass cannot take. Complex
// sketches run the same real kernels on their real embedding with the column pairs
// (y_j, i y_j) interleaved: the triangular factor orthogonalises each y_j against a
// span that is closed under multiplication by i, so the even columns of the result
// are a complex-orthonormal basis. The discarded weight is the small split's plus the
// weight of theta outside span(Q).
#pragma once

#include "cholqr.cuh"
#include "truncate.cuh"

namespace dmrg2 {

constexpr int RSVD_OVERSAMPLE = 10;

// n entries uniform on [-1, 1) (real and imaginary parts independently), a function
// of (seed, index) only
template <typename T>
void rsvd_omega(T* om, ll n, unsigned long long seed, cudaStream_t s);
// real embedding of a complex column block and back (see above)
void embed_pairs(const zc* Y, ll len, int r, double* YR, cudaStream_t s);
void extract_pairs(const double* QR, ll len, int r, zc* Q, cudaStream_t s);

template <typename T>
struct RsvdWork {
  static constexpr int C = ST<T>::cplx ? 2 : 1;  // real columns per sketch column
  T* Om = nullptr;       // lmax x rmax test matrix
  T* Y = nullptr;        // lmax x rmax sketch, then its orthonormal basis (complex)
  double* Z1 = nullptr;  // CholeskyQR operands: C lmax x C rmax doubles each
  double* Z2 = nullptr;
  double* S = nullptr;   // Gram matrix / tiled factor, np x np
  double* cpart = nullptr;
  T* B = nullptr;        // projected theta, rmax x lmax
  T* F = nullptr;        // small factor, lmax x rmax
  double* nrm = nullptr;  // |theta|^2, |B|^2
  int* status = nullptr;
  double* h_nrm = nullptr;  // pinned
  int* h_status = nullptr;  // pinned
  int lmax = 0, rmax = 0, np = 0;
  size_t bytes = 0;
  std::vector<void*> owned;

  // orders the split can take: C r <= CHOL_MAX, C len <= 32 COLNORM_MAX_CHUNKS
  static int rcap() { return CHOL_MAX / C; }
  static int lcap() { return 32 * COLNORM_MAX_CHUNKS / C; }
  static size_t bytes_for(ll lmax, ll rmax) {
    lmax = std::max<ll>(lmax, 1);
    rmax = std::max<ll>(std::min<ll>(rmax, rcap()), 1);
    const ll np = chol_padded((int)(C * rmax));
    return sizeof(T) * (size_t)(4 * lmax * rmax) + sizeof(double) * (size_t)(2 * C * C * lmax * rmax + np * np) +
           sizeof(double) * (size_t)(COLNORM_MAX_CHUNKS * C * rmax + 2) + sizeof(int);
  }
  void* alloc(size_t b) {
    void* p = nullptr;
    p = dev_alloc(std::max<size_t>(b, 16));
    owned.push_back(p);
    bytes += b;
    return p;
  }
  void init(int lmax_, int rmax_) {
    lmax = std::max(lmax_, 1);
    rmax = std::max(std::min(rmax_, rcap()), 1);
    np = chol_padded(C * rmax);
    const size_t lr = (size_t)lmax * rmax;
    Om = (T*)alloc(sizeof(T) * lr);
    Y = (T*)alloc(sizeof(T) * lr);
    B = (T*)alloc(sizeof(T) * lr);
    F = (T*)alloc(sizeof(T) * lr);
    Z1 = (double*)alloc(sizeof(double) * C * C * lr);
    Z2 = (double*)alloc(sizeof(double) * C * C * lr);
    S = (double*)alloc(sizeof(double) * (size_t)np * np);
    cpart = (double*)alloc(sizeof(double) * (size_t)COLNORM_MAX_CHUNKS * C * rmax);
    nrm = (double*)alloc(sizeof(double) * 2);
    status = (int*)alloc(sizeof(int));
    h_nrm = (double*)host_pinned(sizeof(double) * 2);
    h_status = (int*)host_pinned(sizeof(int));
  }
  void release() {
    for (void* p : owned) dev_free(p);
    owned.clear();
    if (h_nrm) host_unpin(h_nrm);
    if (h_status) host_unpin(h_status);
    h_nrm = nullptr;
    h_status = nullptr;
  }
};

// the reference's condition for the randomised split, and the limits of the workspace
template <typename T>
inline bool rsvd_applies(const RsvdWork<T>& W, int m, int nt, char dir, int chi) {
  const int full_k = std::min(m, nt), k = std::min(chi, full_k);
  const int len = (dir == 'R') ? m : nt;
  const int r = std::min(k + RSVD_OVERSAMPLE, full_k);
  return W.rmax > 0 && full_k > k + RSVD_OVERSAMPLE && len > 2 * k && r <= W.rmax && len <= W.lmax &&
         len <= RsvdWork<T>::lcap() && std::max(m, nt) <= W.lmax;
}

// Randomised split of theta (m x nt, row-major) at bond cap chi with the absolute
// cutoff: writes left (m x k) and right (k x nt) as eig_split does and returns its
// summary with trunc_err covering the whole discarded weight; returns false (nothing
// written) when the CholeskyQR passes could not orthonormalise the sketch, and the
// caller then runs the exact split. The host waits twice.
template <typename T>
inline bool rsvd_split(RsvdWork<T>& W, EigWork<T>& ew, RedScratch& red, const T* theta, int m, int nt, char dir,
                       int chi, double cutoff, unsigned long long seed, T* left, T* right, SvdOut& o,
                       cudaStream_t s) {
  constexpr int C = RsvdWork<T>::C;
  const bool R = (dir == 'R');
  const int full_k = std::min(m, nt), k = std::min(chi, full_k);
  const int r = std::min(k + RSVD_OVERSAMPLE, full_k);
  const int len = R ? m : nt;
  if (!rsvd_applies(W, m, nt, dir, chi)) throw std::runtime_error("rsvd_split: shape outside the workspace");
  DMRG2_CUDA(cudaMemsetAsync(W.status, 0, sizeof(int), s));
  // Y = theta Omega ('R', Omega nt x r) or theta^H Omega ('L', Omega m x r)
  rsvd_omega<T>(W.Om, (ll)(R ? nt : m) * r, seed, s);
  {
    Gemm<T> g;
    g.M = len; g.N = r; g.K = R ? nt : m;
    g.A = theta; g.lda = nt;
    if (!R) { g.ta = true; g.ca = true; }
    g.B = W.Om; g.ldb = r;
    g.C = W.Y; g.ldc = r;
    launch_gemm(g, s);
  }
  // orthonormal basis of span(Y): unit columns, shifted CholeskyQR, two plain passes
  const ll rows = (ll)C * len;
  const int cols = C * r;
  const int np = chol_padded(cols);
  double* Z0;
  if constexpr (ST<T>::cplx) {
    embed_pairs(W.Y, len, r, W.Z1, s);
    Z0 = W.Z1;
  } else {
    Z0 = W.Y;
  }
  col_normalize(Z0, rows, cols, W.cpart, W.status, s);
  auto pass = [&](const double* Zin, double* Zout, double shift_rel, double rel_tol) {
    Gemm<double> g;
    g.ta = true;
    g.M = cols; g.N = cols; g.K = (int)rows;
    g.A = Zin; g.lda = cols;
    g.B = Zin; g.ldb = cols;
    g.C = W.S; g.ldc = np;
    launch_gemm(g, s);
    chol_tiles(W.S, cols, np, W.S, np, W.status, rel_tol, shift_rel, s);
    trsm_rows(Zin, rows, cols, W.S, np, Zout, W.status, s);
  };
  const double u = 1.1102230246251565e-16;
  pass(Z0, W.Z2, 11.0 * ((double)rows * cols + (double)cols * (cols + 1)) * u, 1e-10);
  pass(W.Z2, W.Z1, 0.0, 1e-13);
  pass(W.Z1, W.Z2, 0.0, 1e-13);
  const T* Q;
  if constexpr (ST<T>::cplx) {
    extract_pairs(W.Z2, len, r, W.Y, s);
    Q = W.Y;
  } else {
    Q = W.Z2;
  }
  DMRG2_CUDA(cudaMemcpyAsync(W.h_status, W.status, sizeof(int), cudaMemcpyDeviceToHost, s));
  DMRG2_CUDA(cudaStreamSynchronize(s));
  if (*W.h_status) return false;
  // B = Q^H theta ('R', r x nt) or theta Q ('L', m x r)
  {
    Gemm<T> g;
    if (R) {
      g.ta = true; g.ca = true;
      g.M = r; g.N = nt; g.K = m;
      g.A = Q; g.lda = r;
      g.B = theta; g.ldb = nt;
      g.C = W.B; g.ldc = nt;
    } else {
      g.M = m; g.N = r; g.K = nt;
      g.A = theta; g.lda = nt;
      g.B = Q; g.ldb = r;
      g.C = W.B; g.ldc = r;
    }
    launch_gemm(g, s);
  }
  norm2(theta, (ll)m * nt, W.nrm, red, s);
  norm2(W.B, (ll)r * (R ? nt : m), W.nrm + 1, red, s);
  DMRG2_CUDA(cudaMemcpyAsync(W.h_nrm, W.nrm, sizeof(double) * 2, cudaMemcpyDeviceToHost, s));
  if (R) {
    o = eig_split(ew, W.B, r, nt, 'R', chi, cutoff, false, W.F, right, s);
    Gemm<T> g;  // left = Q U_s
    g.M = m; g.N = o.k; g.K = r;
    g.A = Q; g.lda = r;
    g.B = W.F; g.ldb = o.k;
    g.C = left; g.ldc = o.k;
    launch_gemm(g, s);
  } else {
    o = eig_split(ew, W.B, m, r, 'L', chi, cutoff, false, left, W.F, s);
    Gemm<T> g;  // right^T = conj(Q) (V_s^H)^T (nt x k) into B, then transposed
    g.ca = true; g.tb = true;
    g.M = nt; g.N = o.k; g.K = r;
    g.A = Q; g.lda = r;
    g.B = W.F; g.ldb = r;
    g.C = W.B; g.ldc = o.k;
    launch_gemm(g, s);
    transpose<T>(W.B, right, (ll)nt, (ll)o.k, s);
  }
  DMRG2_CUDA(cudaStreamSynchronize(s));  // (eig_split already waited; the norms are read here)
  o.trunc_err += std::max(W.h_nrm[0] - W.h_nrm[1], 0.0);
  return true;
}

}  // namespace dmrg2
