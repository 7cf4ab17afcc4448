// Host driver of the truncated split of theta through the reduced density
// matrix (eig.cu). Replaces the SVD + truncation + gauge split of the
// reference (gpu-rocm/dmrg2-gpu/src/dmrg2_gpu_impl.h:1167-1343).
#pragma once

#include <algorithm>
#include <cstring>
#include <stdexcept>
#include <vector>

#include "cholqr.cuh"
#include "common.cuh"
#include "gemm.cuh"
#include "kernels.cuh"

namespace dmrg2 {

template <typename T>
struct EigWork {
  T* G = nullptr;      // nmax x nmax Gram matrix, then reflectors
  double* d = nullptr;
  double* e = nullptr;
  T* tau = nullptr;
  double* lam = nullptr;
  double* Z = nullptr;   // nmax x Kmax
  double* Z2 = nullptr;  // nmax x Kmax
  double* S = nullptr;   // Kmax x Kmax
  double* scr = nullptr; // 5 * nmax * Kmax
  T* Zg = nullptr;       // nmax x Kmax
  T* Tb = nullptr;       // compact-WY triangles, 16 x 16 per block of reflectors
  double* part = nullptr;
  unsigned* counter = nullptr;
  SvdOut* out = nullptr;
  SvdOut* h_out = nullptr;
  cudaStream_t side = nullptr;  // builds the compact-WY triangles while the eigenvectors are computed
  cudaEvent_t ev_refl = nullptr, ev_wy = nullptr;
  int nmax = 0, Kmax = 0;
  long long ns_extra = 0;      // truncations that needed the two extra Newton-Schulz iterations
  long long floor_raised = 0;  // recomputations with a raised noise floor
  size_t bytes = 0;
  std::vector<void*> owned;

  void* alloc(size_t b) {
    void* p = nullptr;
    DMRG2_CUDA(cudaMalloc(&p, std::max<size_t>(b, 16)));
    owned.push_back(p);
    bytes += b;
    return p;
  }
  void init(int nmax_, int Kmax_) {
    nmax = std::max(nmax_, 1);
    Kmax = std::max(std::min(Kmax_, nmax), 1);
    const size_t nn = (size_t)nmax, kk = (size_t)Kmax;
    G = (T*)alloc(sizeof(T) * nn * nn);
    d = (double*)alloc(sizeof(double) * nn);
    e = (double*)alloc(sizeof(double) * nn);
    tau = (T*)alloc(sizeof(T) * nn);
    lam = (double*)alloc(sizeof(double) * kk);
    Z = (double*)alloc(sizeof(double) * nn * kk);
    Z2 = (double*)alloc(sizeof(double) * nn * kk);
    S = (double*)alloc(sizeof(double) * kk * kk);
    scr = (double*)alloc(sizeof(double) * 5 * nn * kk);
    Zg = (T*)alloc(sizeof(T) * nn * kk);
    Tb = (T*)alloc(sizeof(T) * 256 * (nn + 1));
    part = (double*)alloc(sizeof(double) * 64);
    counter = (unsigned*)alloc(sizeof(unsigned) * 4);
    DMRG2_CUDA(cudaMemset(counter, 0, sizeof(unsigned) * 4));
    out = (SvdOut*)alloc(sizeof(SvdOut));
    DMRG2_CUDA(cudaMallocHost(&h_out, sizeof(SvdOut)));
    DMRG2_CUDA(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
    DMRG2_CUDA(cudaEventCreateWithFlags(&ev_refl, cudaEventDisableTiming));
    DMRG2_CUDA(cudaEventCreateWithFlags(&ev_wy, cudaEventDisableTiming));
  }
  void release() {
    for (void* p : owned) cudaFree(p);
    owned.clear();
    if (h_out) cudaFreeHost(h_out);
    h_out = nullptr;
    if (side) cudaStreamDestroy(side);
    if (ev_refl) cudaEventDestroy(ev_refl);
    if (ev_wy) cudaEventDestroy(ev_wy);
    side = nullptr;
    ev_refl = ev_wy = nullptr;
  }
};

// Truncated split of theta (m x nt, row-major).
//   dir 'R': left (m x k) isometric columns, right (k x nt) = left^H theta
//   dir 'L': right (k x nt) isometric rows,   left (m x k)  = theta right^H
// k = min(chi, rank, #{sigma > cutoff}) (relative: sigma > cutoff * sigma_max),
// singular values below the density-matrix noise floor count as zero.
// The host waits once (to learn k). Returns the device-side summary.
// K_compute (>= chi) eigenpairs are computed; lam_out (optional, host) receives them.
template <typename T>
SvdOut eig_split(EigWork<T>& W, const T* theta, int m, int nt, char dir, int chi, double cutoff,
                 bool relative, T* left, T* right, cudaStream_t s, int K_compute = 0,
                 double* lam_out = nullptr) {
  const bool R = (dir == 'R');
  const int n = R ? m : nt;
  if (n > W.nmax) throw std::runtime_error("eig_split: workspace too small");
  const int K = std::min(std::min(std::max(chi, K_compute), n), W.Kmax);
  chi = std::min(chi, K);
  {  // Gram matrix: R -> conj(theta theta^H) (Hermitian), L -> theta^H theta
    Gemm<T> g;
    g.M = n; g.N = n;
    if (R) {
      g.ca = true; g.tb = true; g.K = nt;
      g.A = theta; g.lda = nt;
      g.B = theta; g.ldb = nt;
    } else {
      g.ta = true; g.ca = true; g.K = m;
      g.A = theta; g.lda = nt;
      g.B = theta; g.ldb = nt;
    }
    g.C = W.G; g.ldc = n;
    launch_gemm(g, s);
  }
  hetrd_cluster<T>(W.G, n, n, W.d, W.e, W.tau, s);
  // the back-transform's WY triangles need only the reflectors: build them on the side stream
  DMRG2_CUDA(cudaEventRecord(W.ev_refl, s));
  DMRG2_CUDA(cudaStreamWaitEvent(W.side, W.ev_refl, 0));
  wy_build<T>(W.G, n, W.tau, n, K, W.Tb, W.side);
  DMRG2_CUDA(cudaEventRecord(W.ev_wy, W.side));
  tridiag_eigvals(W.d, W.e, n, K, W.lam, s);
  eig_truncate(W.d, W.lam, n, K, chi, cutoff, relative, W.out, s);  // k decided before any vector
  constexpr double gtol_rel = 1e-14;  // groups: neighbours within 1e-14 lambda_max
  tridiag_eigvecs(W.d, W.e, n, K, W.lam, W.out, W.Z, W.scr, gtol_rel, s);
  group_mgs(W.Z, n, K, W.lam, W.out, gtol_rel, s);
  // Newton-Schulz GEMMs have K x K (or n x K) outputs, a few 64 x 64 tiles at chi = 256:
  // split their long dimension over CTAs, partials in the (otherwise idle) scratch area
  const size_t scr_len = (size_t)5 * W.nmax * W.Kmax;
  auto split_for = [&](int M, int N, int Kd) {
    int sk = std::min(8, std::max(1, Kd / 64));
    while (sk > 1 && (size_t)sk * M * N > scr_len) --sk;
    return sk;
  };
  // Newton-Schulz polar step Z <- Z (3I - Z^T Z) / 2; an orthogonality error e becomes
  // ~1.5 e^2 per iteration, and iterations after convergence only launch kernels that
  // return at once
  auto ns_iteration = [&]() {
    Gemm<double> g1;
    g1.ta = true;
    g1.M = K; g1.N = K; g1.K = n;
    g1.A = W.Z; g1.lda = K;
    g1.B = W.Z; g1.ldb = K;
    g1.C = W.S; g1.ldc = K;
    g1.skip = &W.out->ns_done;
    g1.splitk = split_for(K, K, n);
    g1.ws = W.scr;
    launch_gemm(g1, s);
    ns_check(W.S, K, W.out, 4e-16 * (double)n, W.part, W.counter, s);
    DMRG2_CUDA(cudaMemcpyAsync(W.Z2, W.Z, sizeof(double) * (size_t)n * K, cudaMemcpyDeviceToDevice, s));
    Gemm<double> g2;
    g2.M = n; g2.N = K; g2.K = K;
    g2.A = W.Z; g2.lda = K;
    g2.B = W.S; g2.ldb = K;
    g2.C = W.Z2; g2.ldc = K;
    g2.alpha = -0.5; g2.beta = 1.5;
    g2.skip = &W.out->ns_done;
    g2.splitk = split_for(n, K, K);
    g2.ws = W.scr;
    launch_gemm(g2, s);
    std::swap(W.Z, W.Z2);
  };
  for (int it = 0; it < 3; ++it) ns_iteration();
  DMRG2_CUDA(cudaStreamWaitEvent(s, W.ev_wy, 0));
  apply_q<T>(W.G, n, W.tau, n, W.Z, K, W.out, W.Zg, W.Tb, s, true);
  DMRG2_CUDA(cudaMemcpyAsync(W.h_out, W.out, sizeof(SvdOut), cudaMemcpyDeviceToHost, s));
  DMRG2_CUDA(cudaStreamSynchronize(s));
  SvdOut o = *W.h_out;
  if (!std::isfinite(o.fro2))
    throw std::runtime_error("eigensolver: non-finite density matrix or tridiagonal reduction");
  auto read_out = [&]() {
    DMRG2_CUDA(cudaMemcpyAsync(W.h_out, W.out, sizeof(SvdOut), cudaMemcpyDeviceToHost, s));
    DMRG2_CUDA(cudaStreamSynchronize(s));
    o = *W.h_out;
  };
  if (!o.ns_done) {
    // not orthonormal after three iterations: close tail eigenvalues just outside one
    // Gram-Schmidt window can leave overlaps near 0.15, which two more iterations bring
    // below 1e-13; then the back-transform again (its WY triangles are still valid)
    for (int it = 0; it < 2; ++it) ns_iteration();
    apply_q<T>(W.G, n, W.tau, n, W.Z, K, W.out, W.Zg, W.Tb, s, true);
    read_out();
    ++W.ns_extra;
  }
  // Still not orthonormal: kept eigenvalues just above the rounding floor, within rounding
  // of one another, have ill-determined and nearly dependent vectors. Raise the floor
  // (those Schmidt values are below ~3e-7 resp. 3e-6 of the largest) and recompute.
  for (int attempt = 0; !o.ns_done && attempt < 2; ++attempt) {
    eig_truncate(W.d, W.lam, n, K, chi, cutoff, relative, W.out, s, attempt == 0 ? 1e-13 : 1e-11);
    tridiag_eigvecs(W.d, W.e, n, K, W.lam, W.out, W.Z, W.scr, gtol_rel, s);
    group_mgs(W.Z, n, K, W.lam, W.out, gtol_rel, s);
    for (int it = 0; it < 5; ++it) ns_iteration();
    apply_q<T>(W.G, n, W.tau, n, W.Z, K, W.out, W.Zg, W.Tb, s, true);
    read_out();
    ++W.floor_raised;
  }
  if (!o.ns_done)
    throw NumericError("eigensolver: kept eigenvectors not orthonormal to 2e-13 (order " + std::to_string(n) +
                       ", " + std::to_string(K) + " vectors) even with the noise floor at 1e-11");
  const int k = o.k;
  if (R) {
    copy_cols_conj<T>(W.Zg, K, m, k, left, s);  // U = conj(eigvecs of conj(G))
    Gemm<T> g;                                  // right = U^H theta = Zg^T theta
    g.ta = true;
    g.M = k; g.N = nt; g.K = m;
    g.A = W.Zg; g.lda = K;
    g.B = theta; g.ldb = nt;
    g.C = right; g.ldc = nt;
    launch_gemm(g, s);
  } else {
    Gemm<T> g;  // left = theta V (before right is written: right may alias theta)
    g.M = m; g.N = k; g.K = nt;
    g.A = theta; g.lda = nt;
    g.B = W.Zg; g.ldb = K;
    g.C = left; g.ldc = k;
    launch_gemm(g, s);
    transpose_conj<T>(W.Zg, K, nt, k, right, s);  // Vh = V^H
  }
  if (lam_out) {
    DMRG2_CUDA(cudaMemcpyAsync(lam_out, W.lam, sizeof(double) * K, cudaMemcpyDeviceToHost, s));
    DMRG2_CUDA(cudaStreamSynchronize(s));
  }
  return o;
}


// ============================================================================
// Warm-started subspace truncation (real FP64).
//
// In a sweep that repeats the previous sweep's bond dimension k, the kept
// subspace of a bond barely moves between sweeps, and the MPS already holds an
// orthonormal basis of last sweep's kept space next to the optimised theta: for
// a left-to-right step the right-canonical site B (k x nt, B B^T = 1), for a
// right-to-left step the left-canonical site A (m x k, A^T A = 1). Three
// half-steps of block power iteration on theta from that basis, each made
// orthonormal by one shifted CholeskyQR pass and one plain pass (the last one by
// two plain passes), give the kept left (or right) isometry; the other factor
// is its projection of theta, so the split is exact for the kept subspace and its
// discarded weight is |theta|^2 - |kept|^2:
//   'R': U1 = qr(theta B^T), V1 = qr(theta^T U1), U = qr2(theta V1),
//        left = U, right = U^T theta
//   'L': V1 = qr(theta^T A), U1 = qr(theta V1), V = qr2(theta^T U1),
//        right = V^T, left = theta V
// The shifted pass handles kept singular values down to ~1e-12 of the largest; a
// pivot of a plain pass below 1e-14 of the largest diagonal entry (an input that
// is not of full rank k) makes it give up, and the caller runs the exact split.
// ============================================================================
struct WstWork {
  double* Ya = nullptr;  // qmax x kmax
  double* Yb = nullptr;
  double* G = nullptr;   // np x np, np = chol_padded(kmax)
  double* rd = nullptr;  // np
  double* nrm = nullptr; // |theta|^2, |kept factor|^2
  int* status = nullptr;
  double* h_buf = nullptr;  // pinned: status (as double), |theta|^2, |kept|^2
  int qmax = 0, kmax = 0, np = 0;
  size_t bytes = 0;
  std::vector<void*> owned;

  void* alloc(size_t b) {
    void* p = nullptr;
    DMRG2_CUDA(cudaMalloc(&p, std::max<size_t>(b, 16)));
    owned.push_back(p);
    bytes += b;
    return p;
  }
  void init(int qmax_, int kmax_) {
    qmax = std::max(qmax_, 1);
    kmax = std::max(std::min(kmax_, CHOL_MAX), 1);
    np = chol_padded(kmax);
    Ya = (double*)alloc(sizeof(double) * (size_t)qmax * kmax);
    Yb = (double*)alloc(sizeof(double) * (size_t)qmax * kmax);
    G = (double*)alloc(sizeof(double) * (size_t)np * np);
    rd = (double*)alloc(sizeof(double) * (size_t)np);
    nrm = (double*)alloc(sizeof(double) * 4);
    status = (int*)alloc(sizeof(int) * 4);
    DMRG2_CUDA(cudaMallocHost(&h_buf, sizeof(double) * 4));
  }
  void release() {
    for (void* p : owned) cudaFree(p);
    owned.clear();
    if (h_buf) cudaFreeHost(h_buf);
    h_buf = nullptr;
  }
};

// device bytes WstWork::init(qmax, kmax) allocates
inline size_t wst_bytes(ll qmax, ll kmax) {
  qmax = std::max<ll>(qmax, 1);
  kmax = std::max<ll>(std::min<ll>(kmax, CHOL_MAX), 1);
  const ll np = chol_padded((int)kmax);
  return sizeof(double) * (size_t)(2 * qmax * kmax + np * np + np + 4) + sizeof(int) * 4;
}

// Y (rows x k) <- Y R^{-1} with R^T R = Y^T Y (+ shift): one shifted CholeskyQR pass,
// which leaves a basis of the same span with condition number ~1/sqrt(shift) (a
// well-conditioned start for the next power step), and `plain` CholeskyQR passes after
// it, which make the basis orthonormal to rounding.
inline void wst_qr(WstWork& W, double* Y, ll rows, int k, int plain, cudaStream_t s) {
  const double u = 1.1102230246251565e-16;
  const double shift_rel = 11.0 * ((double)rows * k + (double)k * (k + 1)) * u;
  for (int it = 0; it <= plain; ++it) {
    Gemm<double> g;  // G = Y^T Y
    g.ta = true;
    g.M = k; g.N = k; g.K = (int)rows;
    g.A = Y; g.lda = k;
    g.B = Y; g.ldb = k;
    g.C = W.G; g.ldc = W.np;
    launch_gemm(g, s);
    chol_factor(W.G, k, W.np, W.rd, W.status, it == 0 ? 1e-300 : 1e-14, s, it == 0 ? shift_rel : 0.0);
    chol_solve_rows(Y, rows, k, k, W.G, W.np, W.rd, W.status, s);
  }
}

// Warm-started split of theta (m x nt) at kept rank k; `warm` is B (k x nt) for 'R',
// A (m x k) for 'L'. Writes left (m x k) and right (k x nt) and returns true, or returns
// false (left / right undefined) when CholeskyQR gave up. The host waits once.
inline bool wst_split(WstWork& W, RedScratch& red, const double* theta, int m, int nt, char dir, int k,
                      const double* warm, double* left, double* right, double& trunc_err, cudaStream_t s) {
  if (k > W.kmax || m > W.qmax || nt > W.qmax) throw std::runtime_error("wst_split: workspace too small");
  DMRG2_CUDA(cudaMemsetAsync(W.status, 0, sizeof(int), s));
  auto mul = [&](bool ta, const double* A, ll lda, int M, int Kd, const double* B, ll ldb, bool tb, double* C) {
    Gemm<double> g;  // C (M x k) = op(A) op(B)
    g.ta = ta; g.tb = tb;
    g.M = M; g.N = k; g.K = Kd;
    g.A = A; g.lda = lda;
    g.B = B; g.ldb = ldb;
    g.C = C; g.ldc = k;
    launch_gemm(g, s);
  };
  if (dir == 'R') {
    mul(false, theta, nt, m, nt, warm, nt, true, W.Ya);  // theta B^T
    wst_qr(W, W.Ya, m, k, 1, s);
    mul(true, theta, nt, nt, m, W.Ya, k, false, W.Yb);   // theta^T U1
    wst_qr(W, W.Yb, nt, k, 1, s);
    mul(false, theta, nt, m, nt, W.Yb, k, false, left);  // theta V1
    wst_qr(W, left, m, k, 2, s);
    Gemm<double> g;  // right = U^T theta
    g.ta = true;
    g.M = k; g.N = nt; g.K = m;
    g.A = left; g.lda = k;
    g.B = theta; g.ldb = nt;
    g.C = right; g.ldc = nt;
    launch_gemm(g, s);
    norm2(right, (ll)k * nt, W.nrm + 1, red, s);
  } else {
    mul(true, theta, nt, nt, m, warm, k, false, W.Ya);   // theta^T A
    wst_qr(W, W.Ya, nt, k, 1, s);
    mul(false, theta, nt, m, nt, W.Ya, k, false, W.Yb);  // theta V1
    wst_qr(W, W.Yb, m, k, 1, s);
    mul(true, theta, nt, nt, m, W.Yb, k, false, W.Ya);   // theta^T U1
    wst_qr(W, W.Ya, nt, k, 2, s);
    transpose(W.Ya, right, (ll)nt, (ll)k, s);            // right = V^T
    mul(false, theta, nt, m, nt, W.Ya, k, false, left);  // left = theta V
    norm2(left, (ll)m * k, W.nrm + 1, red, s);
  }
  norm2(theta, (ll)m * nt, W.nrm, red, s);
  DMRG2_CUDA(cudaMemcpyAsync(W.h_buf + 1, W.nrm, sizeof(double) * 2, cudaMemcpyDeviceToHost, s));
  int st = 0;
  DMRG2_CUDA(cudaMemcpyAsync(W.h_buf, W.status, sizeof(int), cudaMemcpyDeviceToHost, s));
  DMRG2_CUDA(cudaStreamSynchronize(s));
  std::memcpy(&st, W.h_buf, sizeof(int));
  if (st) return false;
  trunc_err = std::max(W.h_buf[1] - W.h_buf[2], 0.0);
  if (!std::isfinite(W.h_buf[1]) || !std::isfinite(W.h_buf[2])) return false;
  return true;
}

}  // namespace dmrg2
