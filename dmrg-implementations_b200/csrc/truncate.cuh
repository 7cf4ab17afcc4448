// Host driver of the truncated split of theta through the reduced density
// matrix (eig.cu). Replaces the SVD + truncation + gauge split of the
// reference (gpu-rocm/dmrg2-gpu/src/dmrg2_gpu_impl.h:1167-1343).
#pragma once

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <vector>

#include "cholqr.cuh"
#include "common.cuh"
#include "gemm.cuh"
#include "graphs.cuh"
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
    p = dev_alloc(std::max<size_t>(b, 16));
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
    h_out = (SvdOut*)host_pinned(sizeof(SvdOut));
    DMRG2_CUDA(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
    DMRG2_CUDA(cudaEventCreateWithFlags(&ev_refl, cudaEventDisableTiming));
    DMRG2_CUDA(cudaEventCreateWithFlags(&ev_wy, cudaEventDisableTiming));
  }
  void release() {
    for (void* p : owned) dev_free(p);
    owned.clear();
    if (h_out) host_unpin(h_out);
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
// half-steps of block power iteration on theta from that basis give the kept
// left (or right) isometry; the other factor is its projection of theta, so the
// split is exact for the kept subspace and its discarded weight is
// |theta|^2 - |kept|^2:
//   'R': U1 = tri(theta B^T), V1 = tri(theta^T U1), U = tri(theta V1),
//        left = U, right = U^T theta
//   'L': V1 = tri(theta^T A), U1 = tri(theta V1), V = tri(theta^T U1),
//        right = V^T, left = theta V
// tri = unit columns, then one CholeskyQR pass (Gram matrix, its tiled Cholesky factor
// in one cluster kernel, then the row solve Z L^{-T} on the tensor cores). Why that is
// enough: the basis a step starts from is orthonormal, ordered by decreasing
// singular value and close to the Schmidt basis of the bond (the exact split
// returns Schmidt vectors, and each later warm split keeps that), so each product
// has nearly orthogonal columns whose norms are the singular values; their spread
// (up to ~1e9 at chi = 256) is all of its condition number, and unit columns leave a
// condition number near 1 (measured 1.0-4.6 on Heisenberg, J1-J2 and Josephson
// chains), for which one CholeskyQR pass is orthonormal to ~25 u. The orthonormal
// factor must be triangular in the columns: it removes from each column the
// larger-singular-value directions that leaked into it and nothing else, which
// keeps the basis aligned with the Schmidt vectors. (A polar factor, e.g. from
// Newton-Schulz, rotates columns into each other by the leak, and the next power
// step amplifies that rotation by the singular-value ratios.) The final basis then
// gets Newton-Schulz steps to rounding (a rotation of order 1e-14 at most). A pivot
// below 1e-10 of the largest (a product that is not of full rank k, or a state that
// moved too far for a warm start) makes the split give up, and the caller runs the
// exact split of the bond.
// ============================================================================
struct WstWork {
  double* Ya = nullptr;  // qmax x kmax
  double* Yb = nullptr;
  double* Yc = nullptr;  // qmax x kmax, the other half of each Newton-Schulz step
  double* S = nullptr;   // Gram matrix, then its tiled Cholesky factor (np x np, np = chol_padded(kmax))
  double* cpart = nullptr;  // column sums of squares per row chunk
  double* ws = nullptr;  // split-K partial products: 8 x qmax x kmax
  double* nrm = nullptr; // |theta|^2, |kept factor|^2
  double* part = nullptr;
  unsigned* counter = nullptr;
  int* status = nullptr;
  SvdOut* out = nullptr;    // k and the Newton-Schulz convergence flag
  // with graphs: the warm factor in, and both factors out, pass through these fixed slots
  // (qmax x kmax each), so one graph serves every bond of a shape
  double *Win = nullptr, *Lout = nullptr, *Rout = nullptr;
  double* h_buf = nullptr;  // pinned: |theta|^2, |kept|^2
  SvdOut* h_out = nullptr;  // pinned
  int* h_status = nullptr;  // pinned
  int qmax = 0, kmax = 0;
  size_t bytes = 0;
  std::vector<void*> owned;
  // the launch sequence of a split, by direction, mode and shapes
  GraphCache graphs;

  void* alloc(size_t b) {
    void* p = nullptr;
    p = dev_alloc(std::max<size_t>(b, 16));
    owned.push_back(p);
    bytes += b;
    return p;
  }
  void init(int qmax_, int kmax_) {
    graphs.cap = 2048;  // ~100 bond shapes x 2 directions x 3 modes in a chi=256 sweep of 100 sites
    graphs.name = "warm split";
    qmax = std::max(qmax_, 1);
    kmax = std::max(std::min(kmax_, CHOL_MAX), 1);
    const size_t qk = (size_t)qmax * kmax;
    Ya = (double*)alloc(sizeof(double) * qk);
    Yb = (double*)alloc(sizeof(double) * qk);
    Yc = (double*)alloc(sizeof(double) * qk);
    Win = (double*)alloc(sizeof(double) * qk);
    Lout = (double*)alloc(sizeof(double) * qk);
    Rout = (double*)alloc(sizeof(double) * qk);
    const size_t np = (size_t)chol_padded(kmax);
    S = (double*)alloc(sizeof(double) * np * np);
    cpart = (double*)alloc(sizeof(double) * (size_t)COLNORM_MAX_CHUNKS * kmax);
    ws = (double*)alloc(sizeof(double) * 8 * qk);
    nrm = (double*)alloc(sizeof(double) * 4);
    part = (double*)alloc(sizeof(double) * 64);
    counter = (unsigned*)alloc(sizeof(unsigned) * 4);
    status = (int*)alloc(sizeof(int) * 4);
    out = (SvdOut*)alloc(sizeof(SvdOut));
    DMRG2_CUDA(cudaMemset(counter, 0, sizeof(unsigned) * 4));
    h_buf = (double*)host_pinned(sizeof(double) * 4);
    h_out = (SvdOut*)host_pinned(sizeof(SvdOut));
    h_status = (int*)host_pinned(sizeof(int));
  }
  void release() {
    graphs.clear();
    for (void* p : owned) dev_free(p);
    owned.clear();
    if (h_buf) host_unpin(h_buf);
    if (h_out) host_unpin(h_out);
    if (h_status) host_unpin(h_status);
    h_buf = nullptr;
    h_out = nullptr;
    h_status = nullptr;
  }
};

// device bytes WstWork::init(qmax, kmax) allocates
inline size_t wst_bytes(ll qmax, ll kmax) {
  qmax = std::max<ll>(qmax, 1);
  kmax = std::max<ll>(std::min<ll>(kmax, CHOL_MAX), 1);
  const ll np = chol_padded((int)kmax);
  return sizeof(double) * (size_t)(14 * qmax * kmax + np * np + COLNORM_MAX_CHUNKS * kmax + 4 + 64) +
         sizeof(unsigned) * 4 + sizeof(int) * 4 + sizeof(SvdOut);
}

// DMRG2_DEBUG_WARM=1: the warm split prints each orthonormalisation's outcome to stderr
inline bool wst_debug() {
  static const bool on = [] {
    const char* e = std::getenv("DMRG2_DEBUG_WARM");
    return e && e[0] == '1';
  }();
  return on;
}

// K split so that a GEMM with few output tiles still spreads over the GPU
inline int wst_splitk(int M, int N, int K) {
  const int tiles = ceil_div(M, GemmTile<double>::BM) * ceil_div(N, GemmTile<double>::BN);
  int sk = 1;
  while (sk < 8 && tiles * sk < 148 && K / (2 * sk) >= 64) sk *= 2;
  return sk;
}

// How many power half-steps a warm split runs:
//   WST_FULL   three, from the warm factor (the scheme above);
//   WST_SHORT  one, from the warm factor: left = tri(theta B^T) ('R'), right^T =
//              tri(theta^T A) ('L'), each polished and the other factor projected;
//   WST_RESUME the two after a WST_SHORT call on the same theta, starting from the
//              basis that call left (in `left` for 'R', in W.Ya for 'L'); together they
//              are WST_FULL.
enum WstMode { WST_FULL = 0, WST_SHORT = 1, WST_RESUME = 2 };

// Warm-started split of theta (m x nt) at kept rank k; `warm` is B (k x nt) for 'R',
// A (m x k) for 'L'. Writes left (m x k) and right (k x nt) and returns true, or returns
// false (left / right undefined) when the warm start was not good enough. The host
// waits once; ev_end, when given, is recorded after the split's kernels. With graphs on (and a stream other than the legacy default one), the work
// between the status reset and that wait is one cached graph per (direction, mode,
// shapes): the warm factor is copied into W.Win and the factors come out of W.Lout and
// W.Rout, so the graph's buffers do not depend on the bond; a key's second call launches
// the kernels and then captures them, later calls replay the capture.
inline bool wst_split(WstWork& W, RedScratch& red, const double* theta, int m, int nt, char dir, int k,
                      const double* warm, double* left, double* right, double& trunc_err, cudaStream_t s,
                      WstMode mode = WST_FULL, bool allow_graph = true, cudaEvent_t ev_end = nullptr) {
  if (k > W.kmax || m > W.qmax || nt > W.qmax) throw std::runtime_error("wst_split: workspace too small");
  if (std::max(m, nt) > 32 * COLNORM_MAX_CHUNKS) return false;  // beyond the column-scaling kernel
  DMRG2_CUDA(cudaMemsetAsync(W.status, 0, sizeof(int), s));
  {
    SvdOut o0{};
    o0.k = k;
    *W.h_out = o0;
    DMRG2_CUDA(cudaMemcpyAsync(W.out, W.h_out, sizeof(SvdOut), cudaMemcpyHostToDevice, s));
  }
  // C (M x N) = alpha op(A) op(B) + beta C, K split over CTAs when the output is small
  auto mul = [&](bool ta, const double* A, ll lda, int M, int N, int Kd, const double* B, ll ldb, bool tb,
                 double* C, ll ldc, double alpha, double beta, const int* skip) {
    Gemm<double> g;
    g.ta = ta; g.tb = tb;
    g.M = M; g.N = N; g.K = Kd;
    g.A = A; g.lda = lda;
    g.B = B; g.ldb = ldb;
    g.C = C; g.ldc = ldc;
    g.alpha = alpha; g.beta = beta;
    g.skip = skip;
    g.splitk = wst_splitk(M, N, Kd);
    g.ws = W.ws;
    launch_gemm(g, s);
  };
  const int* done = &W.out->ns_done;
  // Newton-Schulz polish of the nearly orthonormal Z (rows x k): S = Z^T Z, stop once
  // |S - 1| < tol, Z <- 1.5 Z - 0.5 Z S (iterations after convergence only launch
  // kernels that return); a run that ends unconverged marks the split as failed. The
  // result is left in dst.
  auto orth = [&](double* Z, ll rows, double tol, int iters, double* dst) {
    DMRG2_CUDA(cudaMemsetAsync(&W.out->ns_done, 0, sizeof(int), s));
    double* a = Z;
    double* b = (Z == W.Yc) ? dst : W.Yc;
    for (int it = 0; it < iters; ++it) {
      mul(true, a, k, k, k, (int)rows, a, k, false, W.S, k, 1.0, 0.0, done);
      ns_check(W.S, k, W.out, tol, W.part, W.counter, s);
      DMRG2_CUDA(cudaMemcpyAsync(b, a, sizeof(double) * (size_t)rows * k, cudaMemcpyDeviceToDevice, s));
      mul(false, a, k, (int)rows, k, k, W.S, k, false, b, k, -0.5, 1.5, done);
      std::swap(a, b);
    }
    mark_unconverged(W.out, W.status, s);
    if (a != dst) DMRG2_CUDA(cudaMemcpyAsync(dst, a, sizeof(double) * (size_t)rows * k, cudaMemcpyDeviceToDevice, s));
    if (wst_debug()) {
      DMRG2_CUDA(cudaMemcpyAsync(W.h_out, W.out, sizeof(SvdOut), cudaMemcpyDeviceToHost, s));
      DMRG2_CUDA(cudaMemcpyAsync(W.h_status, W.status, sizeof(int), cudaMemcpyDeviceToHost, s));
      std::vector<double> hs((size_t)k * k);
      DMRG2_CUDA(cudaMemcpyAsync(hs.data(), W.S, sizeof(double) * hs.size(), cudaMemcpyDeviceToHost, s));
      DMRG2_CUDA(cudaStreamSynchronize(s));
      double e = 0.0;
      for (int i = 0; i < k; ++i)
        for (int j = 0; j < k; ++j) e = std::max(e, std::fabs(hs[(size_t)i * k + j] - (i == j ? 1.0 : 0.0)));
      std::fprintf(stderr, "[warm split] orth rows=%lld k=%d tol=%.1e done=%d status=%d last |S-1|=%.3e\n",
                   (long long)rows, k, tol, W.h_out->ns_done, *W.h_status, e);
    }
  };
  // Z (rows x k) <- tri(Z) into dst (dst != Z): unit columns, Gram matrix, its Cholesky factor, Z L^{-T}
  const int ldS = chol_padded(k);
  auto tri = [&](double* Z, ll rows, double* dst) {
    col_normalize(Z, rows, k, W.cpart, W.status, s);
    mul(true, Z, k, k, k, (int)rows, Z, k, false, W.S, ldS, 1.0, 0.0, nullptr);
    chol_tiles(W.S, k, ldS, W.S, ldS, W.status, 1e-10, 0.0, s);  // factor in place of the Gram matrix
    trsm_rows(Z, rows, k, W.S, ldS, dst, W.status, s);
  };
  const bool graph = allow_graph && graphs_enabled() && !wst_debug() && s != nullptr;
  double* const left_out = left;
  double* const right_out = right;
  if (graph) {
    if (mode != WST_RESUME) {
      DMRG2_CUDA(cudaMemcpyAsync(W.Win, warm, sizeof(double) * (size_t)(dir == 'R' ? (ll)k * nt : (ll)m * k),
                                 cudaMemcpyDeviceToDevice, s));
      warm = W.Win;
    }
    left = W.Lout;
    right = W.Rout;
  }
  auto body = [&]() {
  if (dir == 'R') {
    if (mode != WST_RESUME) {
      mul(false, theta, nt, m, k, nt, warm, nt, true, W.Ya, k, 1.0, 0.0, nullptr);  // theta B^T
      tri(W.Ya, m, W.Yb);
    } else {
      DMRG2_CUDA(cudaMemcpyAsync(W.Yb, left, sizeof(double) * (size_t)m * k, cudaMemcpyDeviceToDevice, s));  // U1
    }
    if (mode != WST_SHORT) {
      mul(true, theta, nt, nt, k, m, W.Yb, k, false, W.Ya, k, 1.0, 0.0, nullptr);  // theta^T U1
      tri(W.Ya, nt, W.Yb);
      mul(false, theta, nt, m, k, nt, W.Yb, k, false, W.Ya, k, 1.0, 0.0, nullptr); // theta V1
      tri(W.Ya, m, W.Yb);
    }
    orth(W.Yb, m, 4e-16 * (double)m, 2, left);                                     // polish
    mul(true, left, k, k, nt, m, theta, nt, false, right, nt, 1.0, 0.0, nullptr);  // right = U^T theta
    norm2(right, (ll)k * nt, W.nrm + 1, red, s);
  } else {
    if (mode != WST_RESUME) {
      mul(true, theta, nt, nt, k, m, warm, k, false, W.Ya, k, 1.0, 0.0, nullptr);  // theta^T A
      tri(W.Ya, nt, W.Yb);
    } else {
      DMRG2_CUDA(cudaMemcpyAsync(W.Yb, W.Ya, sizeof(double) * (size_t)nt * k, cudaMemcpyDeviceToDevice, s));  // V1
    }
    if (mode != WST_SHORT) {
      mul(false, theta, nt, m, k, nt, W.Yb, k, false, W.Ya, k, 1.0, 0.0, nullptr); // theta V1
      tri(W.Ya, m, W.Yb);
      mul(true, theta, nt, nt, k, m, W.Yb, k, false, W.Ya, k, 1.0, 0.0, nullptr);  // theta^T U1
      tri(W.Ya, nt, W.Yb);
    }
    orth(W.Yb, nt, 4e-16 * (double)nt, 2, W.Ya);                                   // polish; V in Ya
    transpose(W.Ya, right, (ll)nt, (ll)k, s);                                      // right = V^T
    mul(false, theta, nt, m, k, nt, W.Ya, k, false, left, k, 1.0, 0.0, nullptr);   // left = theta V
    norm2(left, (ll)m * k, W.nrm + 1, red, s);
  }
  norm2(theta, (ll)m * nt, W.nrm, red, s);
  };
  if (graph) {
    const GraphKey key{dir, mode, m, nt, k, (ll)theta, (ll)&W, (ll)red.part, (ll)red.counter, 0, 0, 0, 0, 0, 0, 0};
    if (GraphEntry* G = W.graphs.find(key)) {
      graph_replay(*G, s);
      W.graphs.replays += 1;
    } else if (!W.graphs.seen_before(key)) {
      body();
    } else {
      body();
      GraphEntry* N = W.graphs.slot(key);
      try {
        const auto t0 = std::chrono::steady_clock::now();
        DMRG2_CUDA(cudaGraphCreate(&N->g, 0));
        N->launches = capture_to_graph(s, N->g, body);
        graph_instantiate(W.graphs, *N);
        W.graphs.builds += 1;
        W.graphs.build_s += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      } catch (const std::exception& e) {
        N->reset();
        graphs_disable(e.what());
      }
    }
    DMRG2_CUDA(cudaMemcpyAsync(left_out, W.Lout, sizeof(double) * (size_t)m * k, cudaMemcpyDeviceToDevice, s));
    DMRG2_CUDA(cudaMemcpyAsync(right_out, W.Rout, sizeof(double) * (size_t)k * nt, cudaMemcpyDeviceToDevice, s));
  } else {
    body();
  }
  if (ev_end) DMRG2_CUDA(cudaEventRecord(ev_end, s));  // the split's device work ends here
  DMRG2_CUDA(cudaMemcpyAsync(W.h_buf + 1, W.nrm, sizeof(double) * 2, cudaMemcpyDeviceToHost, s));
  DMRG2_CUDA(cudaMemcpyAsync(W.h_out, W.out, sizeof(SvdOut), cudaMemcpyDeviceToHost, s));
  DMRG2_CUDA(cudaMemcpyAsync(W.h_status, W.status, sizeof(int), cudaMemcpyDeviceToHost, s));
  DMRG2_CUDA(cudaStreamSynchronize(s));
  if (*W.h_status) return false;
  if (!std::isfinite(W.h_buf[1]) || !std::isfinite(W.h_buf[2])) return false;
  trunc_err = std::max(W.h_buf[1] - W.h_buf[2], 0.0);
  return true;
}

}  // namespace dmrg2
