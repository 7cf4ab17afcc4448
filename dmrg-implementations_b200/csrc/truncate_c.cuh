// Warm-started subspace split of complex two-site tensors.
//
// The same power half-steps, modes and acceptance as the real split (wst_split in
// truncate.cuh), with complex DMMA GEMMs for the products with theta. Each
// orthonormalisation runs on the real embedding of the complex column block, with the
// column pairs (y_j, i y_j) interleaved (embed_pairs / extract_pairs). On it, unit
// columns, the Gram matrix, the tiled Cholesky factor and the row solve amount to complex
// Gram-Schmidt: each y_j is orthogonalised against a span closed under multiplication by
// i. So the even columns of the result are a complex-orthonormal basis, triangular in the
// columns as the real split requires. The final Newton-Schulz polish also runs on the
// embedding: for a matrix of that structure each step is the embedding of the complex
// step.
//
//   'R': U1 = tri(theta B^H) [+ V1 = tri(theta^H U1), U2 = tri(theta V1)], left = U,
//        right = U^H theta;
//   'L': V1 = tri(theta^H A) [+ U1 = tri(theta V1), V2 = tri(theta^H U1)], right = V^H,
//        left = theta V.
// theta B^H is formed as the transpose of conj(B) theta^T, because the GEMM conjugates
// only its first operand.
#pragma once

#include "rsvd.cuh"
#include "truncate.cuh"

namespace dmrg2 {

struct WstWorkC {
  zc* Ya = nullptr;      // qmax x kmax
  zc* Yb = nullptr;
  double* Z1 = nullptr;  // real embeddings: (2 qmax) x (2 kmax) each
  double* Z2 = nullptr;
  double* Z3 = nullptr;
  double* S = nullptr;   // Gram matrix, then its tiled factor (np x np, np = chol_padded(2 kmax))
  double* cpart = nullptr;
  double* ws = nullptr;  // split-K partial products: 32 qmax kmax doubles
  double* nrm = nullptr;
  double* part = nullptr;
  unsigned* counter = nullptr;
  int* status = nullptr;
  SvdOut* out = nullptr;
  double* h_buf = nullptr;  // pinned: |theta|^2, |kept|^2
  SvdOut* h_out = nullptr;  // pinned
  int* h_status = nullptr;  // pinned
  int qmax = 0, kmax = 0;
  size_t bytes = 0;
  std::vector<void*> owned;

  void* alloc(size_t b) {
    void* p = dev_alloc(std::max<size_t>(b, 16));
    owned.push_back(p);
    bytes += b;
    return p;
  }
  void init(int qmax_, int kmax_) {
    qmax = std::max(qmax_, 1);
    kmax = std::max(std::min(kmax_, CHOL_MAX / 2), 1);
    const size_t qk = (size_t)qmax * kmax;
    Ya = (zc*)alloc(sizeof(zc) * qk);
    Yb = (zc*)alloc(sizeof(zc) * qk);
    Z1 = (double*)alloc(sizeof(double) * 4 * qk);
    Z2 = (double*)alloc(sizeof(double) * 4 * qk);
    Z3 = (double*)alloc(sizeof(double) * 4 * qk);
    const size_t np = (size_t)chol_padded(2 * kmax);
    S = (double*)alloc(sizeof(double) * np * np);
    cpart = (double*)alloc(sizeof(double) * (size_t)COLNORM_MAX_CHUNKS * 2 * kmax);
    ws = (double*)alloc(sizeof(double) * 32 * qk);
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

// device bytes WstWorkC::init(qmax, kmax) allocates
inline size_t wstc_bytes(ll qmax, ll kmax) {
  qmax = std::max<ll>(qmax, 1);
  kmax = std::max<ll>(std::min<ll>(kmax, CHOL_MAX / 2), 1);
  const ll qk = qmax * kmax;
  const ll np = chol_padded((int)(2 * kmax));
  return sizeof(zc) * (size_t)(2 * qk) +
         sizeof(double) * (size_t)(12 * qk + np * np + COLNORM_MAX_CHUNKS * 2 * kmax + 32 * qk + 4 + 64) +
         sizeof(unsigned) * 4 + sizeof(int) * 4 + sizeof(SvdOut);
}

// Warm-started split of complex theta (m x nt) at kept rank k; `warm` is B (k x nt) for
// 'R', A (m x k) for 'L'. Writes left (m x k) and right (k x nt) and returns true, or
// returns false (left / right undefined) when the warm start was not good enough. The
// host waits once; ev_end, when given, is recorded after the split's kernels.
inline bool wst_split_c(WstWorkC& W, RedScratch& red, const zc* theta, int m, int nt, char dir, int k,
                        const zc* warm, zc* left, zc* right, double& trunc_err, cudaStream_t s,
                        WstMode mode = WST_FULL, cudaEvent_t ev_end = nullptr) {
  if (k > W.kmax || m > W.qmax || nt > W.qmax) throw std::runtime_error("wst_split_c: workspace too small");
  if (2 * std::max(m, nt) > 32 * COLNORM_MAX_CHUNKS) return false;  // beyond the column-scaling kernel
  DMRG2_CUDA(cudaMemsetAsync(W.status, 0, sizeof(int), s));
  {
    SvdOut o0{};
    o0.k = k;
    *W.h_out = o0;
    DMRG2_CUDA(cudaMemcpyAsync(W.out, W.h_out, sizeof(SvdOut), cudaMemcpyHostToDevice, s));
  }
  // complex C (M x N) = op(A) op(B): ta / ca transpose / conjugate A, tb transposes B
  auto mulz = [&](bool ta, bool ca, const zc* A, ll lda, int M, int N, int Kd, const zc* B, ll ldb, bool tb,
                  zc* C, ll ldc) {
    Gemm<zc> g;
    g.ta = ta; g.ca = ca; g.tb = tb;
    g.M = M; g.N = N; g.K = Kd;
    g.A = A; g.lda = lda;
    g.B = B; g.ldb = ldb;
    g.C = C; g.ldc = ldc;
    g.splitk = wst_splitk(M, N, Kd);
    g.ws = (zc*)W.ws;
    launch_gemm(g, s);
  };
  // real C = alpha op(A) op(B) + beta C on the embeddings
  auto mulr = [&](bool ta, const double* A, ll lda, int M, int N, int Kd, const double* B, ll ldb, double* C,
                  ll ldc, double alpha, double beta, const int* skip) {
    Gemm<double> g;
    g.ta = ta;
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
  const int k2 = 2 * k;
  const int ldS = chol_padded(k2);
  // Z (rows x k) -> dst: complex CholeskyQR on the embedding (unit columns, Gram matrix,
  // tiled Cholesky factor, row solve), then the even columns
  auto tri = [&](const zc* Z, ll rows, zc* dst) {
    embed_pairs(Z, rows, k, W.Z1, s);
    col_normalize(W.Z1, 2 * rows, k2, W.cpart, W.status, s);
    mulr(true, W.Z1, k2, k2, k2, (int)(2 * rows), W.Z1, k2, W.S, ldS, 1.0, 0.0, nullptr);
    chol_tiles(W.S, k2, ldS, W.S, ldS, W.status, 1e-10, 0.0, s);
    trsm_rows(W.Z1, 2 * rows, k2, W.S, ldS, W.Z2, W.status, s);
    extract_pairs(W.Z2, rows, k, dst, s);
  };
  // two Newton-Schulz steps on the embedding of Z (rows x k), result into dst; a run that
  // ends unconverged marks the split as failed
  const int* done = &W.out->ns_done;
  auto polish = [&](const zc* Z, ll rows, zc* dst) {
    const ll r2 = 2 * rows;
    embed_pairs(Z, rows, k, W.Z1, s);
    DMRG2_CUDA(cudaMemsetAsync(&W.out->ns_done, 0, sizeof(int), s));
    double* a = W.Z1;
    double* b = W.Z3;
    for (int it = 0; it < 2; ++it) {
      mulr(true, a, k2, k2, k2, (int)r2, a, k2, W.S, k2, 1.0, 0.0, done);
      ns_check(W.S, k2, W.out, 4e-16 * (double)r2, W.part, W.counter, s);
      DMRG2_CUDA(cudaMemcpyAsync(b, a, sizeof(double) * (size_t)r2 * k2, cudaMemcpyDeviceToDevice, s));
      mulr(false, a, k2, (int)r2, k2, k2, W.S, k2, b, k2, -0.5, 1.5, done);
      std::swap(a, b);
    }
    mark_unconverged(W.out, W.status, s);
    extract_pairs(a, rows, k, dst, s);
  };
  if (dir == 'R') {
    if (mode != WST_RESUME) {
      mulz(false, true, warm, nt, k, m, nt, theta, nt, true, W.Yb, m);  // conj(B) theta^T (k x m)
      transpose<zc>(W.Yb, W.Ya, (ll)k, (ll)m, s);                          // theta B^H (m x k)
      tri(W.Ya, m, W.Yb);                                                  // U1
    } else {
      DMRG2_CUDA(cudaMemcpyAsync(W.Yb, left, sizeof(zc) * (size_t)m * k, cudaMemcpyDeviceToDevice, s));
    }
    if (mode != WST_SHORT) {
      mulz(true, true, theta, nt, nt, k, m, W.Yb, k, false, W.Ya, k);  // theta^H U1
      tri(W.Ya, nt, W.Yb);                                             // V1
      mulz(false, false, theta, nt, m, k, nt, W.Yb, k, false, W.Ya, k);  // theta V1
      tri(W.Ya, m, W.Yb);                                                // U2
    }
    polish(W.Yb, m, left);
    mulz(true, true, left, k, k, nt, m, theta, nt, false, right, nt);  // right = U^H theta
    norm2(right, (ll)k * nt, W.nrm + 1, red, s);
  } else {
    if (mode != WST_RESUME) {
      mulz(true, true, theta, nt, nt, k, m, warm, k, false, W.Ya, k);  // theta^H A
      tri(W.Ya, nt, W.Yb);                                             // V1
    } else {
      DMRG2_CUDA(cudaMemcpyAsync(W.Yb, W.Ya, sizeof(zc) * (size_t)nt * k, cudaMemcpyDeviceToDevice, s));
    }
    if (mode != WST_SHORT) {
      mulz(false, false, theta, nt, m, k, nt, W.Yb, k, false, W.Ya, k);  // theta V1
      tri(W.Ya, m, W.Yb);                                                // U1
      mulz(true, true, theta, nt, nt, k, m, W.Yb, k, false, W.Ya, k);    // theta^H U1
      tri(W.Ya, nt, W.Yb);                                               // V2
    }
    polish(W.Yb, nt, W.Ya);                                              // V in Ya
    transpose_conj<zc>(W.Ya, k, nt, k, right, s);                        // right = V^H
    mulz(false, false, theta, nt, m, k, nt, W.Ya, k, false, left, k);    // left = theta V
    norm2(left, (ll)m * k, W.nrm + 1, red, s);
  }
  norm2(theta, (ll)m * nt, W.nrm, red, s);
  if (ev_end) DMRG2_CUDA(cudaEventRecord(ev_end, s));
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
