// Cholesky factorisation and the row triangular solve of CholeskyQR (real FP64),
// the orthonormalisation step of the warm-started subspace truncation.
#pragma once

#include "common.cuh"
#include "kernels.cuh"

namespace dmrg2 {

constexpr int CHOL_NB = 32;     // tile edge
constexpr int CHOL_MAX = 512;   // largest order factorised (16 x 16 tiles)

inline int chol_padded(int k) { return (k + CHOL_NB - 1) / CHOL_NB * CHOL_NB; }

// Lower Cholesky factor of the symmetric positive definite k x k matrix in A (row-major,
// lda >= chol_padded(k), the buffer holding chol_padded(k) rows; only the lower triangle
// is read). On exit the lower triangle of the padded matrix holds L (the padding is the
// identity), rdiag[j] = 1 / L_jj. *status becomes 1 (and stays so until the caller
// clears it) when a pivot falls below rel_tol times the largest diagonal entry of A: the
// matrix is then not numerically positive definite at that tolerance and L is not valid.
// shift_rel > 0 factorises A + shift_rel trace(A) 1 instead (shifted CholeskyQR).
// One 8-CTA cluster; enqueued on s.
void chol_factor(double* A, int k, ll lda, double* rdiag, int* status, double rel_tol, cudaStream_t s,
                 double shift_rel = 0.0);

// X = L^{-1} (k x k row-major, ldx; zeros above the diagonal) where L L^T = G +
// shift_rel trace(G) 1 for the symmetric positive definite k x k G (row-major, ldg; only
// its lower triangle is read), k <= 256. Everything stays in the shared memory of one
// 8-CTA cluster until X is written. *status becomes 1 when a pivot falls below rel_tol
// times the largest (shifted) diagonal entry; X is then not valid.
constexpr int CHOL_INV_MAX = 256;
void chol_inverse(const double* G, int k, ll ldg, double* X, ll ldx, int* status, double rel_tol, double shift_rel,
                  cudaStream_t s);

// *status = 1 unless out->ns_done (a Newton-Schulz run that did not converge)
void mark_unconverged(const SvdOut* out, int* status, cudaStream_t s);

// every column of the rows x k row-major Y scaled to unit norm (*status = 1 on a zero
// or non-finite column); part holds COLNORM_MAX_CHUNKS x k doubles of partial sums
// (rows <= 32 COLNORM_MAX_CHUNKS)
constexpr int COLNORM_MAX_CHUNKS = 64;
void col_normalize(double* Y, ll rows, int k, double* part, int* status, cudaStream_t s);

// Y <- Y L^{-T} in place for the m x k row-major Y (ldy): the orthonormal factor of
// CholeskyQR when L L^T = Y^T Y. L and rdiag as chol_factor left them.
void chol_solve_rows(double* Y, ll m, int k, ll ldy, const double* L, ll lda, const double* rdiag,
                     const int* status, cudaStream_t s);

}  // namespace dmrg2
