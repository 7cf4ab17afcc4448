// Cholesky factorisation and the row triangular solve of CholeskyQR (real FP64),
// the orthonormalisation step of the warm-started subspace truncation.
#pragma once

#include "common.cuh"
#include "kernels.cuh"

namespace dmrg2 {

constexpr int CHOL_NB = 32;     // tile edge
constexpr int CHOL_MAX = 512;   // largest order factorised (16 x 16 tiles)

inline int chol_padded(int k) { return (k + CHOL_NB - 1) / CHOL_NB * CHOL_NB; }

// Tiled Cholesky factor of the symmetric positive definite k x k matrix G (row-major,
// ldg; only its lower triangle is read), k <= 512, of G + shift_rel trace(G) 1 when
// shift_rel > 0. LX (np x np row-major, np = chol_padded(k), ldx >= np) receives the
// factor in the form the row solve uses: the tiles of L below the diagonal, and in each
// diagonal tile the inverse X_bb = L_bb^{-1} of L's diagonal tile (zeros above its
// diagonal); tiles above the diagonal are not written. Orders beyond k are padded with
// the identity. *status becomes 1 (and stays so until the caller clears it) when a
// pivot falls below rel_tol times the largest (shifted) diagonal entry: the matrix is
// then not numerically positive definite at that tolerance and LX is not valid. One
// cluster of 8 (np <= 256) or 16 CTAs; LX may be the buffer G is in (each CTA writes
// only the block row it read). Enqueued on s.
void chol_tiles(const double* G, int k, ll ldg, double* LX, ll ldx, int* status, double rel_tol, double shift_rel,
                cudaStream_t s);

// Y = Z L^{-T} for the rows x k row-major Z (ld k) and the factor chol_tiles left in LX:
// the orthonormal factor of CholeskyQR when L L^T = Z^T Z. Y (ld k) must not overlap Z.
// Does nothing while *status is set.
void trsm_rows(const double* Z, ll rows, int k, const double* LX, ll ldx, double* Y, const int* status,
               cudaStream_t s);

// *status = 1 unless out->ns_done (a Newton-Schulz run that did not converge)
void mark_unconverged(const SvdOut* out, int* status, cudaStream_t s);

// every column of the rows x k row-major Y scaled to unit norm (*status = 1 on a zero
// or non-finite column); part holds COLNORM_MAX_CHUNKS x k doubles of partial sums
// (rows <= 32 COLNORM_MAX_CHUNKS)
constexpr int COLNORM_MAX_CHUNKS = 64;
void col_normalize(double* Y, ll rows, int k, double* part, int* status, cudaStream_t s);

}  // namespace dmrg2
