// Launchers for the Krylov, SVD and data-movement kernels.
#pragma once

#include "common.cuh"

namespace dmrg2 {

constexpr int KRYLOV_CAP = 128;   // hard cap on Krylov vectors per Lanczos pass
constexpr int VEC_THREADS = 256;

// Device-resident state of one Lanczos solve (one per engine).
struct LanczosDev {
  double alpha[KRYLOV_CAP];
  double beta[KRYLOV_CAP];
  double coef[2 * (KRYLOV_CAP + 1)];   // projection coefficients of the current pass (re, im)
  double ritz[KRYLOV_CAP];             // Ritz coefficients (real: T is real symmetric)
  double nrm2;                         // squared norm produced by the last reduction
  double e_prev, e_cur;
  double tol;
  int done;                            // 1 once converged / broken down / Krylov space full
  int converged;
  int n_iter;                          // size of the tridiagonal matrix
  int randomized;
  int kmax;
  int j;                               // Krylov index of the device-looped solve's current step
  int guard;                           // loop bodies run so far (bounds the device loop)
  unsigned seed_in;                    // the device-looped solve's seed (copied in per solve)
  unsigned long long t_mark;           // %globaltimer when the current matvec was issued
  unsigned long long mv_ns;            // matvec time accumulated by the device-looped solve
};

// Reduction scratch shared by the vector kernels.
struct RedScratch {
  double* part = nullptr;   // [nblk][ncoef*2]
  unsigned* counter = nullptr;
  int nblk = 0;
};

int vec_blocks(ll n);

// w <- H v is done by the caller; these kernels implement one Lanczos step.
template <typename T>
void lz_dots(const T* V, int nv, ll n, const T* w, LanczosDev* st, RedScratch& r, cudaStream_t s);
template <typename T>
void lz_update_dots(const T* V, int nv, ll n, T* w, LanczosDev* st, RedScratch& r, cudaStream_t s);
template <typename T>
void lz_update_norm_check(const T* V, int nv, ll n, T* w, LanczosDev* st, RedScratch& r, int j,
                          int kmax, cudaStream_t s);
template <typename T>
void lz_normalize_next(T* vnext, const T* w, ll n, LanczosDev* st, cudaStream_t s);
// start: nrm(theta) -> (random fill if ~0) -> v0 = theta/|theta| (also into cur when given)
template <typename T>
void lz_start(T* theta, T* v0, ll n, LanczosDev* st, RedScratch& r, unsigned seed, double tol,
              int kmax, cudaStream_t s, T* cur = nullptr, const unsigned* seed_dev = nullptr);
// The same step with the Krylov index read on the device (st->j), for a loop that runs
// without the host: the three passes over w = H v_j, then v_(j+1) into V and into cur
// (the matvec's fixed input).
template <typename T>
void lz_step_dev(const T* V, ll n, T* w, T* cur, LanczosDev* st, RedScratch& r, int kmax, cudaStream_t s);
// Ends one body of the device loop: advances st->j and sets the loop condition to
// "not done and fewer than kmax bodies run".
void lz_loop_next(LanczosDev* st, cudaGraphConditionalHandle h, int kmax, cudaStream_t s);
// Ritz vector out = sum_i ritz_i V_i, normalised.
template <typename T>
void lz_ritz(const T* V, ll n, T* out, LanczosDev* st, RedScratch& r, cudaStream_t s);

// ---------------------------------------------------------------- SVD
struct JacobiCtl {
  unsigned bar_count;
  unsigned bar_gen;
  int err;
  int sweeps;
  int rotated[64];
};

struct SvdOut {
  int k;            // kept rank
  int nonzero;
  double trunc_err; // sum of discarded sigma^2
  double sigma_max;
  double sigma_max2;
  double fro2;
  int jacobi_sweeps;
  int jacobi_err;
  int ns_done;      // eigenvector block already orthonormal (Newton-Schulz steps skipped)
};

template <typename T>
void svd_jacobi(T* X, T* Q, int nvec, ll len, JacobiCtl* ctl, int max_sweeps, double tol,
                const double* fro2_dev, cudaStream_t s);  // fro2_dev: |X|_F^2 on device, or null for 1
template <typename T>
void svd_sort_truncate(const T* X, int nvec, ll len, double* sigma, int* perm, SvdOut* out,
                       int chi_max, double cutoff, bool relative_cutoff, const JacobiCtl* ctl,
                       cudaStream_t s);
// gather: left (rows x k) and right (k x cols) factors from X (rotated vectors) / Q.
//   mode 0 ('R'): vectors were rows of theta: left = conj(Q^T) cols, right = X rows
//   mode 1 ('L'): vectors were columns:       left = X^T,            right = conj(Q) rows
template <typename T>
void svd_gather(const T* X, const T* Q, const int* perm, int nvec, ll len, int k, int mode,
                T* left, T* right, cudaStream_t s);

// boundary merge of the parallel sweep: the k kept singular values in sorted order,
// v <- 1 / max(v, floor), and out = diag(v) in (or diag(1/v) in) for a rows x cols block
void gather_sigma(const double* sigma, const int* perm, int k, double* out, cudaStream_t s);
void inv_clip(double* v, int k, double floor, cudaStream_t s);
template <typename T>
void row_scale(const T* in, const double* v, int rows, ll cols, T* out, bool invert, cudaStream_t s);

// ---------------------------------------------------------------- eigen path (eig.cu)
template <typename T>
void hetrd_cluster(T* G, int n, ll ld, double* d, double* e, T* tau, cudaStream_t s);
void tridiag_eigvals(const double* d, const double* e, int n, int K, double* lam, cudaStream_t s);
// gtol_rel: the group tolerance (relative to lam[0]) that group_mgs will use on the result
void tridiag_eigvecs(const double* d, const double* e, int n, int K, const double* lam,
                     const SvdOut* tr, double* Z, double* scratch, double gtol_rel, cudaStream_t s);
void group_mgs(double* Z, int n, int K, const double* lam, const SvdOut* tr, double gtol_rel,
               cudaStream_t s);
// compact-WY triangles of the reflector blocks that apply_q uses for (n, K); apply_q builds
// them itself unless wy_ready says they were built already (e.g. on a side stream)
template <typename T>
void wy_build(const T* R, ll ld, const T* tau, int n, int K, T* Tb, cudaStream_t s);
template <typename T>
void apply_q(const T* R, ll ld, const T* tau, int n, const double* Z, int K, const SvdOut* tr, T* Zg,
             T* Tb, cudaStream_t s, bool wy_ready = false);
void ns_check(const double* S, int K, SvdOut* out, double tol, double* part, unsigned* counter,
              cudaStream_t s);
// k from the eigenvalues: min(chi_max, K, #lam above max(cutoff^2 (x lam_max if relative),
// floor_rel lam_max)); eigenvalues at or below floor_rel lam_max are rounding noise
constexpr double EIG_NOISE_FLOOR = 16.0 * 2.2e-16;
void eig_truncate(const double* d, const double* lam, int n, int K, int chi_max, double cutoff,
                  bool relative, SvdOut* out, cudaStream_t s, double floor_rel = EIG_NOISE_FLOOR);
template <typename T>
void copy_cols_conj(const T* in, ll ldi, int rows, int k, T* out, cudaStream_t s);
template <typename T>
void transpose_conj(const T* in, ll ldi, int rows, int k, T* out, cudaStream_t s);

// ---------------------------------------------------------------- misc
template <typename T>
void transpose(const T* in, T* out, ll rows, ll cols, cudaStream_t s);  // out[c][r] = in[r][c]
template <typename T>
void set_identity(T* Q, int n, cudaStream_t s);
template <typename T>
void scale_inplace(T* x, ll n, const double* inv_scale_dev, cudaStream_t s);
template <typename T>
void norm2(const T* x, ll n, double* out_dev, RedScratch& r, cudaStream_t s);
template <typename T>
void trace_real(const T* M, int n, ll ld, double* out_re, double* out_im, cudaStream_t s);
// flag = 1 when the n x n matrix P equals the identity to tol (max |P - 1|)
template <typename T>
void identity_check(const T* P, int n, double tol, int* flag, cudaStream_t s);

}  // namespace dmrg2
