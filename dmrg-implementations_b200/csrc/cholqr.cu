// CholeskyQR building blocks (real FP64) for the warm-started subspace truncation.
//
// chol_cluster_kernel: right-looking blocked Cholesky of a symmetric positive
// definite matrix of order <= 512 in 32 x 32 tiles, one cluster of 8 CTAs. The
// matrix stays in global memory (it is L2-resident: 2 MB at most) and is read and
// written with L2-only accesses, so the cluster barriers (release / acquire at
// cluster scope) are the only synchronisation. Per tile column p:
//   D  one warp factors the diagonal tile with register shuffles (the sqrt chain
//      of the 32 columns is the critical path of the whole factorisation);
//   P  one warp per sub-diagonal tile solves L_ip L_pp^T = A_ip row by row
//      (forward substitution, one lane per row);
//   T  one warp per trailing tile subtracts L_ip L_jp^T.
// Pivots below rel_tol times the largest diagonal entry mark the matrix as not
// numerically positive definite (the caller falls back to the exact split).
// With shift_rel > 0 the matrix factorised is A + shift_rel trace(A) 1: shifted
// CholeskyQR (Fukaya, Kannan, Nakatsukasa, Yamamoto and Yanagisawa, SIAM J. Sci.
// Comput. 42 (2020)) takes shift 11 (m k + k (k+1)) u |Y|_F^2 for the Gram matrix
// A = Y^T Y of an m x k block, which keeps the factorisation stable for any
// condition number of Y below ~1/u and leaves Y R^{-1} with a condition number
// of at most ~1/sqrt(shift_rel), so plain CholeskyQR can finish it.
//
// chol_solve_rows_kernel: Y <- Y L^{-T}, 8 rows of Y per CTA, tile column by tile
// column: the update by the finished columns, then the forward substitution
// with the diagonal tile (one lane per row).
#include <cooperative_groups.h>

#include "cholqr.cuh"

namespace cg = cooperative_groups;

namespace dmrg2 {

namespace {

constexpr int NB = CHOL_NB;
constexpr int CC = 8;    // CTAs in the factorisation cluster
constexpr int CT = 256;  // threads per CTA (8 warps)
constexpr int NW = CT / 32;
constexpr int TP = NB + 1;  // padded tile row in shared memory

__device__ inline double ldg_l2(const double* p) { return __ldcg(p); }
__device__ inline void stg_l2(double* p, double v) { __stcg(p, v); }

// column J of the in-register Cholesky of one diagonal tile (lane i holds row i), then
// the columns after it; compile-time J keeps every index of a[] static
template <int J>
__device__ __forceinline__ void chol_tile_col(double (&a)[NB], int lane, double piv_min, double piv_sub,
                                              bool& bad, double* rd) {
  double piv = __shfl_sync(0xffffffffu, a[J], J);
  if (!(piv > piv_min)) {  // also catches NaN
    bad = true;
    piv = piv_sub;
  }
  const double l = sqrt(piv);
  const double r = 1.0 / l;
  if (lane == J) {
    a[J] = l;
    rd[J] = r;
  } else if (lane > J) {
    a[J] *= r;
  }
#pragma unroll
  for (int c = J + 1; c < NB; ++c) {
    const double lc = __shfl_sync(0xffffffffu, a[J], c);
    if (lane >= c) a[c] -= a[J] * lc;
  }
  if constexpr (J + 1 < NB) chol_tile_col<J + 1>(a, lane, piv_min, piv_sub, bad, rd);
}

__global__ void __launch_bounds__(CT, 1)
    chol_cluster_kernel(double* __restrict__ A, int k, int np, ll lda, double* __restrict__ rdiag,
                        int* __restrict__ status, double rel_tol, double shift_rel) {
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = (int)cluster.block_rank();
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nblk = np / NB;
  extern __shared__ __align__(16) double csm[];
  double* Lp = csm;                         // L_pp [NB][TP]
  double* Rp = Lp + NB * TP;                // 1 / diag of L_pp [NB]
  double* Wt = Rp + NB;                     // per warp: an L_jp tile [NW][NB][TP]
  __shared__ double dmax_s, shift_s;

  // padding rows r >= k become identity rows (lower triangle only)
  for (int r = k + rank; r < np; r += CC)
    for (int c = tid; c <= r; c += CT) stg_l2(A + (ll)r * lda + c, c == r ? 1.0 : 0.0);
  if (warp == 0) {
    double m = 0.0, tr = 0.0;
    for (int i = lane; i < k; i += 32) {
      const double a = ldg_l2(A + (ll)i * lda + i);
      m = fmax(m, a);
      tr += a;
    }
    for (int o = 16; o > 0; o >>= 1) {
      m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
      tr += __shfl_xor_sync(0xffffffffu, tr, o);
    }
    if (lane == 0) {
      shift_s = shift_rel * tr;
      dmax_s = m + shift_s;
    }
  }
  cluster.sync();  // padding written, every CTA has read the unshifted diagonal
  if (shift_rel > 0.0) {
    for (int i = rank * CT + tid; i < k; i += CC * CT) stg_l2(A + (ll)i * lda + i, ldg_l2(A + (ll)i * lda + i) + shift_s);
    cluster.sync();
  }
  const double piv_min = rel_tol * dmax_s;
  const double piv_sub = dmax_s > 0.0 ? dmax_s : 1.0;

  for (int p = 0; p < nblk; ++p) {
    double* App = A + (ll)(p * NB) * lda + p * NB;
    // ---- D: diagonal tile, one warp (lane i holds row i)
    if (rank == p % CC && warp == 0) {
      double a[NB];
#pragma unroll
      for (int j = 0; j < NB; ++j) a[j] = (j <= lane) ? ldg_l2(App + (ll)lane * lda + j) : 0.0;
      bool bad = false;
      chol_tile_col<0>(a, lane, piv_min, piv_sub, bad, rdiag + p * NB);
#pragma unroll
      for (int j = 0; j < NB; ++j) stg_l2(App + (ll)lane * lda + j, j <= lane ? a[j] : 0.0);
      if (bad && lane == 0) atomicExch(status, 1);
    }
    cluster.sync();
    if (p + 1 == nblk) break;
    // ---- P: sub-diagonal tiles of column p
    const int np_tiles = nblk - p - 1;
    if (rank < np_tiles) {  // CTAs with a panel tile load L_pp and 1 / diag
      for (int e = tid; e < NB * NB; e += CT) Lp[(e / NB) * TP + (e % NB)] = ldg_l2(App + (ll)(e / NB) * lda + e % NB);
      if (tid < NB) Rp[tid] = ldg_l2(rdiag + p * NB + tid);
    }
    __syncthreads();
    for (int g = rank + CC * warp; g < np_tiles; g += CC * NW) {
      const int i = p + 1 + g;
      double* Aip = A + (ll)(i * NB) * lda + p * NB;
      double x[NB];
#pragma unroll
      for (int c = 0; c < NB; ++c) x[c] = ldg_l2(Aip + (ll)lane * lda + c);
#pragma unroll
      for (int c = 0; c < NB; ++c) {
        x[c] *= Rp[c];
#pragma unroll
        for (int c2 = c + 1; c2 < NB; ++c2) x[c2] -= x[c] * Lp[c2 * TP + c];
      }
#pragma unroll
      for (int c = 0; c < NB; ++c) stg_l2(Aip + (ll)lane * lda + c, x[c]);
    }
    cluster.sync();
    // ---- T: trailing tiles (i, j), p < j <= i, in row order
    const int nt = np_tiles * (np_tiles + 1) / 2;
    double* Ww = Wt + warp * NB * TP;
    for (int g = rank + CC * warp; g < nt; g += CC * NW) {
      int i = p + 1, rem = g;
      while (rem >= i - p) {
        rem -= i - p;
        ++i;
      }
      const int j = p + 1 + rem;
      const double* Ljp = A + (ll)(j * NB) * lda + p * NB;
      const double* Lip = A + (ll)(i * NB) * lda + p * NB;
      double* Aij = A + (ll)(i * NB) * lda + j * NB;
#pragma unroll 4
      for (int r = 0; r < NB; ++r) Ww[r * TP + lane] = ldg_l2(Ljp + (ll)r * lda + lane);
      __syncwarp();
      double x[NB], acc[NB];
#pragma unroll
      for (int t = 0; t < NB; ++t) {
        x[t] = ldg_l2(Lip + (ll)lane * lda + t);
        acc[t] = 0.0;
      }
#pragma unroll
      for (int t = 0; t < NB; ++t)
#pragma unroll
        for (int c = 0; c < NB; ++c) acc[c] += x[t] * Ww[c * TP + t];
      const int cmax = (i == j) ? lane : NB - 1;  // the diagonal tile keeps its lower part only
#pragma unroll
      for (int c = 0; c < NB; ++c)
        if (c <= cmax) stg_l2(Aij + (ll)lane * lda + c, ldg_l2(Aij + (ll)lane * lda + c) - acc[c]);
      __syncwarp();
    }
    cluster.sync();
  }
}

constexpr int SR = 8;        // rows of Y per CTA in the solve
constexpr int ST_THREADS = 64;

__global__ void __launch_bounds__(ST_THREADS)
    chol_solve_rows_kernel(double* __restrict__ Y, ll m, int k, int np, ll ldy, const double* __restrict__ L,
                           ll lda, const double* __restrict__ rdiag, const int* __restrict__ status) {
  if (*((volatile const int*)status)) return;  // the factor is not valid: the caller falls back
  extern __shared__ __align__(16) double ssm[];
  double* Qs = ssm;                // [SR][np + 1]: finished columns of these rows
  double* Lt = Qs + SR * (np + 1);  // one L tile [NB][TP]
  double* Us = Lt + NB * TP;       // updated block [SR][TP]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const ll r0 = (ll)blockIdx.x * SR;
  const int nrows = (int)min((ll)SR, m - r0);
  const int nblk = np / NB;
  const int QP = np + 1;
  for (int p = 0; p < nblk; ++p) {
    // this block of Y (columns >= k are zero)
    double acc[SR / 2];
#pragma unroll
    for (int q = 0; q < SR / 2; ++q) {
      const int r = warp * (SR / 2) + q;
      const int c = p * NB + lane;
      acc[q] = (r < nrows && c < k) ? Y[(r0 + r) * ldy + c] : 0.0;
    }
    // minus the finished columns times L_pj^T
    for (int j = 0; j < p; ++j) {
      __syncthreads();
      for (int e = tid; e < NB * NB; e += ST_THREADS)
        Lt[(e / NB) * TP + (e % NB)] = __ldg(L + (ll)(p * NB + e / NB) * lda + j * NB + e % NB);
      __syncthreads();
#pragma unroll 8
      for (int t = 0; t < NB; ++t) {
        const double l = Lt[lane * TP + t];  // L[p*NB + lane][j*NB + t]
#pragma unroll
        for (int q = 0; q < SR / 2; ++q) acc[q] -= Qs[(warp * (SR / 2) + q) * QP + j * NB + t] * l;
      }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < SR / 2; ++q) Us[(warp * (SR / 2) + q) * TP + lane] = acc[q];
    for (int e = tid; e < NB * NB; e += ST_THREADS)
      Lt[(e / NB) * TP + (e % NB)] = __ldg(L + (ll)(p * NB + e / NB) * lda + p * NB + e % NB);
    __syncthreads();
    // forward substitution with L_pp, one thread per row
    if (tid < SR) {
      double x[NB];
#pragma unroll
      for (int c = 0; c < NB; ++c) x[c] = Us[tid * TP + c];
#pragma unroll
      for (int c = 0; c < NB; ++c) {
        x[c] *= __ldg(rdiag + p * NB + c);
#pragma unroll
        for (int c2 = c + 1; c2 < NB; ++c2) x[c2] -= x[c] * Lt[c2 * TP + c];
      }
#pragma unroll
      for (int c = 0; c < NB; ++c) Qs[tid * QP + p * NB + c] = x[c];
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < SR / 2; ++q) {
      const int r = warp * (SR / 2) + q;
      const int c = p * NB + lane;
      if (r < nrows && c < k) Y[(r0 + r) * ldy + c] = Qs[r * QP + c];
    }
  }
}

}  // namespace

void chol_factor(double* A, int k, ll lda, double* rdiag, int* status, double rel_tol, cudaStream_t s,
                 double shift_rel) {
  const int np = chol_padded(k);
  if (k < 1 || np > CHOL_MAX) throw std::invalid_argument("chol_factor: order outside 1..512");
  if (lda < np) throw std::invalid_argument("chol_factor: lda below the padded order");
  static std::atomic<unsigned long long> attr{0};
  const int smem = (int)sizeof(double) * (NB * TP + NB + NW * NB * TP);
  set_smem_attr_once(attr, (const void*)chol_cluster_kernel, smem);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(CC);
  cfg.blockDim = dim3(CT);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = CC;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  DMRG2_CUDA(cudaLaunchKernelEx(&cfg, chol_cluster_kernel, A, k, np, lda, rdiag, status, rel_tol, shift_rel));
  DMRG2_CHECK_LAUNCH();
}

void chol_solve_rows(double* Y, ll m, int k, ll ldy, const double* L, ll lda, const double* rdiag,
                     const int* status, cudaStream_t s) {
  const int np = chol_padded(k);
  if (m < 1) return;
  static std::atomic<unsigned long long> attr{0};
  const int smem = (int)sizeof(double) * (SR * (np + 1) + NB * TP + SR * TP);
  constexpr int smem_max = (int)sizeof(double) * (SR * (CHOL_MAX + 1) + NB * TP + SR * TP);
  set_smem_attr_once(attr, (const void*)chol_solve_rows_kernel, smem_max);  // covers every order
  const ll grid = (m + SR - 1) / SR;
  if (grid > 2147483647LL) throw std::invalid_argument("chol_solve_rows: too many rows");
  chol_solve_rows_kernel<<<(unsigned)grid, ST_THREADS, smem, s>>>(Y, m, k, np, ldy, L, lda, rdiag, status);
  DMRG2_CHECK_LAUNCH();
}

}  // namespace dmrg2
