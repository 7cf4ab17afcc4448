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

// ---------------------------------------------------------------------------
// cholinv_cluster_kernel: X = L^{-1}, L L^T = G (+ shift), for orders k <= 256, in one
// cluster of 8 CTAs with every tile in shared memory: CTA r holds block row r of G
// (turned into L in place) and block row r of X, and stages the tiles it needs from
// its peers (distributed shared memory) in a third area. Per tile column p:
//   D  CTA p, warp 0: in-register Cholesky of the diagonal tile (rsqrt, one shuffle
//      broadcast per column); warp 1 then inverts it into X_pp off the critical path
//      (after the CTA has arrived at the cluster barrier);
//   P  CTAs r > p: L_rp = A_rp L_pp^{-T} by forward substitution (lane = row);
//   T  CTAs r > p: A_rj -= L_rp L_jp^T for p < j <= r (one warp per tile). CTA p+1
//      owns only tile (p+1, p+1) and factors it right after (look-ahead: no barrier
//      between its update and the next diagonal factorisation).
// Then X by tile diagonals s = 1 .. nblk-1: X_{r,r-s} = -X_rr sum_j L_rj X_{j,r-s}
// (CTA r, its peers' X tiles staged), and each CTA writes its block row of X (zeros
// above the diagonal) to global memory. Two cluster barriers per tile column and one
// per tile diagonal; nothing leaves shared memory until the end.
// ---------------------------------------------------------------------------
constexpr int CI_MAXB = 8;
constexpr int CI_THREADS = 256;
constexpr int CI_TILE = NB * TP;  // doubles per padded tile
constexpr size_t CI_SMEM = sizeof(double) * (3 * CI_MAXB * CI_TILE + 2 * NB);

__device__ inline void cl_arrive() { asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory"); }
__device__ inline void cl_wait() { asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory"); }

// column J of the in-register Cholesky of one diagonal tile (lane i holds row i) with a
// reciprocal square root per pivot, then the columns after it
template <int J>
__device__ __forceinline__ void ci_tile_col(double (&a)[NB], int lane, double piv_min, double piv_sub,
                                            bool& bad, double* rd) {
  double piv = __shfl_sync(0xffffffffu, a[J], J);
  if (!(piv > piv_min)) {  // also catches NaN
    bad = true;
    piv = piv_sub;
  }
  const double r = rsqrt(piv);
  if (lane == J) {
    a[J] = piv * r;
    rd[J] = r;
  } else if (lane > J) {
    a[J] *= r;
  }
#pragma unroll
  for (int c = J + 1; c < NB; ++c) {
    const double lc = __shfl_sync(0xffffffffu, a[J], c);
    if (lane >= c) a[c] -= a[J] * lc;
  }
  if constexpr (J + 1 < NB) ci_tile_col<J + 1>(a, lane, piv_min, piv_sub, bad, rd);
}

__global__ void __launch_bounds__(CI_THREADS, 1)
    cholinv_cluster_kernel(const double* __restrict__ G, int k, int np, ll ldg, double* __restrict__ X, ll ldx,
                           int* __restrict__ status, double rel_tol, double shift_rel) {
  cg::cluster_group cluster = cg::this_cluster();
  const int r = (int)cluster.block_rank();
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nblk = np / NB;
  extern __shared__ __align__(16) double cism[];
  double* Lt = cism;                           // [CI_MAXB] tiles: block row r of G -> L
  double* Xt = Lt + CI_MAXB * CI_TILE;         // [CI_MAXB] tiles: block row r of X
  double* St = Xt + CI_MAXB * CI_TILE;         // [CI_MAXB] staged tiles of peers
  double* Rd = St + CI_MAXB * CI_TILE;         // 1 / diag of this CTA's L_rr
  double* Rs = Rd + NB;                        // staged 1 / diag of L_pp
  __shared__ double tr_s, dmax_s;
  auto T_ = [](double* base, int t) { return base + t * CI_TILE; };

  // trace and largest diagonal entry of G (every CTA reads them from global memory)
  if (warp == 0) {
    double m = 0.0, tr = 0.0;
    for (int i = lane; i < k; i += 32) {
      const double a = G[(ll)i * ldg + i];
      m = fmax(m, a);
      tr += a;
    }
    for (int o = 16; o > 0; o >>= 1) {
      m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
      tr += __shfl_xor_sync(0xffffffffu, tr, o);
    }
    if (lane == 0) {
      tr_s = tr;
      dmax_s = m + shift_rel * tr;
    }
  }
  __syncthreads();
  const double shift = shift_rel * tr_s;
  const double piv_min = rel_tol * dmax_s;
  const double piv_sub = dmax_s > 0.0 ? dmax_s : 1.0;
  // block row r of G (+ shift on the diagonal; identity beyond k; lower part of the diagonal tile)
  if (r < nblk)
    for (int j = 0; j <= r; ++j)
      for (int e = tid; e < NB * NB; e += CI_THREADS) {
        const int row = e >> 5, col = e & 31;
        const int gi = r * NB + row, gj = j * NB + col;
        double v;
        if (gi < k && gj < k) v = (j < r || col <= row) ? G[(ll)gi * ldg + gj] + (gi == gj ? shift : 0.0) : 0.0;
        else v = (gi == gj) ? 1.0 : 0.0;
        T_(Lt, j)[row * TP + col] = v;
      }
  cluster.sync();

  for (int p = 0; p < nblk; ++p) {
    // ---- D: diagonal tile of CTA p (its tile p, already updated by every earlier column)
    if (r == p && warp == 0) {
      double a[NB];
      double* Lpp = T_(Lt, p);
#pragma unroll
      for (int j = 0; j < NB; ++j) a[j] = (j <= lane) ? Lpp[lane * TP + j] : 0.0;
      bool bad = false;
      ci_tile_col<0>(a, lane, piv_min, piv_sub, bad, Rd);
#pragma unroll
      for (int j = 0; j < NB; ++j) Lpp[lane * TP + j] = (j <= lane) ? a[j] : 0.0;
      if (bad && lane == 0) atomicExch(status, 1);
    }
    __syncthreads();  // L_pp and Rd written before the barrier and before warp 1 reads them
    cl_arrive();
    if (r == p && warp == 1) {
      // X_pp = L_pp^{-1}: lane c forms column c by forward substitution
      const double* Lpp = T_(Lt, p);
      double x[NB];
#pragma unroll
      for (int i = 0; i < NB; ++i) {
        double s = (i == lane) ? 1.0 : 0.0;
#pragma unroll
        for (int j = 0; j < i; ++j) s -= Lpp[i * TP + j] * x[j];
        x[i] = s * Rd[i];
      }
#pragma unroll
      for (int i = 0; i < NB; ++i) T_(Xt, p)[i * TP + lane] = x[i];
    }
    cl_wait();
    // ---- P: L_rp = A_rp L_pp^{-T}
    if (r > p && r < nblk) {
      const double* Rpp = cluster.map_shared_rank(T_(Lt, p), p);
      const double* Rrd = cluster.map_shared_rank(Rd, p);
      for (int e = tid; e < NB * NB; e += CI_THREADS) St[(e >> 5) * TP + (e & 31)] = Rpp[(e >> 5) * TP + (e & 31)];
      if (tid < NB) Rs[tid] = Rrd[tid];
      __syncthreads();
      if (warp == 0) {
        double* Arp = T_(Lt, p);
        double x[NB];
#pragma unroll
        for (int c = 0; c < NB; ++c) x[c] = Arp[lane * TP + c];
#pragma unroll
        for (int c = 0; c < NB; ++c) {
          x[c] *= Rs[c];
#pragma unroll
          for (int c2 = c + 1; c2 < NB; ++c2) x[c2] -= x[c] * St[c2 * TP + c];
        }
#pragma unroll
        for (int c = 0; c < NB; ++c) Arp[lane * TP + c] = x[c];
      }
    }
    cluster.sync();  // every L_rp of this column is final
    // ---- T: A_rj -= L_rp L_jp^T, p < j <= r
    if (r > p && r < nblk) {
      for (int j = p + 1; j < r; ++j) {  // peers' L_jp into staging slot j
        const double* src = cluster.map_shared_rank(T_(Lt, p), j);
        for (int e = tid; e < NB * NB; e += CI_THREADS) T_(St, j)[(e >> 5) * TP + (e & 31)] = src[(e >> 5) * TP + (e & 31)];
      }
      __syncthreads();
      const int j = p + 1 + warp;
      if (j <= r) {
        const double* Ljp = (j == r) ? T_(Lt, p) : T_(St, j);
        const double* Lrp = T_(Lt, p);
        double x[NB], acc[NB];
#pragma unroll
        for (int t = 0; t < NB; ++t) {
          x[t] = Lrp[lane * TP + t];
          acc[t] = 0.0;
        }
#pragma unroll
        for (int t = 0; t < NB; ++t)
#pragma unroll
          for (int c = 0; c < NB; ++c) acc[c] += x[t] * Ljp[c * TP + t];
        double* Arj = T_(Lt, j);
        const int cmax = (j == r) ? lane : NB - 1;
#pragma unroll
        for (int c = 0; c < NB; ++c)
          if (c <= cmax) Arj[lane * TP + c] -= acc[c];
      }
      __syncthreads();  // staging reused by the next column; tile (r, p+1) final before D / P
    }
  }
  cluster.sync();  // every X_pp is written
  // ---- X below the diagonal, one tile diagonal at a time
  for (int s = 1; s < nblk; ++s) {
    if (r >= s && r < nblk) {
      const int q = r - s;
      for (int j = q; j < r; ++j) {  // X_{j,q} of CTA j into staging slot j - q
        const double* src = cluster.map_shared_rank(T_(Xt, q), j);
        for (int e = tid; e < NB * NB; e += CI_THREADS) T_(St, j - q)[(e >> 5) * TP + (e & 31)] = src[(e >> 5) * TP + (e & 31)];
      }
      __syncthreads();
      // W = sum_j L_rj X_jq: warp w rows 4w..4w+3, lane = column
      double w4[4] = {0.0, 0.0, 0.0, 0.0};
      for (int j = q; j < r; ++j) {
        const double* Lrj = T_(Lt, j);
        const double* Xjq = T_(St, j - q);
#pragma unroll 8
        for (int t = 0; t < NB; ++t) {
          const double xv = Xjq[t * TP + lane];
#pragma unroll
          for (int u = 0; u < 4; ++u) w4[u] += Lrj[(4 * warp + u) * TP + t] * xv;
        }
      }
      double* Wt = T_(St, CI_MAXB - 1);  // free: at most 7 tiles are staged
#pragma unroll
      for (int u = 0; u < 4; ++u) Wt[(4 * warp + u) * TP + lane] = w4[u];
      __syncthreads();
      // X_rq = -X_rr W
      const double* Xrr = T_(Xt, r);
      double o4[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 8
      for (int t = 0; t < NB; ++t) {
        const double wv = Wt[t * TP + lane];
#pragma unroll
        for (int u = 0; u < 4; ++u) o4[u] -= Xrr[(4 * warp + u) * TP + t] * wv;
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) T_(Xt, q)[(4 * warp + u) * TP + lane] = o4[u];
    }
    cluster.sync();  // X tiles of this diagonal visible to the peers
  }
  // ---- block row r of X to global memory (lower triangle, zeros above)
  if (r < nblk)
    for (int j = 0; j < nblk; ++j)
      for (int e = tid; e < NB * NB; e += CI_THREADS) {
        const int row = e >> 5, col = e & 31;
        const int gi = r * NB + row, gj = j * NB + col;
        if (gi < k && gj < k) X[(ll)gi * ldx + gj] = (j < r || (j == r && col <= row)) ? T_(Xt, j)[row * TP + col] : 0.0;
      }
  cluster.sync();  // no CTA leaves while a peer may still read its shared memory
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

// every column of Y (rows x k, ld k) scaled to unit norm; a zero or non-finite column
// sets *status. Two passes over a grid of 32-column x CN_ROWS-row blocks: partial
// sums of squares per block (lane = column, warps stride the rows), then every block
// adds the partials of its columns and scales its rows.
constexpr int CN_ROWS = 32;
__global__ void __launch_bounds__(256) col_sumsq_kernel(const double* __restrict__ Y, ll rows, int k,
                                                        double* __restrict__ part) {
  __shared__ double ps[8][33];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int c = blockIdx.x * 32 + lane;
  const ll r0 = (ll)blockIdx.y * CN_ROWS, r1 = min(rows, r0 + CN_ROWS);
  double sq = 0.0;
  if (c < k)
    for (ll r = r0 + warp; r < r1; r += 8) {
      const double v = Y[r * k + c];
      sq += v * v;
    }
  ps[warp][lane] = sq;
  __syncthreads();
  if (warp == 0 && c < k) {
    double t = 0.0;
#pragma unroll
    for (int w = 0; w < 8; ++w) t += ps[w][lane];
    part[(ll)blockIdx.y * k + c] = t;
  }
}

__global__ void __launch_bounds__(256) col_scale_kernel(double* __restrict__ Y, ll rows, int k,
                                                        const double* __restrict__ part, int nchunks,
                                                        int* __restrict__ status) {
  __shared__ double inv[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int c = blockIdx.x * 32 + lane;
  if (warp == 0) {
    double sc = 0.0;
    if (c < k) {
      double t = 0.0;
      for (int q = 0; q < nchunks; ++q) t += part[(ll)q * k + c];  // the same order in every block
      if (t > 0.0 && isfinite(t)) sc = rsqrt(t);
      else if (blockIdx.y == 0) atomicExch(status, 1);
    }
    inv[lane] = sc;
  }
  __syncthreads();
  const ll r0 = (ll)blockIdx.y * CN_ROWS, r1 = min(rows, r0 + CN_ROWS);
  if (c < k)
    for (ll r = r0 + warp; r < r1; r += 8) Y[r * k + c] *= inv[lane];
}

__global__ void mark_unconverged_kernel(const SvdOut* out, int* status) {
  if (!out->ns_done) *status = 1;
}

}  // namespace

void mark_unconverged(const SvdOut* out, int* status, cudaStream_t s) {
  mark_unconverged_kernel<<<1, 1, 0, s>>>(out, status);
  DMRG2_CHECK_LAUNCH();
}

void col_normalize(double* Y, ll rows, int k, double* part, int* status, cudaStream_t s) {
  if (rows < 1 || k < 1) return;
  const ll nch = (rows + CN_ROWS - 1) / CN_ROWS;
  if (nch > COLNORM_MAX_CHUNKS) throw std::invalid_argument("col_normalize: too many rows");
  dim3 g((unsigned)((k + 31) / 32), (unsigned)nch);
  col_sumsq_kernel<<<g, 256, 0, s>>>(Y, rows, k, part);
  DMRG2_CHECK_LAUNCH();
  col_scale_kernel<<<g, 256, 0, s>>>(Y, rows, k, part, (int)nch, status);
  DMRG2_CHECK_LAUNCH();
}

void chol_inverse(const double* G, int k, ll ldg, double* X, ll ldx, int* status, double rel_tol, double shift_rel,
                  cudaStream_t s) {
  const int np = chol_padded(k);
  if (k < 1 || np > CI_MAXB * NB) throw std::invalid_argument("chol_inverse: order outside 1..256");
  static std::atomic<unsigned long long> attr{0};
  set_smem_attr_once(attr, (const void*)cholinv_cluster_kernel, (int)CI_SMEM);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(CI_MAXB);
  cfg.blockDim = dim3(CI_THREADS);
  cfg.dynamicSmemBytes = CI_SMEM;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = CI_MAXB;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  DMRG2_CUDA(cudaLaunchKernelEx(&cfg, cholinv_cluster_kernel, G, k, np, ldg, X, ldx, status, rel_tol, shift_rel));
  DMRG2_CHECK_LAUNCH();
}

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
