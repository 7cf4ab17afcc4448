// CholeskyQR building blocks (real FP64) for the warm-started subspace truncation.
//
// chol_tiles_kernel: blocked Cholesky factorisation of an order <= 512 symmetric
// positive definite matrix in 32 x 32 tiles, in one cluster of C = 8 or 16 CTAs.
// CTA r owns block row r in its shared memory and turns it into L's block row
// (right-looking: at tile column t it forms L_rt, then subtracts L_rt L_jt^T from
// its tiles t < j <= r). There is no cluster barrier inside the factorisation: each
// CTA publishes how many tiles of its row are final (a counter in its shared memory,
// written with release semantics after the tiles), and a CTA that needs a peer's
// tile polls that counter (acquire, bounded) and then reads the tile straight from
// the peer's shared memory. A published tile is never written again, and nothing is
// copied asynchronously, so the only exit condition is the final cluster barrier
// (no CTA leaves while a peer may still read it). Per tile column t:
//   P  CTA r > t: L_rt = A_rt X_tt^T with X_tt = L_tt^{-1} from CTA t (rows split
//      over the 8 warps);
//   T  CTA r > t: A_rj -= L_rt L_jt^T for the peers' tiles t < j < r (one warp per
//      tile, the peer tile staged in that warp's buffer) and the lower part of the
//      diagonal tile j = r (rows split over the warps);
//   D  CTA t, once its row is updated: in-register Cholesky of the diagonal tile
//      (one warp, lane = row; the chain of pivots is the critical path), then X_tt by
//      forward substitution (lane = column), then the counter says "row complete".
// The critical path is one P, one diagonal update and one D per tile column; the
// wider updates of the rows further down overlap with it. A poll that runs out marks
// the result invalid (status) and the CTA carries on with what it has, so every CTA
// reaches the final barrier.
//
// trsm_rows_kernel: Y = Z L^{-T}, 16 rows of Z per CTA, column block by column block:
// Y_b = (Z_b - sum_{j<b} Y_j L_bj^T) X_bb^T on the FP64 tensor cores (DMMA), the tiles
// of L streamed through shared memory with cp.async double buffering.
#include <cooperative_groups.h>

#include "cholqr.cuh"
#include "gemm.cuh"

namespace cg = cooperative_groups;

namespace dmrg2 {

namespace {

constexpr int NB = CHOL_NB;
constexpr int TP = NB + 1;           // padded tile row in shared memory (conflict-free columns)
constexpr int TT = NB * TP;          // doubles per padded tile
constexpr int CT_THREADS = 256;      // 8 warps
constexpr int CT_WARPS = CT_THREADS / 32;
constexpr long long CT_SPIN = 1ll << 22;  // polls of a peer's counter before giving up

__device__ inline int ld_acquire_cluster(const int* p) {
  int v;
  asm volatile("ld.acquire.cluster.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ inline void st_release_cluster(int* p, int v) {
  asm volatile("st.release.cluster.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
// true once *peer_done >= need (the calling thread acquires), false after CT_SPIN polls
__device__ inline bool wait_tiles(const int* peer_done, int need) {
  for (long long it = 0; it < CT_SPIN; ++it)
    if (ld_acquire_cluster(peer_done) >= need) return true;
  return false;
}

// column J of the in-register Cholesky of one diagonal tile (lane i holds row i) with a
// reciprocal square root per pivot, then the columns after it; compile-time J keeps
// every index of a[] static
template <int J>
__device__ __forceinline__ void tile_chol_col(double (&a)[NB], int lane, double piv_min, double piv_sub, bool& bad,
                                              double* rd) {
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
  if constexpr (J + 1 < NB) tile_chol_col<J + 1>(a, lane, piv_min, piv_sub, bad, rd);
}

template <int C>
__global__ void __launch_bounds__(CT_THREADS, 1)
    chol_tiles_kernel(const double* __restrict__ G, int k, int nb, ll ldg, double* __restrict__ LX, ll ldx,
                      int* __restrict__ status, double rel_tol, double shift_rel) {
  cg::cluster_group cluster = cg::this_cluster();
  const int r = (int)cluster.block_rank();
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  extern __shared__ __align__(16) double ctsm[];
  double* Lt = ctsm;                 // [C] tiles of block row r: A_rj, turned into L_rj
  double* Xr = Lt + C * TT;          // X_rr = L_rr^{-1} (zeros above the diagonal)
  double* Xs = Xr + TT;              // X_tt of the tile column being solved, staged
  double* Ws = Xs + TT;              // [CT_WARPS] a peer's L_jt, staged per warp
  double* Rd = Ws + CT_WARPS * TT;   // 1 / diag of L_rr
  __shared__ int done_s;             // tiles of this block row that are final (read by peers)
  __shared__ int fail_s;
  __shared__ double tr_s, dmax_s;
  auto T_ = [](double* base, int t) { return base + t * TT; };

  if (tid == 0) {
    done_s = 0;
    fail_s = 0;
  }
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
  if (r < nb)
    for (int j = 0; j <= r; ++j)
      for (int e = tid; e < NB * NB; e += CT_THREADS) {
        const int row = e >> 5, col = e & 31;
        const int gi = r * NB + row, gj = j * NB + col;
        double v;
        if (gi < k && gj < k) v = (j < r || col <= row) ? G[(ll)gi * ldg + gj] + (gi == gj ? shift : 0.0) : 0.0;
        else v = (gi == gj) ? 1.0 : 0.0;
        T_(Lt, j)[row * TP + col] = v;
      }
  // every counter is initialised and every block row read before any CTA polls a peer
  // or writes LX (which may be the buffer G is in)
  cluster.sync();

  bool bad = false;
  if (r < nb) {
    for (int t = 0; t < r; ++t) {
      // ---- P: L_rt = A_rt X_tt^T once CTA t has published X_tt (its row complete); one
      // thread polls (the peer's shared memory serves its critical factorisation meanwhile)
      // and the CTA barrier passes what it acquired on to the other threads
      if (tid == 0 && !wait_tiles(cluster.map_shared_rank(&done_s, t), t + 1)) fail_s = 1;
      __syncthreads();
      {
        const double* Xp = cluster.map_shared_rank(Xr, t);
        for (int e = tid; e < NB * NB; e += CT_THREADS) Xs[(e >> 5) * TP + (e & 31)] = Xp[(e >> 5) * TP + (e & 31)];
      }
      __syncthreads();
      {
        double* Art = T_(Lt, t);
        double o[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 8
        for (int s = 0; s < NB; ++s) {
          const double xv = Xs[lane * TP + s];  // X_tt[c = lane][s]
#pragma unroll
          for (int u = 0; u < 4; ++u) o[u] += Art[(4 * warp + u) * TP + s] * xv;
        }
        __syncwarp();  // the warp's rows are read before they are overwritten
#pragma unroll
        for (int u = 0; u < 4; ++u) Art[(4 * warp + u) * TP + lane] = o[u];
      }
      __syncthreads();
      if (tid == 0) st_release_cluster(&done_s, t + 1);  // L_rt is final
      // ---- T: A_rj -= L_rt L_jt^T for t < j <= r
      const double* Lrt = T_(Lt, t);
      for (int q = warp; q < r - t - 1; q += CT_WARPS) {  // the peers' tiles j = t+1 .. r-1
        const int j = t + 1 + q;
        if (lane == 0 && !wait_tiles(cluster.map_shared_rank(&done_s, j), t + 1)) fail_s = 1;
        __syncwarp();  // lane 0 acquired the tile for the warp
        const double* src = cluster.map_shared_rank(T_(Lt, t), j);  // L_jt in CTA j
        double* W = T_(Ws, warp);
        {
          double v[NB];
#pragma unroll
          for (int c = 0; c < NB; ++c) v[c] = src[c * TP + lane];
#pragma unroll
          for (int c = 0; c < NB; ++c) W[c * TP + lane] = v[c];
        }
        __syncwarp();
        double x[NB], acc[NB];  // lane = row i of A_rj: acc[c] = sum_s L_rt[i][s] L_jt[c][s]
#pragma unroll
        for (int s = 0; s < NB; ++s) {
          x[s] = Lrt[lane * TP + s];
          acc[s] = 0.0;
        }
#pragma unroll
        for (int s = 0; s < NB; ++s)
#pragma unroll
          for (int c = 0; c < NB; ++c) acc[c] += x[s] * W[c * TP + s];
        double* Arj = T_(Lt, j);
#pragma unroll
        for (int c = 0; c < NB; ++c) Arj[lane * TP + c] -= acc[c];
        __syncwarp();  // W is staged again by this warp's next tile
      }
      {  // the diagonal tile: rows 4w .. 4w+3, lane = column, lower part only
        double* Arr = T_(Lt, r);
        double o[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 8
        for (int s = 0; s < NB; ++s) {
          const double lv = Lrt[lane * TP + s];
#pragma unroll
          for (int u = 0; u < 4; ++u) o[u] += Lrt[(4 * warp + u) * TP + s] * lv;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
          if (lane <= 4 * warp + u) Arr[(4 * warp + u) * TP + lane] -= o[u];
      }
      __syncthreads();  // tile (r, t+1) and the diagonal tile are final for this column
    }
    // ---- D: L_rr (registers, lane = row), then X_rr = L_rr^{-1} (lane = column)
    if (warp == 0) {
      double* Lrr = T_(Lt, r);
      double a[NB];
#pragma unroll
      for (int j = 0; j < NB; ++j) a[j] = (j <= lane) ? Lrr[lane * TP + j] : 0.0;
      tile_chol_col<0>(a, lane, piv_min, piv_sub, bad, Rd);
#pragma unroll
      for (int j = 0; j < NB; ++j) Lrr[lane * TP + j] = (j <= lane) ? a[j] : 0.0;
      __syncwarp();
      double x[NB];
#pragma unroll
      for (int i = 0; i < NB; ++i) {
        // four partial sums break the dependent chain of the row's dot product
        double s0 = (i == lane) ? 1.0 : 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
#pragma unroll
        for (int j = 0; j + 3 < i; j += 4) {
          s0 -= Lrr[i * TP + j] * x[j];
          s1 -= Lrr[i * TP + j + 1] * x[j + 1];
          s2 -= Lrr[i * TP + j + 2] * x[j + 2];
          s3 -= Lrr[i * TP + j + 3] * x[j + 3];
        }
#pragma unroll
        for (int j = i & ~3; j < i; ++j) s0 -= Lrr[i * TP + j] * x[j];
        x[i] = ((s0 + s1) + (s2 + s3)) * Rd[i];
      }
#pragma unroll
      for (int i = 0; i < NB; ++i) Xr[i * TP + lane] = x[i];
    }
    __syncthreads();
    if (tid == 0) st_release_cluster(&done_s, r + 1);  // the whole row, X_rr included
    // ---- block row r of LX: L_rj below the diagonal, X_rr on it
    for (int j = 0; j <= r; ++j) {
      const double* src = (j < r) ? T_(Lt, j) : Xr;
      for (int e = tid; e < NB * NB; e += CT_THREADS)
        LX[(ll)(r * NB + (e >> 5)) * ldx + j * NB + (e & 31)] = src[(e >> 5) * TP + (e & 31)];
    }
  }
  if (bad) atomicExch(status, 1);
  cluster.sync();  // no CTA leaves while a peer may still read its shared memory
  if (tid == 0 && fail_s) atomicExch(status, 1);
}

// ---------------------------------------------------------------------------
// trsm_rows_kernel
// ---------------------------------------------------------------------------
constexpr int TR_R = 16;                     // rows of Z per CTA (one DMMA row block)
constexpr int TR_THREADS = 128;              // warp w: output columns 8w .. 8w+7 of a block
constexpr int TR_LP = NB + 4;                // staged tile row: 288 bytes (16-byte aligned rows)
constexpr int TR_TILE = NB * TR_LP;

__device__ inline void tr_stage(double* dst, const double* LX, ll ldx, int b, int j, int tid) {
  // tile (b, j) of LX: 32 rows x 32 doubles = 512 chunks of 16 bytes, four per thread
#pragma unroll
  for (int h = 0; h < 4; ++h) {
    const int e = tid + h * TR_THREADS;
    const int row = e >> 4, c2 = (e & 15) * 2;
    cp_async_16(dst + row * TR_LP + c2, LX + (ll)(b * NB + row) * ldx + j * NB + c2, true);
  }
}

__global__ void __launch_bounds__(TR_THREADS)
    trsm_rows_kernel(const double* __restrict__ Z, ll rows, int k, int nb, const double* __restrict__ LX, ll ldx,
                     double* __restrict__ Y, const int* __restrict__ status) {
  if (*((volatile const int*)status)) return;  // the factor is not valid: the caller falls back
  extern __shared__ __align__(16) double tsm[];
  const int YP = nb * NB + 4;     // row of the finished blocks
  double* Yf = tsm;               // [TR_R][YP]: Y of this CTA's rows, block by block
  double* Lb = Yf + TR_R * YP;    // [2][TR_TILE]: staged tiles
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int gq = lane >> 2, tq = lane & 3;
  const ll r0 = (ll)blockIdx.x * TR_R;
  const int ntiles = nb * (nb + 1) / 2;  // (b, j) for j <= b, in that order
  // tile s of the sequence -> (b, j)
  auto tile_of = [](int s, int& b, int& j) {
    b = 0;
    while (s > b) {
      s -= b + 1;
      ++b;
    }
    j = s;
  };
  {
    int b, j;
    tile_of(0, b, j);
    tr_stage(Lb, LX, ldx, b, j, tid);
    cp_async_commit();
  }
  int s = 0;
  for (int b = 0; b < nb; ++b) {
    const int c0 = b * NB + warp * 8 + 2 * tq;  // this lane's two output columns
    double acc[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const ll row = r0 + gq + ((q & 2) ? 8 : 0);
      const int col = c0 + (q & 1);
      acc[q] = (row < rows && col < k) ? Z[row * k + col] : 0.0;
    }
    for (int j = 0; j <= b; ++j, ++s) {
      if (j == b) {
        // the update of block b is complete: store it for the X_bb product (no warp
        // reads block b of Yf before the barrier below)
#pragma unroll
        for (int q = 0; q < 4; ++q) Yf[(gq + ((q & 2) ? 8 : 0)) * YP + c0 + (q & 1)] = acc[q];
      }
      if (s + 1 < ntiles) {  // prefetch the next tile into the other buffer
        int bn, jn;
        tile_of(s + 1, bn, jn);
        tr_stage(Lb + ((s + 1) & 1) * TR_TILE, LX, ldx, bn, jn, tid);
      }
      cp_async_commit();
      cp_async_wait<1>();
      __syncthreads();  // tile s staged (and, for j == b, the updated block in Yf)
      const double* Lt = Lb + (s & 1) * TR_TILE;
      if (j < b) {
        // acc -= Y_j L_bj^T: A = Y_j (16 x 32), B[kk][n] = L_bj[n][kk]
#pragma unroll
        for (int kk = 0; kk < NB; kk += 4) {
          const double a0 = -Yf[gq * YP + j * NB + kk + tq];
          const double a1 = -Yf[(gq + 8) * YP + j * NB + kk + tq];
          const double b0 = Lt[(warp * 8 + gq) * TR_LP + kk + tq];
          dmma16x8x4(acc, a0, a1, b0);
        }
      } else {
        // Y_b = (Z_b - ...) X_bb^T: the updated block is in Yf (written before the
        // barrier above), the product goes to registers, then back to Yf and Y
        double out[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int kk = 0; kk < NB; kk += 4) {
          const double a0 = Yf[gq * YP + b * NB + kk + tq];
          const double a1 = Yf[(gq + 8) * YP + b * NB + kk + tq];
          const double b0 = Lt[(warp * 8 + gq) * TR_LP + kk + tq];
          dmma16x8x4(out, a0, a1, b0);
        }
        __syncthreads();  // every warp has read the updated block
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int rr = gq + ((q & 2) ? 8 : 0);
          const int col = c0 + (q & 1);
          Yf[rr * YP + col] = out[q];
          if (r0 + rr < rows && col < k) Y[(r0 + rr) * k + col] = out[q];
        }
      }
      __syncthreads();  // buffer s & 1 is free for the prefetch of tile s + 2
    }
  }
  cp_async_wait<0>();
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

template <int C>
void chol_tiles_launch(const double* G, int k, int nb, ll ldg, double* LX, ll ldx, int* status, double rel_tol,
                       double shift_rel, cudaStream_t s) {
  constexpr size_t smem = sizeof(double) * ((size_t)(C + 2 + CT_WARPS) * TT + NB);
  static std::atomic<unsigned long long> attr{0};
  set_smem_attr_once(attr, (const void*)chol_tiles_kernel<C>, (int)smem);
  if constexpr (C > 8) {
    static std::atomic<unsigned long long> attr_c{0};
    func_attr_once(attr_c, (const void*)chol_tiles_kernel<C>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(C);
  cfg.blockDim = dim3(CT_THREADS);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = C;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  DMRG2_CUDA(cudaLaunchKernelEx(&cfg, chol_tiles_kernel<C>, G, k, nb, ldg, LX, ldx, status, rel_tol, shift_rel));
  DMRG2_CHECK_LAUNCH();
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

void chol_tiles(const double* G, int k, ll ldg, double* LX, ll ldx, int* status, double rel_tol, double shift_rel,
                cudaStream_t s) {
  const int np = chol_padded(k);
  if (k < 1 || np > CHOL_MAX) throw std::invalid_argument("chol_tiles: order outside 1..512");
  if (ldg < k || ldx < np) throw std::invalid_argument("chol_tiles: leading dimension too small");
  const int nb = np / NB;
  if (nb <= 8) chol_tiles_launch<8>(G, k, nb, ldg, LX, ldx, status, rel_tol, shift_rel, s);
  else chol_tiles_launch<16>(G, k, nb, ldg, LX, ldx, status, rel_tol, shift_rel, s);
}

void trsm_rows(const double* Z, ll rows, int k, const double* LX, ll ldx, double* Y, const int* status,
               cudaStream_t s) {
  if (rows < 1) return;
  const int np = chol_padded(k);
  if (k < 1 || np > CHOL_MAX) throw std::invalid_argument("trsm_rows: order outside 1..512");
  if (ldx < np || (ldx & 1)) throw std::invalid_argument("trsm_rows: LX leading dimension");
  const int nb = np / NB;
  const size_t smem = sizeof(double) * ((size_t)TR_R * (nb * NB + 4) + 2 * TR_TILE);
  constexpr size_t smem_max = sizeof(double) * ((size_t)TR_R * (CHOL_MAX + 4) + 2 * TR_TILE);
  static std::atomic<unsigned long long> attr{0};
  set_smem_attr_once(attr, (const void*)trsm_rows_kernel, (int)smem_max);  // covers every order
  const ll grid = (rows + TR_R - 1) / TR_R;
  if (grid > 2147483647LL) throw std::invalid_argument("trsm_rows: too many rows");
  trsm_rows_kernel<<<(unsigned)grid, TR_THREADS, smem, s>>>(Z, rows, k, nb, LX, ldx, Y, status);
  DMRG2_CHECK_LAUNCH();
}

}  // namespace dmrg2
