// FP64 / complex128 GEMM on the sm_100a double-precision tensor cores.
//
// Blackwell's tcgen05 tensor-core instructions have no FP64 kind; FP64 tensor
// work on sm_100a is issued with the warp-level DMMA instruction
// mma.sync.m16n8k4.f64. This kernel stages A/B tiles in shared memory with a
// 3-deep cp.async pipeline and runs 32x32 (real) or 32x16 (complex) warp tiles
// of DMMA. Complex products are four real DMMAs on interleaved (re, im) tiles.
//
// C[z] (M x N, row-major, ldc) = alpha * op(A[z]) * op(B[z]) + beta * C[z]
//   op(A) = A, A^T, conj(A) or A^H (M x K); op(B) = B or B^T (K x N)
//   storage: A[m*lda+k] (no trans) / A[k*lda+m] (trans), same for B.
// Batches form a 2-level grid z = z1 * nb2 + z2 with independent strides, so
// the strided views of the DMRG contractions map onto one launch each.
#pragma once

#include <cooperative_groups.h>

#include "common.cuh"

namespace dmrg2 {

struct GemmArgs {
  int M, N, K;
  const void* A;
  ll lda, sA1, sA2;
  const void* B;
  ll ldb, sB1, sB2;
  void* C;
  ll ldc, sC1, sC2;
  int nb2;
  double alpha_re, alpha_im, beta_re, beta_im;
  const int* skip;  // optional device flag: when non-zero the launch does nothing
  int kchunk;       // split-K: blockIdx.z selects the K slice [z*kchunk, (z+1)*kchunk) (0 = off)
  int kcluster;     // > 1: the K slices of a tile form one thread-block cluster and are summed
                    // in it, C = alpha sum + beta C written by the cluster (0: partials to C)
};

__device__ __forceinline__ void cp_async_8(void* smem, const void* gmem, bool pred) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  int n = pred ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}
__device__ __forceinline__ void cp_async_16(void* smem, const void* gmem, bool pred) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  int n = pred ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

__device__ __forceinline__ void dmma16x8x4(double (&c)[4], double a0, double a1, double b0) {
  asm volatile(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, "
      "{%0,%1,%2,%3};\n"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a0), "d"(a1), "d"(b0));
}

// CTA tile: BM x BN outputs, BK deep per pipeline stage, warps of WM x WN
template <int BM_, int BN_, int BK_, int WM_, int WN_, int MNPAD_>
struct TileCfg {
  static constexpr int BM = BM_, BN = BN_, BK = BK_, WM = WM_, WN = WN_, STAGES = 3;
  static constexpr int THREADS = (BM / WM) * (BN / WN) * 32;
  static constexpr int KPAD = 4, MNPAD = MNPAD_;
};
using TileD64 = TileCfg<64, 64, 16, 32, 32, 4>;  // real, the default
using TileD32 = TileCfg<32, 32, 16, 16, 16, 4>;  // real, small outputs (more CTAs)
using TileZ64 = TileCfg<64, 32, 8, 32, 16, 2>;   // complex

// the default tile of each scalar type (split-K heuristics of the callers use it)
template <typename T>
struct GemmTile;
template <>
struct GemmTile<double> : TileD64 {};
template <>
struct GemmTile<zc> : TileZ64 {};

template <typename T, typename G, bool TA, bool TB>
struct GemmSmem {
  // A: K-contiguous [BM][BK+pad] when not transposed, M-contiguous [BK][BM+pad] otherwise
  static constexpr int PA = TA ? (G::BM + G::MNPAD) : (G::BK + G::KPAD);
  static constexpr int SA = TA ? G::BK * PA : G::BM * PA;
  // B: N-contiguous [BK][BN+pad] when not transposed, K-contiguous [BN][BK+pad] otherwise
  static constexpr int PB = TB ? (G::BK + G::KPAD) : (G::BN + G::MNPAD);
  static constexpr int SB = TB ? G::BN * PB : G::BK * PB;
  static constexpr int STAGE = SA + SB;
  static constexpr size_t BYTES = (size_t)G::STAGES * STAGE * sizeof(T);
  __device__ static int a_idx(int m, int k) { return TA ? k * PA + m : m * PA + k; }
  __device__ static int b_idx(int k, int n) { return TB ? n * PB + k : k * PB + n; }
};

template <typename T, typename G, bool TA, bool TB, bool CA>
__global__ void __launch_bounds__(G::THREADS) gemm_kernel(GemmArgs g) {
  using S = GemmSmem<T, G, TA, TB>;
  constexpr int BM = G::BM, BN = G::BN, BK = G::BK, WM = G::WM, WN = G::WN;
  constexpr int MI = WM / 16, NI = WN / 8;
  constexpr bool CPLX = ST<T>::cplx;
  if (g.skip && *((volatile const int*)g.skip)) return;

  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* smem = reinterpret_cast<T*>(smem_raw);

  const int z = blockIdx.z;
  const int z1 = z / g.nb2, z2 = z - z1 * g.nb2;
  const T* Ab = reinterpret_cast<const T*>(g.A) + z1 * g.sA1 + z2 * g.sA2;
  const T* Bb = reinterpret_cast<const T*>(g.B) + z1 * g.sB1 + z2 * g.sB2;
  T* Cb = reinterpret_cast<T*>(g.C) + z1 * g.sC1 + z2 * g.sC2;
  const int M = g.M, N = g.N;
  // split-K: this CTA covers K range [kbeg, K)
  const int kbeg = g.kchunk > 0 ? z * g.kchunk : 0;
  const int K = g.kchunk > 0 ? min(g.K, kbeg + g.kchunk) : g.K;
  const ll lda = g.lda, ldb = g.ldb, ldc = g.ldc;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;

  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const int wm = warp / (BN / WN), wn = warp % (BN / WN);
  const int gq = lane >> 2, tq = lane & 3;

  auto load_stage = [&](int stage, int kt) {
    T* As = smem + stage * S::STAGE;
    T* Bs = As + S::SA;
    const int k0 = kbeg + kt * BK;
#pragma unroll
    for (int j = 0; j < (BM * BK) / G::THREADS; ++j) {
      int e = tid + j * G::THREADS;
      int m, k;
      if (!TA) { m = e / BK; k = e % BK; } else { k = e / BM; m = e % BM; }
      int gm = m0 + m, gk = k0 + k;
      bool p = (gm < M) && (gk < K);
      const T* src = p ? (Ab + (TA ? (ll)gk * lda + gm : (ll)gm * lda + gk)) : Ab;
      if constexpr (CPLX) cp_async_16(As + S::a_idx(m, k), src, p);
      else cp_async_8(As + S::a_idx(m, k), src, p);
    }
#pragma unroll
    for (int j = 0; j < (BN * BK) / G::THREADS; ++j) {
      int e = tid + j * G::THREADS;
      int n, k;
      if (TB) { n = e / BK; k = e % BK; } else { k = e / BN; n = e % BN; }
      int gn = n0 + n, gk = k0 + k;
      bool p = (gn < N) && (gk < K);
      const T* src = p ? (Bb + (TB ? (ll)gn * ldb + gk : (ll)gk * ldb + gn)) : Bb;
      if constexpr (CPLX) cp_async_16(Bs + S::b_idx(k, n), src, p);
      else cp_async_8(Bs + S::b_idx(k, n), src, p);
    }
  };

  double acc_re[MI][NI][4];
  double acc_im[CPLX ? MI : 1][CPLX ? NI : 1][4];
#pragma unroll
  for (int i = 0; i < MI; ++i)
#pragma unroll
    for (int j = 0; j < NI; ++j)
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        acc_re[i][j][r] = 0.0;
        if constexpr (CPLX) acc_im[i][j][r] = 0.0;
      }

  const int nk = (K - kbeg + BK - 1) / BK;
#pragma unroll
  for (int s = 0; s < G::STAGES - 1; ++s) {
    if (s < nk) load_stage(s, s);
    cp_async_commit();
  }

  for (int kt = 0; kt < nk; ++kt) {
    cp_async_wait<G::STAGES - 2>();
    __syncthreads();
    {
      int nxt = kt + G::STAGES - 1;
      if (nxt < nk) load_stage(nxt % G::STAGES, nxt);
      cp_async_commit();
    }
    const T* As = smem + (kt % G::STAGES) * S::STAGE;
    const T* Bs = As + S::SA;
#pragma unroll
    for (int kk = 0; kk < BK; kk += 4) {
      if constexpr (!CPLX) {
        double a[MI][2], b[NI];
#pragma unroll
        for (int i = 0; i < MI; ++i) {
          int m = wm * WM + i * 16 + gq;
          a[i][0] = As[S::a_idx(m, kk + tq)];
          a[i][1] = As[S::a_idx(m + 8, kk + tq)];
        }
#pragma unroll
        for (int j = 0; j < NI; ++j) b[j] = Bs[S::b_idx(kk + tq, wn * WN + j * 8 + gq)];
#pragma unroll
        for (int i = 0; i < MI; ++i)
#pragma unroll
          for (int j = 0; j < NI; ++j) dmma16x8x4(acc_re[i][j], a[i][0], a[i][1], b[j]);
      } else {
        double ar[MI][2], ai[MI][2], nai[MI][2], br[NI], bi[NI];
#pragma unroll
        for (int i = 0; i < MI; ++i) {
          int m = wm * WM + i * 16 + gq;
          zc v0 = As[S::a_idx(m, kk + tq)];
          zc v1 = As[S::a_idx(m + 8, kk + tq)];
          ar[i][0] = v0.re; ai[i][0] = CA ? -v0.im : v0.im;
          ar[i][1] = v1.re; ai[i][1] = CA ? -v1.im : v1.im;
          nai[i][0] = -ai[i][0]; nai[i][1] = -ai[i][1];
        }
#pragma unroll
        for (int j = 0; j < NI; ++j) {
          zc v = Bs[S::b_idx(kk + tq, wn * WN + j * 8 + gq)];
          br[j] = v.re; bi[j] = v.im;
        }
#pragma unroll
        for (int i = 0; i < MI; ++i)
#pragma unroll
          for (int j = 0; j < NI; ++j) {
            dmma16x8x4(acc_re[i][j], ar[i][0], ar[i][1], br[j]);
            dmma16x8x4(acc_re[i][j], nai[i][0], nai[i][1], bi[j]);
            dmma16x8x4(acc_im[i][j], ar[i][0], ar[i][1], bi[j]);
            dmma16x8x4(acc_im[i][j], ai[i][0], ai[i][1], br[j]);
          }
      }
    }
  }
  cp_async_wait<0>();

  const bool use_beta = (g.beta_re != 0.0) || (g.beta_im != 0.0);
  if (g.kcluster > 1) {
    // split-K inside a cluster: each slice leaves its partial tile in shared memory (the
    // pipeline buffers are free now), then each CTA sums a share of the tile's rows over
    // the slices, in slice order, reading its peers' tiles (distributed shared memory)
    constexpr int PP = BN + (CPLX ? 2 : 4);  // row pitch of the partial tile
    static_assert(BM * PP <= G::STAGES * S::STAGE, "partial tile must fit the pipeline buffers");
    __syncthreads();
    T* part = smem;
#pragma unroll
    for (int i = 0; i < MI; ++i)
#pragma unroll
      for (int j = 0; j < NI; ++j)
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const int lr = wm * WM + i * 16 + gq + ((r & 2) ? 8 : 0);
          const int lc = wn * WN + j * 8 + 2 * tq + (r & 1);
          if constexpr (!CPLX) part[lr * PP + lc] = acc_re[i][j][r];
          else part[lr * PP + lc] = mkz(acc_re[i][j][r], acc_im[i][j][r]);
        }
    cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
    cl.sync();
    const int ns = g.kcluster, q = (int)cl.block_rank();
    const int rows_per = (BM + ns - 1) / ns;
    const int rb = q * rows_per, re = min(BM, rb + rows_per);
    for (int e = tid; e < (re - rb) * BN; e += G::THREADS) {
      const int lr = rb + e / BN, lc = e % BN;
      const int row = m0 + lr, col = n0 + lc;
      if (row < M && col < N) {
        T sum = ST<T>::zero();
        for (int z2 = 0; z2 < ns; ++z2) sum = sum + cl.map_shared_rank(part, z2)[lr * PP + lc];
        T* dst = Cb + (ll)row * ldc + col;
        if constexpr (!CPLX) {
          double v = g.alpha_re * sum;
          if (use_beta) v += g.beta_re * (*dst);
          *dst = v;
        } else {
          zc v = mkz(g.alpha_re * sum.re - g.alpha_im * sum.im, g.alpha_re * sum.im + g.alpha_im * sum.re);
          if (use_beta) {
            zc o = *dst;
            v.re += g.beta_re * o.re - g.beta_im * o.im;
            v.im += g.beta_re * o.im + g.beta_im * o.re;
          }
          *dst = v;
        }
      }
    }
    cl.sync();  // no CTA leaves while a peer may still read its partial tile
    return;
  }

  // epilogue
#pragma unroll
  for (int i = 0; i < MI; ++i)
#pragma unroll
    for (int j = 0; j < NI; ++j)
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        int row = m0 + wm * WM + i * 16 + gq + ((r & 2) ? 8 : 0);
        int col = n0 + wn * WN + j * 8 + 2 * tq + (r & 1);
        if (row < M && col < N) {
          T* dst = Cb + (ll)row * ldc + col;
          if constexpr (!CPLX) {
            double v = g.alpha_re * acc_re[i][j][r];
            if (use_beta) v += g.beta_re * (*dst);
            *dst = v;
          } else {
            double cr = acc_re[i][j][r], ci = acc_im[i][j][r];
            zc v = mkz(g.alpha_re * cr - g.alpha_im * ci, g.alpha_re * ci + g.alpha_im * cr);
            if (use_beta) {
              zc o = *dst;
              v.re += g.beta_re * o.re - g.beta_im * o.im;
              v.im += g.beta_re * o.im + g.beta_im * o.re;
            }
            *dst = v;
          }
        }
      }
}

// Host-side description of one (possibly batched) GEMM.
template <typename T>
struct Gemm {
  bool ta = false, tb = false, ca = false;
  int M = 0, N = 0, K = 0;
  const T* A = nullptr;
  ll lda = 0, sA1 = 0, sA2 = 0;
  const T* B = nullptr;
  ll ldb = 0, sB1 = 0, sB2 = 0;
  T* C = nullptr;
  ll ldc = 0, sC1 = 0, sC2 = 0;
  int nb1 = 1, nb2 = 1;
  T alpha = ST<T>::one(), beta = ST<T>::zero();
  const int* skip = nullptr;
  int splitk = 1;     // >1: K is split over CTAs, partials go to ws, then summed into C
  T* ws = nullptr;    // splitk * M * N scratch (single, non-batched GEMMs only)
};

template <typename T>
void launch_gemm(const Gemm<T>& d, cudaStream_t st);

}  // namespace dmrg2
