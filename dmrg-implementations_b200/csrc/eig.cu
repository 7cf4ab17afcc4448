// Dense Hermitian eigen-decomposition for the theta truncation.
//
// The reference truncates theta with a full SVD (rocsolver gesvdj/gesvd,
// gpu-rocm/dmrg2-gpu/src/dmrg2_gpu_impl.h:1167-1202). Here the truncation uses
// the reduced density matrix of the side that becomes isometric (G = theta
// theta^H for a left move, theta^H theta for a right move): its dominant
// eigenvectors ARE the kept singular vectors, its eigenvalues the squared
// singular values, and both factors of the split come out without dividing
// by a singular value (left move: A_i = U_k, A_{i+1} = U_k^H theta).
//
// Pipeline (textbook methods, written for sm_100a):
//   1. hetrd_cluster: Householder reduction G = Q T Q^H to real symmetric
//      tridiagonal form (Golub & Van Loan, Alg. 8.3.1) by ONE thread-block
//      cluster of up to 16 CTAs, rows distributed cyclically over the CTAs.
//      Real G up to order 512 keeps the trailing matrix in registers and does
//      each column in one register pass (1b, 1c below), exchanging p by bulk
//      copies into the peers' shared memory; complex or larger G keeps it in
//      shared memory (or L2) and pulls p through distributed shared memory
//      after one cluster barrier per column.
//   2. tridiag_bisect: the K largest eigenvalues of T by Sturm-count
//      multisection, one CTA per eigenvalue, 64 points per round.
//   3. tridiag_invit: eigenvectors of T by inverse iteration with partial
//      pivoting, one thread per eigenvector, seeded random starts, factors and
//      iterate in shared memory.
//   4. group_mgs: classical Gram-Schmidt with re-orthogonalisation inside
//      groups of (numerically) degenerate eigenvalues (SU(2) multiplets, the
//      tail near the noise floor), then a Newton-Schulz polar step on the whole
//      block (GEMMs) restores orthogonality to ~eps.
//   5. apply_q: eigenvectors of G = Q z, each CTA applying all reflectors in
//      compact-WY blocks to its own slab of columns (columns are independent).
#include <cooperative_groups.h>

#include <cstdlib>

#include "kernels.cuh"

namespace cg = cooperative_groups;

namespace dmrg2 {

static constexpr int HT_THREADS = 512;

__device__ inline double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <typename T>
__device__ inline T warp_sum_t(T v);
template <>
__device__ inline double warp_sum_t<double>(double v) { return warp_sum_d(v); }
template <>
__device__ inline zc warp_sum_t<zc>(zc v) { return mkz(warp_sum_d(v.re), warp_sum_d(v.im)); }

// block-wide sum of a T value (all threads receive the result)
template <typename T>
__device__ T block_sum_t(T v, T* sh) {
  v = warp_sum_t<T>(v);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  if (w == 0) {
    T r = (l < nw) ? sh[l] : ST<T>::zero();
    r = warp_sum_t<T>(r);
    if (l == 0) sh[32] = r;
  }
  __syncthreads();
  T r = sh[32];
  __syncthreads();
  return r;
}

// ----------------------------------------------------------------------------
// 1. Householder tridiagonalisation by one thread-block cluster
//    G: n x n Hermitian, row-major (ld). On exit row k of G holds the reflector
//    v_k in columns k+1..n-1 (v_k[k+1] = 1). Row r is owned by CTA r % C; with
//    SROWS the owned rows live in shared memory for the whole reduction.
//    One cluster barrier per column: every CTA writes its slice of p = tau G v
//    and of column k+1 into its OWN shared memory, the cluster synchronises
//    once, and every thread pulls the entries it needs from the owning CTA
//    (remote stores drained by a release barrier cost several times more on
//    sm_100a than one pull phase). Each CTA then forms s = p^H v, w, its rank-2
//    update and the next column locally (identically in every CTA).
// ----------------------------------------------------------------------------
template <typename T, bool SROWS>
__global__ void __launch_bounds__(HT_THREADS)
    hetrd_cluster_kernel(T* __restrict__ G, int n, ll ld, double* __restrict__ dg,
                         double* __restrict__ eg, T* __restrict__ tau) {
  cg::cluster_group cluster = cg::this_cluster();
  const int C = (int)cluster.num_blocks();
  const int rank = (int)cluster.block_rank();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* x = reinterpret_cast<T*>(smem_raw);  // current column k
  T* v = x + n;                           // Householder vector
  T* w = v + n;                           // w (full, local)
  T* pf = w + n;                          // p, all rows (pulled)
  T* cf = pf + n;                         // column k+1 before step k, all rows (pulled)
  T* po0 = cf + n;                        // own entries of p / column k+1, two parity buffers
  T* po1 = po0 + n;
  T* co0 = po1 + n;
  T* co1 = co0 + n;
  T* red = co1 + n;                       // [34] reduction scratch
  T* rows = red + 34;                     // own rows (SROWS): [ceil(n/C)][n]
  __shared__ T sh_tau, sh_alpha2;
  __shared__ double sh_beta;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = blockDim.x >> 5;
  auto own_row = [&](int r) -> T* {
    if (SROWS) return rows + (ll)(r / C) * n;
    return G + (ll)r * ld;
  };
  if (SROWS) {
    for (int q = warp; q * C + rank < n; q += nwarp) {
      const T* src = G + (ll)(q * C + rank) * ld;
      T* dst = rows + (ll)q * n;
      for (int j = lane; j < n; j += 32) dst[j] = src[j];
    }
  }
  double* xnp = reinterpret_cast<double*>(red + 17);  // per-warp partial |x[k+2:]|^2 (16 slots)
  {
    double part = 0.0;
    for (int r = tid; r < n; r += blockDim.x) {
      x[r] = ST<T>::conj(G[r]);  // column 0 = conj(row 0)
      if (r >= 2) part += ST<T>::abs2(x[r]);
    }
    part = warp_sum_d(part);
    if (lane == 0) xnp[warp] = part;
  }
  __syncthreads();
  cluster.sync();  // all CTAs loaded before any rank 0 reflector store to global row 0

  for (int k = 0; k < n - 1; ++k) {
    const int par = k & 1;
    T* po = par ? po1 : po0;
    T* co = par ? co1 : co0;
    const int r0 = k + 1 + ((rank - (k + 1)) % C + C) % C;  // first own row >= k+1
    // (a) reflector of x[k+1..n-1] (identical in every CTA), computed by warp 0:
    //     H^H x = beta e_1, v = [1, x[k+2:] * sc], tau = (beta - alpha) / beta
    if (warp == 0) {
      double xn2 = (lane < nwarp) ? xnp[lane] : 0.0;
      xn2 = warp_sum_d(xn2);
      if (lane == 0) {
        T alpha = x[k + 1];
        double ar = ST<T>::re(alpha), ai = ST<T>::im(alpha);
        if (xn2 == 0.0 && ai == 0.0) {
          sh_tau = ST<T>::zero();
          sh_beta = ar;
          sh_alpha2 = ST<T>::zero();  // scale of v[k+2:] (zero vector)
        } else {
          const double beta = -copysign(sqrt(ar * ar + ai * ai + xn2), ar);
          const double ib = 1.0 / beta;
          sh_tau = ST<T>::make((beta - ar) * ib, -ai * ib);
          sh_beta = beta;
          const double dr = ar - beta, iden = 1.0 / (dr * dr + ai * ai);
          sh_alpha2 = ST<T>::make(dr * iden, -ai * iden);  // 1 / (alpha - beta)
        }
        if (rank == 0) {
          dg[k] = ST<T>::re(x[k]);
          eg[k] = sh_beta;
          tau[k] = sh_tau;
        }
      }
    }
    __syncthreads();
    const T tk = sh_tau;
    const T sc = sh_alpha2;
    // (b) p = tau * G v on own rows (v applied on the fly) and G[r][k+1] (column
    //     k+1 before this step's update), into this CTA's own exchange buffers
    for (int r = r0 + warp * C; r < n; r += nwarp * C) {
      const T* row = own_row(r);
      T a0 = ST<T>::zero(), a1 = ST<T>::zero(), a2 = ST<T>::zero(), a3 = ST<T>::zero();
      int j = k + 2 + lane;
      for (; j + 96 < n; j += 128) {  // four independent chains hide load + FMA latency
        a0 = a0 + ST<T>::mul(row[j], x[j]);
        a1 = a1 + ST<T>::mul(row[j + 32], x[j + 32]);
        a2 = a2 + ST<T>::mul(row[j + 64], x[j + 64]);
        a3 = a3 + ST<T>::mul(row[j + 96], x[j + 96]);
      }
      for (; j < n; j += 32) a0 = a0 + ST<T>::mul(row[j], x[j]);
      T acc = warp_sum_t<T>((a0 + a1) + (a2 + a3));
      const T col = row[k + 1];
      if (lane == 0) {
        po[r] = ST<T>::mul(tk, col + ST<T>::mul(sc, acc));
        co[r] = col;
      }
    }
    cluster.sync();  // the only inter-CTA barrier of the step
    // (c) pull p and column k+1; v, s = p^H v, w = p - 1/2 tau s v (thread-private r's)
    {
      T sp = ST<T>::zero();
      for (int r = k + 1 + tid; r < n; r += blockDim.x) {
        const int owner = r % C;
        const T pr = cluster.map_shared_rank(po, owner)[r];
        cf[r] = cluster.map_shared_rank(co, owner)[r];
        pf[r] = pr;
        const T vr = (r == k + 1) ? ST<T>::one() : ST<T>::mul(x[r], sc);
        v[r] = vr;
        sp = sp + ST<T>::cmul(pr, vr);
      }
      sp = warp_sum_t<T>(sp);
      if (lane == 0) red[warp] = sp;
      __syncthreads();
      T s = ST<T>::zero();
      for (int q = 0; q < nwarp; ++q) s = s + red[q];
      const T a2 = ST<T>::scale(-0.5, ST<T>::mul(tk, s));
      for (int r = k + 1 + tid; r < n; r += blockDim.x) w[r] = pf[r] + ST<T>::mul(a2, v[r]);
      __syncthreads();
    }
    // (d) rank-2 update of own rows: G -= v w^H + w v^H
    for (int r = r0 + warp * C; r < n; r += nwarp * C) {
      T* row = own_row(r);
      const T vr = v[r], wr = w[r];
#pragma unroll 4
      for (int j = k + 1 + lane; j < n; j += 32)
        row[j] = row[j] - ST<T>::mul(vr, ST<T>::conj(w[j])) - ST<T>::mul(wr, ST<T>::conj(v[j]));
    }
    // (e) next column = column k+1 before this step - rank-2 correction (with the norm
    //     partials of the next reflector); (f) reflector row k
    {
      const T wk = ST<T>::conj(w[k + 1]), vk = ST<T>::conj(v[k + 1]);
      double part = 0.0;
      for (int r = k + 1 + tid; r < n; r += blockDim.x) {
        const T xr = cf[r] - ST<T>::mul(v[r], wk) - ST<T>::mul(w[r], vk);
        x[r] = xr;
        if (r >= k + 3) part += ST<T>::abs2(xr);
      }
      part = warp_sum_d(part);
      if (lane == 0) xnp[warp] = part;
      if (rank == 0)
        for (int j = k + 1 + tid; j < n; j += blockDim.x) G[(ll)k * ld + j] = v[j];
    }
    __syncthreads();
  }
  if (rank == 0 && tid == 0) {
    dg[n - 1] = ST<T>::re(x[n - 1]);
    eg[n - 1] = 0.0;
  }
  cluster.sync();  // peers may still write into this CTA's shared memory
}

// ----------------------------------------------------------------------------
// 1b. Real symmetric G of order n <= 512 with the trailing matrix held in
//     registers. Row r belongs to CTA r % C (local row q = r / C) and, inside
//     it, to warp q % 16 (slot q / 16 < RW); lane l holds the column pairs
//     j = 2l + 64u + {0, 1} (NT columns), so the fused pass reads its vectors
//     with 16-byte shared loads. Each warp forms v, w and the next column
//     x' = column k+1 - (v w^T + w v^T)[:, k+1], applies the rank-2 update to its
//     rows and, in the same pass, accumulates the next step's symv
//     sum_j G'[r][j] x'[j] (the reflector of x' only scales it, and every warp
//     derives that reflector itself from x'). The reflector scalars cost one
//     division (house_real1).
// ----------------------------------------------------------------------------
__device__ inline void house_real1(double alpha, double xn2, double& tk, double& sc, double& beta) {
  if (xn2 == 0.0) {
    tk = 0.0;
    sc = 0.0;
    beta = alpha;
    return;
  }
  beta = -copysign(sqrt(alpha * alpha + xn2), alpha);
  const double dr = alpha - beta;  // |dr| >= sqrt(xn2) > 0
  const double r = 1.0 / (beta * dr);
  tk = -dr * dr * r;  // (beta - alpha) / beta
  sc = beta * r;      // 1 / (alpha - beta)
}

// ----------------------------------------------------------------------------
// 1c. The register-resident reduction with a push exchange and a split step.
//     Exchange: instead of a cluster barrier followed by remote loads, every CTA
//     writes one block per step into its own slot of its inbox, [(p'_r, column
//     (k+2)_r) of its rows][its warps' partials of s'], and copies that block
//     into the same slot of every peer's inbox with cp.async.bulk (shared::cta to
//     shared::cluster, one copy per peer), which counts the bytes on the receiver's
//     mbarrier; a CTA starts step k once its barrier has seen every peer's block
//     of step k. Two parity inboxes (and barriers) carry consecutive steps. A
//     slot is rewritten two steps after it was read, and its writer can only get
//     there after receiving the reader's next block, which the reader sends after
//     its last read (behind a CTA barrier; the copy's complete_tx releases at
//     cluster scope, the wait acquires), so no further barrier is needed.
//     Step: (a) one thread per column forms v_j, w_j and the next column x'_j
//     (and the reflector row); after a CTA barrier (b) every warp derives the
//     next reflector from the shared norm partials and (c) applies the rank-2
//     update to its rows with the next symv in the same register pass.
//     Waits are bounded: a CTA that gives up marks the whole cluster failed and
//     the result is poisoned (d[0] = NaN) instead of hanging. A failed cluster
//     drains before it exits: once every CTA has left its loop (so no further
//     copy is issued), each publishes the last step it sent, and each receiver
//     waits for exactly the blocks that were sent to it and not yet consumed
//     (the bytes of peers that never sent are completed on its own barrier).
//     A sender is at most one step ahead of any receiver, so at most one phase
//     per barrier is outstanding. Only then does the final cluster barrier let
//     the CTAs exit, so no bulk copy can land in a CTA that has left.
// ----------------------------------------------------------------------------
static constexpr int HP_SPIN = 1 << 20;  // polls of one barrier phase before giving up

__device__ inline uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ inline uint32_t cluster_addr(uint32_t a, int cta) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(cta));
  return r;
}
__device__ inline void bar_expect(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
// counts bytes that will never arrive as arrived (drain of a failed cluster)
__device__ inline void bar_complete(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.complete_tx.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
// bounded wait for the phase of the given parity, without the failure shortcut
__device__ inline bool bar_wait_drain(uint32_t bar, uint32_t parity) {
  for (int it = 0; it < HP_SPIN; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}
// true once the phase of the given parity has completed, false after HP_SPIN polls
// or when the cluster has been marked failed
__device__ inline bool bar_wait(uint32_t bar, uint32_t parity, const volatile int* fail) {
  for (int it = 0; it < HP_SPIN; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    if (ok) return true;
    if (*fail) return false;
  }
  return false;
}

template <int NT, int RW, int C>
__global__ void __launch_bounds__(HT_THREADS, 1)
    hetrd_push_kernel(double* __restrict__ G, int n, ll ld, double* __restrict__ dg,
                      double* __restrict__ eg, double* __restrict__ tau) {
  static_assert((C & (C - 1)) == 0 && C <= 32, "cluster size: power of two <= 32");
  static_assert(NT % 2 == 0, "column slots come in pairs");
  cg::cluster_group cluster = cg::this_cluster();
  constexpr int NW = HT_THREADS / 32;
  constexpr int lgC = (C >= 32) ? 5 : (C >= 16) ? 4 : (C >= 8) ? 3 : (C >= 4) ? 2 : (C >= 2) ? 1 : 0;
  constexpr int NP = NT / 2;
  const int rank = (int)cluster.block_rank();
  extern __shared__ __align__(16) double hsm[];
  __shared__ __align__(8) unsigned long long bars[2];
  __shared__ int fail_s;
  __shared__ int peer_sent[C];  // last step each peer sent to this CTA (published after the loop)
  const int n2 = (n + 1) & ~1;
  // inbox of a step: one block per CTA, [Q (p, c) pairs of its rows by local index][NW partials
  // of s]; a CTA writes its own block and bulk-copies it into the same slot of every peer
  constexpr int Q = RW * NW;
  constexpr int BLK = 2 * Q + NW;  // doubles; a multiple of 2 (16-byte blocks)
  double* ib0 = hsm;               // inbox, step parity 0
  double* ib1 = ib0 + C * BLK;     // parity 1
  double* xs0 = ib1 + C * BLK;     // column k (parity buffers, computed locally)
  double* xs1 = xs0 + n2;
  double* vv = xs1 + n2;           // v of this step by column (0 outside the active block)
  double* ww = vv + n2;            // w of this step by column
  double* xa = ww + n2;            // next column where it enters the next symv (j >= k+3), else 0
  __shared__ double nrmw[NW], anext_s, dnext_s;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  auto col = [&](int t) { return 2 * lane + 64 * (t >> 1) + (t & 1); };
  const uint32_t bar0 = smem_u32(&bars[0]), bar1 = smem_u32(&bars[1]);
  // bytes the peers copy in per step: one block each
  auto step_bytes = [&]() { return (uint32_t)(8 * BLK * (C - 1)); };
  // thread d < C, d != rank, copies this CTA's block to CTA d
  uint32_t d_ib0 = 0, d_bar0 = 0;
  if (tid < C) {
    d_ib0 = cluster_addr(smem_u32(ib0 + rank * BLK), tid);
    d_bar0 = cluster_addr(bar0, tid);
  }
  const uint32_t o_ib1 = 8u * C * BLK;  // bytes from ib0 to ib1
  auto send_block = [&](int parity) {   // after a CTA barrier that follows the block's writes
    if (tid < C && tid != rank) {
      const uint32_t src = smem_u32((parity ? ib1 : ib0) + rank * BLK);
      asm volatile(
          "cp.async.bulk.shared::cluster.shared::cta.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
              d_ib0 + (parity ? o_ib1 : 0u)),
          "r"(src), "r"(8u * BLK), "r"(d_bar0 + (parity ? 8u : 0u))
          : "memory");
    }
  };
  volatile int* failv = &fail_s;
  auto give_up = [&]() {
    if (!*failv)
      for (int c = 0; c < C; ++c) {
        const uint32_t a = cluster_addr(smem_u32(&fail_s), c);
        asm volatile("st.shared::cluster.u32 [%0], %1;" ::"r"(a), "r"(1) : "memory");
      }
  };
  if (tid == 0) {
    fail_s = 0;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar0), "r"(1) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar1), "r"(1) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    bar_expect(bar0, step_bytes());                  // step 0 (pushed by the prologue)
    if (n - 2 >= 1) bar_expect(bar1, step_bytes());  // step 1
  }
  // drain bookkeeping (uniform in the CTA; arming is done by thread 0)
  int sent_last = 0;                       // the prologue sends step 0
  int waited = n - 1;                      // steps 0 .. waited-1 were consumed
  int armed_last = (n - 2 >= 1) ? 1 : 0;   // steps 0 .. armed_last have an armed phase

  int rr[RW];
  double g[RW][NT];
#pragma unroll
  for (int i = 0; i < RW; ++i) {
    rr[i] = (warp + NW * i) * C + rank;
#pragma unroll
    for (int t = 0; t < NT; ++t) {
      const int j = col(t);
      g[i][t] = (rr[i] < n && j < n) ? G[(ll)rr[i] * ld + j] : 0.0;
    }
  }
  for (int j = tid; j < n; j += HT_THREADS) xs0[j] = G[j];
  // barriers initialised and armed everywhere, every row loaded (rank 0 overwrites row k
  // from step k on)
  cluster.sync();
  // ---- prologue: column 0 (row 0 by symmetry), its reflector, the first symv, pushed
  double tk, sc, beta;
  {
    double xn2 = 0.0;
    for (int j = 2 + lane; j < n; j += 32) xn2 += xs0[j] * xs0[j];
    xn2 = warp_sum_d(xn2);
    house_real1(xs0[1], xn2, tk, sc, beta);
    if (rank == 0 && tid == 0) {
      dg[0] = xs0[0];
      eg[0] = beta;
      tau[0] = tk;
    }
    double sp = 0.0;
#pragma unroll
    for (int i = 0; i < RW; ++i) {
      const int r = rr[i];
      double acc = 0.0;
#pragma unroll
      for (int t = 0; t < NT; ++t) {
        const int j = col(t);
        if (j >= 2 && j < n) acc += g[i][t] * xs0[j];
      }
      acc = warp_sum_d(acc);
      const double c1 = __shfl_sync(0xffffffffu, g[i][1], 0);  // column 1 sits in lane 0, slot 1
      if (r < n) {
        double p = 0.0;
        if (r >= 1) {
          p = tk * (c1 + sc * acc);
          sp += p * ((r == 1) ? 1.0 : xs0[r] * sc);
        }
        if (lane == 0) *reinterpret_cast<double2*>(ib0 + rank * BLK + 2 * (r >> lgC)) = make_double2(p, c1);
      }
    }
    if (lane == 0) ib0[rank * BLK + 2 * Q + warp] = sp;
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    send_block(0);
  }

  for (int k = 0; k < n - 1; ++k) {
    const int par = k & 1;
    const double* ib = par ? ib1 : ib0;
    double* ibn = par ? ib0 : ib1;
    const double* xs = par ? xs1 : xs0;
    double* xsn = par ? xs0 : xs1;
    const uint32_t bar = par ? bar1 : bar0;
    auto pval = [&](int j) { return ib[(j & (C - 1)) * BLK + 2 * (j >> lgC)]; };
    auto cval = [&](int j) { return ib[(j & (C - 1)) * BLK + 2 * (j >> lgC) + 1]; };
    // (1) every CTA's pushes of step k have landed; a CTA that gave up, or learned
    //     that a peer did, leaves the loop as a whole (step k not consumed)
    const bool got = bar_wait(bar, (uint32_t)((k >> 1) & 1), failv);
    if (!got) give_up();
    // also makes this CTA's own entries and column k (written last step) visible to all
    if (__syncthreads_or(!got || *failv)) {
      waited = k;
      break;
    }
    if (k + 2 <= n - 2) {  // re-arm for step k+2
      if (tid == 0) bar_expect(bar, step_bytes());
      armed_last = k + 2;
    }
    double ssum = 0.0;
    for (int q = lane; q < C * NW; q += 32) ssum += ib[(q / NW) * BLK + 2 * Q + (q % NW)];
    ssum = warp_sum_d(ssum);
    // (2a) one column per thread: v, w and the next column x' = column k+1 after the
    //      rank-2 update, its norm partial and the reflector row (rank 0)
    const double a2 = -0.5 * tk * ssum;
    const double wk1 = pval(k + 1) + a2;  // v[k+1] = 1
    {
      double nr = 0.0;
      for (int j = tid; j < n; j += HT_THREADS) {
        double vj = 0.0, wj = 0.0, xj = 0.0;
        if (j >= k + 1) {
          vj = (j == k + 1) ? 1.0 : xs[j] * sc;
          wj = pval(j) + a2 * vj;
          const double xn = cval(j) - vj * wk1 - wj;
          xsn[j] = xn;
          if (j >= k + 3) {
            xj = xn;
            nr += xn * xn;
          }
          if (j == k + 2) anext_s = xn;
          if (j == k + 1) dnext_s = xn;
          if (rank == 0) G[(ll)k * ld + j] = vj;
        }
        vv[j] = vj;
        ww[j] = wj;
        xa[j] = xj;
      }
      nr = warp_sum_d(nr);
      if (lane == 0) nrmw[warp] = nr;
    }
    __syncthreads();  // v, w, x' and the norm partials visible to every warp
    // (3a) next reflector (every warp derives the same one, in a fixed order)
    double nrm = (lane < NW) ? nrmw[lane] : 0.0;
    nrm = warp_sum_d(nrm);
    const double a_next = anext_s, d_next = dnext_s;
    double tk2 = 0.0, sc2 = 0.0, beta2 = 0.0;
    if (k + 2 <= n - 1) house_real1(a_next, nrm, tk2, sc2, beta2);
    if (rank == 0 && tid == 32) {
      dg[k + 1] = d_next;
      eg[k + 1] = beta2;
      if (k + 1 < n - 1) tau[k + 1] = tk2;
    }
    // (2b) rank-2 update of this warp's rows and the next symv sum_j G'[r][j] x'[j]
    double vr[RW], wr[RW], acc[RW], c2[RW];
    bool act[RW];
#pragma unroll
    for (int i = 0; i < RW; ++i) {
      const int r = rr[i];
      act[i] = (r >= k + 1 && r < n);
      vr[i] = act[i] ? vv[r] : 0.0;
      wr[i] = act[i] ? ww[r] : 0.0;
      acc[i] = 0.0;
      c2[i] = 0.0;
    }
#pragma unroll
    for (int u = 0; u < NP; ++u) {
      const int base = 64 * u;
      if (base + 64 <= k + 1 || base >= n) continue;
      const int j0 = base + 2 * lane;
      if (base >= k + 3 && base + 64 <= n) {
        const double2 v2 = *reinterpret_cast<const double2*>(vv + j0);
        const double2 w2 = *reinterpret_cast<const double2*>(ww + j0);
        const double2 x2 = *reinterpret_cast<const double2*>(xa + j0);
#pragma unroll
        for (int i = 0; i < RW; ++i) {
          if (act[i]) {
            const double g0 = g[i][2 * u] - vr[i] * w2.x - wr[i] * v2.x;
            const double g1 = g[i][2 * u + 1] - vr[i] * w2.y - wr[i] * v2.y;
            g[i][2 * u] = g0;
            g[i][2 * u + 1] = g1;
            acc[i] += g0 * x2.x;
            acc[i] += g1 * x2.y;
          }
        }
      } else {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int j = j0 + h;
          if (j >= k + 1 && j < n) {
            const double vj = vv[j], wj = ww[j], xj = xa[j];
#pragma unroll
            for (int i = 0; i < RW; ++i) {
              if (act[i]) {
                const double gg = g[i][2 * u + h] - vr[i] * wj - wr[i] * vj;
                g[i][2 * u + h] = gg;
                acc[i] += gg * xj;
                if (j == k + 2) c2[i] = gg;
              }
            }
          }
        }
      }
    }
    const bool push = (k + 1 <= n - 2);  // step k+1 exists
    double sp = 0.0;
#pragma unroll
    for (int i = 0; i < RW; ++i) {
      const int r = rr[i];
      const double a = warp_sum_d(acc[i]);
      const double c = __shfl_sync(0xffffffffu, c2[i], ((k + 2) & 63) >> 1);
      if (r < n) {
        double p = 0.0;
        if (r >= k + 2) {
          p = tk2 * (c + sc2 * a);
          sp += p * ((r == k + 2) ? 1.0 : xsn[r] * sc2);
        }
        if (push && lane == 0) *reinterpret_cast<double2*>(ibn + rank * BLK + 2 * (warp + NW * i)) = make_double2(p, c);
      }
    }
    if (push) {
      if (lane == 0) ibn[rank * BLK + 2 * Q + warp] = sp;
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncthreads();  // the block is complete
      send_block(par ^ 1);
      sent_last = k + 1;
    }
    tk = tk2;
    sc = sc2;
  }
  // publish the last step this CTA sent (peers need it only if the cluster failed,
  // which a CTA cannot know yet)
  if (tid < C && tid != rank) {
    const uint32_t a = cluster_addr(smem_u32(&peer_sent[rank]), tid);
    asm volatile("st.shared::cluster.u32 [%0], %1;" ::"r"(a), "r"(sent_last) : "memory");
  }
  // every CTA has left its loop: no further copy is issued, every failure mark and
  // published step is visible
  cluster.sync();
  if (*failv && tid == 0) {
    // wait for the blocks sent to this CTA and not consumed: steps waited and waited+1
    int max_s = -1;
    for (int c = 0; c < C; ++c)
      if (c != rank) max_s = max(max_s, peer_sent[c]);
    for (int st = waited; st <= max_s && st <= waited + 1; ++st) {
      int senders = 0;
      for (int c = 0; c < C; ++c)
        if (c != rank && peer_sent[c] >= st) ++senders;
      const uint32_t expect = (uint32_t)(8 * BLK * senders);
      const uint32_t b = (st & 1) ? bar1 : bar0;
      if (st <= armed_last) {
        if (step_bytes() > expect) bar_complete(b, step_bytes() - expect);
      } else {
        bar_expect(b, expect);
      }
      (void)bar_wait_drain(b, (uint32_t)((st >> 1) & 1));
    }
  }
  cluster.sync();  // no CTA leaves while a copy into it may be in flight
  if (rank == 0 && tid == 0 && *failv) dg[0] = __longlong_as_double(0x7ff8000000000000ll);
}

template <int NT, int RW, int C>
static cudaError_t hetrd_push_launch(double* G, int n, ll ld, double* d, double* e, double* tau,
                                      cudaStream_t s) {
  static std::atomic<unsigned long long> attr_cluster{0};
  func_attr_once(attr_cluster, (const void*)hetrd_push_kernel<NT, RW, C>,
                 cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(C);
  cfg.blockDim = dim3(HT_THREADS);
  const size_t n2 = (size_t)((n + 1) & ~1);
  constexpr size_t NW = HT_THREADS / 32, BLK = 2 * RW * NW + NW;
  cfg.dynamicSmemBytes = sizeof(double) * (5 * n2 + 2 * (size_t)C * BLK);
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, hetrd_push_kernel<NT, RW, C>, G, n, ld, d, e, tau);
}

// register-resident reduction for real G with 32 <= n <= 512; false when the device
// refused the cluster (the caller then takes the shared-memory kernel)
static bool hetrd_reg(double* G, int n, ll ld, double* d, double* e, double* tau, cudaStream_t s) {
  static std::atomic<int> refused{0};
  if (n < 32 || n > 512 || refused.load()) return false;
  cudaError_t err;
  if (n <= 128) err = hetrd_push_launch<4, 1, 8>(G, n, ld, d, e, tau, s);
  else if (n <= 256) err = hetrd_push_launch<8, 1, 16>(G, n, ld, d, e, tau, s);
  else err = hetrd_push_launch<16, 2, 16>(G, n, ld, d, e, tau, s);
  if (err == cudaSuccess) return true;
  if (err == cudaErrorInvalidClusterSize || err == cudaErrorLaunchOutOfResources || err == cudaErrorInvalidValue) {
    (void)cudaGetLastError();
    refused.store(1);
    return false;
  }
  DMRG2_CUDA(err);
  return false;
}

// ----------------------------------------------------------------------------
// 2. K largest eigenvalues of (d, e) by Sturm-count multisection, one CTA per
//    eigenvalue (blockDim+1 points per round)
// ----------------------------------------------------------------------------
// Number of eigenvalues of (d, e) below x: sign changes along the leading principal
// minors P_0 = 1, P_1 = d_0 - x, P_{i+1} = (d_i - x) P_i - e_{i-1}^2 P_{i-1} (Sturm).
// Compared with the ratio form q_i = P_i / P_{i-1} (LDL^T pivots) it needs no
// division. Each step perturbs d_i - x and e_{i-1}^2 by a few ulps relative, the
// same backward error as the ratio form. The pair (P_{i-1}, P_i) is rescaled by an
// exact power of two every four steps to stay in range; an exact zero minor is
// replaced by -2^-60 P_{i-1}, the ratio form's negative tiny pivot. The steps run in
// groups of 8 with the next group's shared loads issued ahead of the current group's
// chain.
__device__ inline int sturm_lt(const double* d, const double* e2, int n, double x) {
  constexpr int G = 8;
  double a = 1.0, b = d[0] - x;
  if (b == 0.0) b = -0x1p-60;
  int c = (b < 0.0);
  const int ng = (n - 1) / G;  // full groups cover steps 1 .. ng G
  double dd[G], ee[G];
  if (ng > 0) {
#pragma unroll
    for (int u = 0; u < G; ++u) {
      dd[u] = d[1 + u];
      ee[u] = e2[u];
    }
  }
  for (int g = 0; g < ng; ++g) {
    double dn[G], en[G];
    const int base = 1 + (g + 1) * G;
#pragma unroll
    for (int u = 0; u < G; ++u) {  // next group (clamped reads past the end are not used)
      const int i = min(base + u, n - 1);
      dn[u] = d[i];
      en[u] = e2[i - 1];
    }
#pragma unroll
    for (int u = 0; u < G; ++u) {
      double nb = fma(dd[u] - x, b, -ee[u] * a);
      if (nb == 0.0) nb = -0x1p-60 * b;
      c += ((nb < 0.0) != (b < 0.0));
      a = b;
      b = nb;
      if (u == 3 || u == 7) {
        const double m = fmax(fabs(a), fabs(b));
        const double f = (m > 0x1p+256) ? 0x1p-256 : (m < 0x1p-256) ? 0x1p+256 : 1.0;
        a *= f;
        b *= f;
      }
    }
#pragma unroll
    for (int u = 0; u < G; ++u) {
      dd[u] = dn[u];
      ee[u] = en[u];
    }
  }
  for (int i = 1 + ng * G; i < n; ++i) {
    double nb = fma(d[i] - x, b, -e2[i - 1] * a);
    if (nb == 0.0) nb = -0x1p-60 * b;
    c += ((nb < 0.0) != (b < 0.0));
    a = b;
    b = nb;
  }
  return c;
}

__global__ void __launch_bounds__(256)
    tridiag_bisect_kernel(const double* __restrict__ dg, const double* __restrict__ eg, int n, int K,
                          double* __restrict__ lam) {
  extern __shared__ double sm[];
  double* d = sm;
  double* e2 = sm + n;
  __shared__ double a_s, b_s, afloor_s, lo_w[32], hi_w[32];
  __shared__ int tmin;
  const int j = blockIdx.x;
  if (j >= K) return;
  // Gershgorin bounds, reduced over the block
  double lo = 1e300, hi = -1e300;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    d[i] = dg[i];
    e2[i] = (i < n - 1) ? eg[i] * eg[i] : 0.0;
    const double r = (i > 0 ? fabs(eg[i - 1]) : 0.0) + (i < n - 1 ? fabs(eg[i]) : 0.0);
    lo = fmin(lo, dg[i] - r);
    hi = fmax(hi, dg[i] + r);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  if ((threadIdx.x & 31) == 0) {
    lo_w[threadIdx.x >> 5] = lo;
    hi_w[threadIdx.x >> 5] = hi;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w2 = 1; w2 < (int)(blockDim.x >> 5); ++w2) {
      lo = fmin(lo, lo_w[w2]);
      hi = fmax(hi, hi_w[w2]);
    }
    double w = fmax(hi - lo, fmax(fabs(hi), 1e-300));
    a_s = lo - 2e-15 * w;
    b_s = hi + 2e-15 * w;
    afloor_s = 2.2e-16 * fmax(fabs(lo), fabs(hi));  // Sturm counts resolve eps*|T| at best
  }
  __syncthreads();
  const int t = n - 1 - j;  // ascending index of the wanted eigenvalue
  const int NT = blockDim.x;
  for (int round = 0; round < 24; ++round) {
    const double a = a_s, b = b_s;
    const double step = (b - a) / (double)(NT + 1);
    const double x = a + step * (threadIdx.x + 1);
    const int c = sturm_lt(d, e2, n, x);
    if (threadIdx.x == 0) tmin = NT;
    __syncthreads();
    if (c >= t + 1) atomicMin(&tmin, (int)threadIdx.x);
    __syncthreads();
    if (threadIdx.x == 0) {
      const int l = tmin;
      if (l == NT) {
        a_s = a + step * NT;
      } else {
        b_s = a + step * (l + 1);
        a_s = a + step * l;
      }
    }
    __syncthreads();
    if (b_s - a_s <= 2.2e-16 * fmax(fabs(a_s), fabs(b_s)) + afloor_s) break;
  }
  if (threadIdx.x == 0) lam[j] = 0.5 * (a_s + b_s);
}

// ----------------------------------------------------------------------------
// 3. inverse iteration for the k kept eigenvalues: one thread per eigenvector,
//    LU factors with partial pivoting and the iterate in shared memory, the
//    recurrences carried in registers. Columns k..K-1 of Z are zeroed.
//    A numerically degenerate cluster (neighbours within 8 eps |T|: SU(2)
//    multiplets, exactly repeated singular values) splits T into nearly
//    decoupled blocks; with its own eigenvalue as shift every member would
//    converge to the block whose eigenvalue happens to lie nearest, i.e. to the
//    same vector. Its members therefore share one shift placed 4 max(width,
//    8 eps |T|) outside the cluster, on the side of the larger gap: every
//    cluster direction is amplified alike (to 25%), the random starts give a
//    well-conditioned basis of the cluster space that the group Gram-Schmidt
//    orthonormalises, and a neighbour at distance gap is damped by
//    (shift distance / gap)^2 over the two iterations. Where either gap is
//    below 1e4 times the shift distance, or where the cluster is wider than the group
//    tolerance (its members would not all share one Gram-Schmidt window), the
//    members keep their own shifts.
// ----------------------------------------------------------------------------
__device__ inline double hash_unit(unsigned long long x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  x ^= x >> 31;
  return (double)(x >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
}

__global__ void tridiag_invit_kernel(const double* __restrict__ dg, const double* __restrict__ eg,
                                     int n, int K, const double* __restrict__ lam,
                                     const SvdOut* __restrict__ tr, double* __restrict__ Z, double gtol_rel) {
  extern __shared__ double dsh[];
  __shared__ double tn_s;
  const int vpb = blockDim.x;  // one vector per thread
  double* d = dsh;
  double* e = dsh + n;
  double* base = dsh + 2 * n;  // [6][n][vpb]: factors, then the iterate
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    d[i] = dg[i];
    e[i] = (i < n - 1) ? eg[i] : 0.0;
  }
  __syncthreads();
  if (threadIdx.x == 0) {  // |T|_inf once per CTA
    double tn = 0.0;
    for (int i = 0; i < n; ++i) tn = fmax(tn, fabs(d[i]) + fabs(i > 0 ? e[i - 1] : 0.0) + fabs(e[i]));
    tn_s = tn;
  }
  __syncthreads();
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= K) return;
  if (j >= tr->k) {
    for (int i = 0; i < n; ++i) Z[(ll)i * K + j] = 0.0;
    return;
  }
  const int t = threadIdx.x;
#define SX(a, i) base[((ll)(a) * n + (i)) * vpb + t]
  // arrays: 0 = 1/u0, 1 = u1, 2 = u2, 3 = multiplier, 4 = swap flag, 5 = iterate
  const double tiny = fmax(tn_s, 1e-300) * 2.2e-16;
  double sft = lam[j];
  {
    const double tight = 8.0 * tiny;
    int first = j, last = j;
    while (first > 0 && lam[first - 1] - lam[first] <= tight) --first;
    while (last + 1 < K && lam[last] - lam[last + 1] <= tight) ++last;
    // the group Gram-Schmidt must see the whole cluster in every member's window: its
    // width stays within the group tolerance
    if (last > first && lam[first] - lam[last] <= gtol_rel * fabs(lam[0])) {
      const double width = lam[first] - lam[last];
      const double shift = 4.0 * fmax(width, tight);
      // eigenvalues past the K computed ones are unknown: no gap below is taken as known
      const double gap_up = (first > 0) ? lam[first - 1] - lam[first] : 1e300;
      const double gap_dn = (last + 1 < K) ? lam[last] - lam[last + 1] : 0.0;
      // only where both gaps keep a neighbour's share below 1e-8 after two iterations (the
      // neighbour on the far side is damped only by shift / (gap + shift) per iteration)
      if (fmin(gap_up, gap_dn) >= 1e4 * shift) sft = (gap_up >= gap_dn) ? lam[first] + shift : lam[last] - shift;
    }
  }
  double c0 = d[0] - sft, c1 = e[0];
  for (int i = 0; i < n - 1; ++i) {
    const double s = e[i];
    const double dn = d[i + 1] - sft;
    const double en = e[i + 1];
    if (fabs(c0) >= fabs(s)) {
      if (fabs(c0) < tiny) c0 = (c0 < 0 ? -tiny : tiny);
      const double r = 1.0 / c0;
      const double m = s * r;
      SX(0, i) = r;
      SX(1, i) = c1;
      SX(2, i) = 0.0;
      SX(3, i) = m;
      SX(4, i) = 0.0;
      c0 = dn - m * c1;
      c1 = en;
    } else {
      const double r = 1.0 / s;
      const double m = c0 * r;
      SX(0, i) = r;
      SX(1, i) = dn;
      SX(2, i) = en;
      SX(3, i) = m;
      SX(4, i) = 1.0;
      c0 = c1 - m * dn;
      c1 = -m * en;
    }
  }
  if (fabs(c0) < tiny) c0 = (c0 < 0 ? -tiny : tiny);
  SX(0, n - 1) = 1.0 / c0;
  SX(1, n - 1) = 0.0;
  SX(2, n - 1) = 0.0;
  // the iterate lives in shared memory next to the factors; column j of Z is written at the end
#define IZ(i) SX(5, i)
  for (int i = 0; i < n; ++i) IZ(i) = hash_unit(((unsigned long long)(j + 1) << 32) ^ (unsigned long long)i);
  for (int it = 0; it < 2; ++it) {
    double y = IZ(0);
    for (int i = 0; i < n - 1; ++i) {
      double yn = IZ(i + 1), yi = y;
      if (SX(4, i) != 0.0) { yi = yn; yn = y; }
      IZ(i) = yi;
      y = yn - SX(3, i) * yi;
    }
    IZ(n - 1) = y;
    double x1 = 0.0, x2 = 0.0, nrm = 0.0;
    for (int i = n - 1; i >= 0; --i) {
      const double xi = (IZ(i) - SX(1, i) * x1 - SX(2, i) * x2) * SX(0, i);
      IZ(i) = xi;
      nrm += xi * xi;
      x2 = x1;
      x1 = xi;
    }
    nrm = sqrt(nrm);
    if (!(nrm > 0.0) || !isfinite(nrm)) {
      for (int i = 0; i < n; ++i) IZ(i) = (i == (n - 1 - j) % n) ? 1.0 : 0.0;
      break;
    }
    const double inv = 1.0 / nrm;
    for (int i = 0; i < n; ++i) IZ(i) *= inv;
  }
  for (int i = 0; i < n; ++i) Z[(ll)i * K + j] = IZ(i);
#undef IZ
#undef SX
}

// ----------------------------------------------------------------------------
// 4. Gram-Schmidt inside groups of nearly equal eigenvalues. A group is a run
//    of consecutive eigenvalues (descending) whose neighbours differ by at most
//    gtol; each CTA takes candidate group starts j = blockIdx.x + m * gridDim.x
//    and skips those that do not start a group of two or more.
//    Vector q of a group is orthogonalised against its window: the earlier
//    members p with lam_p - lam_q <= gtol. Pairs further apart than gtol are
//    treated like pairs in different groups (their overlap is bounded by the
//    eigenvector perturbation bound eps |T| / gap and removed by the
//    Newton-Schulz step that follows). In the dense tail of a DMRG spectrum
//    the runs chain over tens of eigenvalues while each window holds a few.
//    Classical Gram-Schmidt with one re-orthogonalisation pass (CGS2, "twice
//    is enough": Giraud, Langou and Rozloznik 2005): per vector the dots with
//    the window members are formed at once, one warp per member, then
//    subtracted in one pass. The window members live in a ring of R vectors
//    in shared memory (column-contiguous); the next vector is fetched into
//    registers while the current one is processed. A group whose largest
//    window does not fit the ring takes the whole-group path on global memory.
// ----------------------------------------------------------------------------
static constexpr int GS_THREADS = 512;
static constexpr int GS_SMEM = 200 * 1024;
static constexpr int GS_RP = 4;  // rows per thread of the ring path (n <= GS_RP * GS_THREADS)

__global__ void __launch_bounds__(GS_THREADS, 1)
    group_cgs_kernel(double* __restrict__ Z, int n, int K, const double* __restrict__ lam,
                     const SvdOut* __restrict__ tr, double gtol_rel) {
  extern __shared__ __align__(16) double gsm[];
  __shared__ double red[GS_THREADS / 32 + 1];
  __shared__ int wmax_s;
  constexpr int NW = GS_THREADS / 32;
  const int kk = tr->k;
  const double gtol = gtol_rel * fmax(fabs(lam[0]), 1e-300);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const size_t cap = GS_SMEM / sizeof(double);
  for (int j = blockIdx.x; j < kk; j += gridDim.x) {  // candidate group starts, grid-strided
    if (j > 0 && fabs(lam[j - 1] - lam[j]) <= gtol) continue;  // not a group start
    int end = j + 1;
    while (end < kk && fabs(lam[end - 1] - lam[end]) <= gtol) ++end;
    const int g = end - j;
    if (g < 2) continue;
    // shared layout: lam of the group [g], window starts [g] (ints in a double slot each),
    // window coefficients [g], the ring [R][n]
    double* lam_s = gsm;
    int* lo_s = reinterpret_cast<int*>(gsm + g);
    double* cfs = gsm + 2 * (size_t)g;
    double* ring = gsm + 3 * (size_t)g;
    const int R = (int)min((size_t)g, (cap - 3 * (size_t)g) / (size_t)n);
    if (tid == 0) wmax_s = 0;
    for (int q = tid; q < g; q += GS_THREADS) lam_s[q] = lam[j + q];
    __syncthreads();
    for (int q = tid; q < g; q += GS_THREADS) {
      int lo = q;
      while (lo > 0 && lam_s[lo - 1] - lam_s[q] <= gtol) --lo;
      lo_s[q] = lo;
      atomicMax(&wmax_s, q - lo);
    }
    __syncthreads();
    if (wmax_s <= R - 1 && n <= GS_RP * GS_THREADS) {
      // ---- windowed ring path (vectors are fetched two ahead into registers)
      double cur[GS_RP], pre1[GS_RP], pre2[GS_RP];
#pragma unroll
      for (int m = 0; m < GS_RP; ++m) {
        const int i = tid + m * GS_THREADS;
        pre1[m] = (i < n) ? Z[(ll)i * K + j] : 0.0;
        pre2[m] = (i < n) ? Z[(ll)i * K + j + 1] : 0.0;  // g >= 2
      }
      for (int q = 0; q < g; ++q) {
        const int sq_slot = q % R;
        double* vq = ring + (size_t)sq_slot * n;
#pragma unroll
        for (int m = 0; m < GS_RP; ++m) {
          const int i = tid + m * GS_THREADS;
          cur[m] = pre1[m];
          pre1[m] = pre2[m];
          if (i < n) vq[i] = cur[m];
        }
        if (q + 2 < g)
#pragma unroll
          for (int m = 0; m < GS_RP; ++m) {
            const int i = tid + m * GS_THREADS;
            if (i < n) pre2[m] = Z[(ll)i * K + j + q + 2];
          }
        const int lo = lo_s[q], w = q - lo;
        const int lo_slot = lo % R;
        __syncthreads();  // vector q staged; the previous vector final
        double sq = 0.0;
        for (int pass = 0; pass < 2 && w > 0; ++pass) {
          for (int p = warp; p < w; p += NW) {
            const int slot = lo_slot + p < R ? lo_slot + p : lo_slot + p - R;
            const double* vp = ring + (size_t)slot * n;
            double sum = 0.0;
            for (int i = lane; i < n; i += 32) sum += vp[i] * vq[i];
            sum = warp_sum_d(sum);
            if (lane == 0) cfs[p] = sum;
          }
          __syncthreads();  // coefficients ready
          // a second pass only when the first removed more than half of the (unit) norm:
          // |v'|^2 = 1 - sum cf^2 < 1/2 (Daniel, Gragg, Kaufman and Stewart 1976)
          double c2 = 0.0;
          for (int p = 0; p < w; ++p) c2 += cfs[p] * cfs[p];
          const bool again = (pass == 0) && (c2 > 0.5);
          sq = 0.0;
#pragma unroll
          for (int m = 0; m < GS_RP; ++m) {
            const int i = tid + m * GS_THREADS;
            if (i < n) {
              double v = cur[m];
              int slot = lo_slot;
              for (int p = 0; p < w; ++p) {
                v -= cfs[p] * ring[(size_t)slot * n + i];
                slot = (slot + 1 == R) ? 0 : slot + 1;
              }
              cur[m] = v;
              vq[i] = v;
              sq += v * v;
            }
          }
          if (!again) break;
          __syncthreads();  // vq updated before the second pass's dots
        }
        if (w == 0) {
#pragma unroll
          for (int m = 0; m < GS_RP; ++m) sq += cur[m] * cur[m];
        }
        sq = warp_sum_d(sq);
        if (lane == 0) red[warp] = sq;
        __syncthreads();  // partial norms ready (and every read of the window done)
        double tot = 0.0;
#pragma unroll
        for (int w2 = 0; w2 < NW; ++w2) tot += red[w2];
        const double inv = tot > 0.0 ? 1.0 / sqrt(tot) : 0.0;
#pragma unroll
        for (int m = 0; m < GS_RP; ++m) {
          const int i = tid + m * GS_THREADS;
          if (i < n) {
            const double v = cur[m] * inv;
            vq[i] = v;
            Z[(ll)i * K + j + q] = v;
          }
        }
      }
      __syncthreads();  // the shared area is reused by this CTA's next group
      continue;
    }
    // ---- whole-group path (a window larger than the ring): every earlier member, on
    //      global memory
    double* cf = gsm + 3 * (size_t)g;  // coefficients, 4 g <= cap always (g <= K <= n)
    auto at = [&](int q, int i) -> double& { return Z[(ll)i * K + j + q]; };
    for (int q = 0; q < g; ++q) {
      for (int pass = 0; pass < 2 && q > 0; ++pass) {
        for (int p = warp; p < q; p += NW) {
          double sum = 0.0;
          for (int i = lane; i < n; i += 32) sum += at(p, i) * at(q, i);
          sum = warp_sum_d(sum);
          if (lane == 0) cf[p] = sum;
        }
        __syncthreads();
        for (int i = tid; i < n; i += GS_THREADS) {
          double v = at(q, i);
          for (int p = 0; p < q; ++p) v -= cf[p] * at(p, i);
          at(q, i) = v;
        }
        __syncthreads();
      }
      double sq = 0.0;
      for (int i = tid; i < n; i += GS_THREADS) {
        const double v = at(q, i);
        sq += v * v;
      }
      sq = warp_sum_d(sq);
      if (lane == 0) red[warp] = sq;
      __syncthreads();
      if (warp == 0) {
        double t = lane < NW ? red[lane] : 0.0;
        t = warp_sum_d(t);
        if (lane == 0) red[NW] = t;
      }
      __syncthreads();
      const double tot = red[NW];
      const double inv = tot > 0.0 ? 1.0 / sqrt(tot) : 0.0;
      for (int i = tid; i < n; i += GS_THREADS) at(q, i) *= inv;
      __syncthreads();
    }
  }
}

// ----------------------------------------------------------------------------
// 5. Zg = Q Z with Q = H_0 H_1 ... H_{n-2}; reflector i in row i of R (cols i+1..).
//    Reflectors are grouped in blocks of nb in compact WY form
//    H_lo ... H_hi = I - V T V^H (Schreiber & Van Loan), T upper triangular
//    (wy_build); apply_q then costs three barriers per block. Each CTA owns
//    a slab of 2, 4 or 8 columns of Z (columns are independent).
// ----------------------------------------------------------------------------
static constexpr int AQ_COLS = 8;
static constexpr int AQ_MAXNB = 16;
static constexpr int AQ_THREADS = 512;

template <typename T>
__global__ void wy_build_kernel(const T* __restrict__ R, ll ld, const T* __restrict__ tau, int n,
                                int nb, T* __restrict__ Tb) {
  __shared__ T gram[AQ_MAXNB][AQ_MAXNB];
  const int blk = blockIdx.x;
  const int lo = blk * nb;
  const int hi = min(n - 2, lo + nb - 1);
  const int cnt = hi - lo + 1;
  for (int e = threadIdx.x; e < AQ_MAXNB * AQ_MAXNB; e += blockDim.x) {
    const int p = e / AQ_MAXNB, q = e % AQ_MAXNB;
    T acc = ST<T>::zero();
    if (p < cnt && q < cnt && p < q) {
      const int ip = lo + p, iq = lo + q;
      for (int r = iq + 1; r < n; ++r) acc = acc + ST<T>::cmul(R[(ll)ip * ld + r], R[(ll)iq * ld + r]);
    }
    gram[p][q] = acc;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    T* Tm = Tb + (ll)blk * AQ_MAXNB * AQ_MAXNB;
    for (int e = 0; e < AQ_MAXNB * AQ_MAXNB; ++e) Tm[e] = ST<T>::zero();
    for (int q = 0; q < cnt; ++q) {
      const T tq = tau[lo + q];
      Tm[q * AQ_MAXNB + q] = tq;
      for (int p = 0; p < q; ++p) {  // T(p, q) = -tau_q sum_{l=p}^{q-1} T(p, l) (v_l^H v_q)
        T acc = ST<T>::zero();
        for (int l = p; l < q; ++l) acc = acc + ST<T>::mul(Tm[p * AQ_MAXNB + l], gram[l][q]);
        Tm[p * AQ_MAXNB + q] = ST<T>::scale(-1.0, ST<T>::mul(tq, acc));
      }
    }
  }
}

// one element into shared memory through the async copy path
__device__ inline void cp_async_elem(double* dst, const double* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
               : "memory");
}
__device__ inline void cp_async_elem(zc* dst, const zc* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
               : "memory");
}

// Reflector blocks are double-buffered: block blk - 1 is copied from L2 with
// cp.async while block blk is applied. Entries left of each reflector's first
// element are masked in the arithmetic instead of zeroed in the copy.
template <typename T, int COLS>
__global__ void __launch_bounds__(AQ_THREADS, 1)
    apply_q_kernel(const T* __restrict__ R, ll ld, const T* __restrict__ Tb, int n, int nb,
                   const double* __restrict__ Z, int K, const SvdOut* __restrict__ tr,
                   T* __restrict__ Zg) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* zs = reinterpret_cast<T*>(smem_raw);  // [COLS][n] (rows contiguous: conflict-free)
  T* vbuf0 = zs + (ll)n * COLS;         // [nb][n], two buffers
  T* vbuf1 = vbuf0 + (ll)nb * n;
  __shared__ T W[AQ_MAXNB][COLS];
  __shared__ T W2[AQ_MAXNB][COLS];
  const int c0 = blockIdx.x * COLS;
  const int kk = min(tr->k, K);
  if (c0 >= kk) return;
  const int nc = min(COLS, kk - c0);
  for (int e = threadIdx.x; e < n * COLS; e += blockDim.x) {
    int i = e / COLS, c = e % COLS;
    zs[(ll)c * n + i] = (c < nc) ? ST<T>::make(Z[(ll)i * K + c0 + c], 0.0) : ST<T>::zero();
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nblk = (n - 1 + nb - 1) / nb;
  auto prefetch = [&](int blk, T* dst) {
    const int lo = blk * nb;
    const int cnt = min(n - 2, lo + nb - 1) - lo + 1;
    for (int e = threadIdx.x; e < cnt * n; e += blockDim.x) {
      const int q = e / n, r = e % n;
      cp_async_elem(dst + (ll)q * n + r, R + (ll)(lo + q) * ld + r);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  prefetch(nblk - 1, vbuf0);
  for (int blk = nblk - 1; blk >= 0; --blk) {
    const int lo = blk * nb;
    const int hi = min(n - 2, lo + nb - 1);
    const int cnt = hi - lo + 1;
    T* vb = ((nblk - 1 - blk) & 1) ? vbuf1 : vbuf0;
    T* vnext = ((nblk - 1 - blk) & 1) ? vbuf0 : vbuf1;
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncthreads();  // block blk has landed; the previous block's buffer is free again
    if (blk > 0) prefetch(blk - 1, vnext);
    // W = V^H Z  (warp q -> row q of W)
    for (int q = warp; q < cnt; q += AQ_THREADS / 32) {
      T acc[COLS];
#pragma unroll
      for (int c = 0; c < COLS; ++c) acc[c] = ST<T>::zero();
      const T* vq = vb + (ll)q * n;
      for (int r = lo + q + 1 + lane; r < n; r += 32) {
        const T vr = ST<T>::conj(vq[r]);
#pragma unroll
        for (int c = 0; c < COLS; ++c) acc[c] = acc[c] + ST<T>::mul(vr, zs[(ll)c * n + r]);
      }
#pragma unroll
      for (int c = 0; c < COLS; ++c) {
        T sm2 = warp_sum_t<T>(acc[c]);
        if (lane == 0) W[q][c] = sm2;
      }
    }
    __syncthreads();
    // W2 = T W  (T upper triangular)
    if (threadIdx.x < cnt * COLS) {
      const int q = threadIdx.x / COLS, c = threadIdx.x % COLS;
      const T* Tm = Tb + (ll)blk * AQ_MAXNB * AQ_MAXNB;
      T acc = ST<T>::zero();
      for (int p = q; p < cnt; ++p) acc = acc + ST<T>::mul(Tm[q * AQ_MAXNB + p], W[p][c]);
      W2[q][c] = acc;
    }
    __syncthreads();
    // Z -= V W2
    for (int r = lo + 1 + threadIdx.x; r < n; r += blockDim.x) {
      T acc[COLS];
#pragma unroll
      for (int c = 0; c < COLS; ++c) acc[c] = ST<T>::zero();
      for (int q = 0; q < cnt; ++q) {
        const T vr = (r > lo + q) ? vb[(ll)q * n + r] : ST<T>::zero();
#pragma unroll
        for (int c = 0; c < COLS; ++c) acc[c] = acc[c] + ST<T>::mul(vr, W2[q][c]);
      }
#pragma unroll
      for (int c = 0; c < COLS; ++c) zs[(ll)c * n + r] = zs[(ll)c * n + r] - acc[c];
    }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < n * COLS; e += blockDim.x) {
    int i = e / COLS, c = e % COLS;
    if (c < nc) Zg[(ll)i * K + c0 + c] = zs[(ll)c * n + i];
  }
}

// max |S - I| over the leading k x k block; sets out->ns_done once below tol.
// Partial maxima per CTA, the last CTA to arrive decides.
__global__ void ns_check_kernel(const double* __restrict__ S, int K, SvdOut* out, double tol,
                                double* part, unsigned* counter) {
  __shared__ double mx[256];
  __shared__ int last;
  const int k = min(out->k, K);
  double m = 0.0;
  if (!out->ns_done)
    for (ll e = (ll)blockIdx.x * blockDim.x + threadIdx.x; e < (ll)k * k; e += (ll)gridDim.x * blockDim.x) {
      const int a = (int)(e / k), b = (int)(e % k);
      m = fmax(m, fabs(S[(ll)a * K + b] - (a == b ? 1.0 : 0.0)));
    }
  mx[threadIdx.x] = m;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) mx[threadIdx.x] = fmax(mx[threadIdx.x], mx[threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[blockIdx.x] = mx[0];
    __threadfence();
    last = (atomicAdd(counter, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    double t = 0.0;
    for (int b = 0; b < (int)gridDim.x; ++b) t = fmax(t, part[b]);
    if (!out->ns_done && t < tol) out->ns_done = 1;
    *counter = 0u;
  }
}

// ----------------------------------------------------------------------------
// truncation decision from the eigenvalues (one CTA)
// ----------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
    eig_truncate_kernel(const double* __restrict__ dg, const double* __restrict__ lam, int n, int K,
                        int chi_max, double cutoff, int relative, double floor_rel, SvdOut* out) {
  __shared__ double sh[33];
  __shared__ int kmin;
  const int tid = threadIdx.x;
  double tr = 0.0;
  for (int i = tid; i < n; i += blockDim.x) tr += dg[i];
  tr = block_sum_t<double>(tr, sh);
  const double l0 = fmax(lam[0], 0.0);
  // density-matrix rounding floor: eigenvalues below ~16 eps lambda_max are noise
  // (floor_rel; a caller may raise it where the vectors of a noise cluster did not
  // come out orthonormal)
  const double noise = floor_rel * l0;
  double thr = relative ? (cutoff * cutoff) * l0 : cutoff * cutoff;
  thr = fmax(thr, noise);
  const int kcap = chi_max < K ? chi_max : K;
  if (tid == 0) kmin = kcap;
  __syncthreads();
  for (int r = tid; r < kcap; r += blockDim.x)
    if (!(lam[r] > thr)) atomicMin(&kmin, r);  // the first eigenvalue at or below the threshold
  __syncthreads();
  const int k = max(kmin, 1);
  double kept = 0.0, nz = 0.0;
  for (int r = tid; r < K; r += blockDim.x) {
    if (r < k) kept += fmax(lam[r], 0.0);
    if (lam[r] > noise) nz += 1.0;
  }
  kept = block_sum_t<double>(kept, sh);
  nz = block_sum_t<double>(nz, sh);
  if (tid == 0) {
    out->k = k;
    out->nonzero = (int)nz;
    out->trunc_err = fmax(tr - kept, 0.0);
    out->sigma_max = sqrt(l0);
    out->sigma_max2 = l0;
    out->fro2 = tr;
    out->jacobi_sweeps = 0;
    out->jacobi_err = 0;
    out->ns_done = 0;
  }
}

// ----------------------------------------------------------------------------
template <typename T, bool SROWS>
static void hetrd_launch(T* G, int n, ll ld, double* d, double* e, T* tau, int C, size_t smem,
                         cudaStream_t s, cudaError_t* err) {
  static std::atomic<unsigned long long> attr_cluster{0}, attr_smem{0};
  func_attr_once(attr_cluster, (const void*)hetrd_cluster_kernel<T, SROWS>,
                 cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  set_smem_attr_once(attr_smem, (const void*)hetrd_cluster_kernel<T, SROWS>, 220 * 1024);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(C);
  cfg.blockDim = dim3(HT_THREADS);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  *err = cudaLaunchKernelEx(&cfg, hetrd_cluster_kernel<T, SROWS>, G, n, ld, d, e, tau);
}

template <typename T>
void hetrd_cluster(T* G, int n, ll ld, double* d, double* e, T* tau, cudaStream_t s) {
  if constexpr (!ST<T>::cplx) {
    if (hetrd_reg((double*)G, n, ld, d, e, (double*)tau, s)) {
      ++launch_counter();
      return;
    }
  }
  const size_t base = sizeof(T) * ((size_t)9 * n + 34);
  if (base > 200 * 1024) throw std::runtime_error("hetrd: matrix order too large for one cluster");
  int C = 16;
  if (n < 64) C = 1;
  else if (n < 128) C = 4;
  else if (n < 256) C = 8;
  static std::atomic<int> c_cap{16};  // largest cluster size the device accepted
  if (C > c_cap.load()) C = c_cap.load();
  for (;;) {
    const size_t rows = sizeof(T) * (size_t)((n + C - 1) / C) * n;
    const bool srows = base + rows <= 220 * 1024;
    cudaError_t err;
    if (srows) hetrd_launch<T, true>(G, n, ld, d, e, tau, C, base + rows, s, &err);
    else hetrd_launch<T, false>(G, n, ld, d, e, tau, C, base, s, &err);
    if (err == cudaSuccess) break;
    if (C > 1 && (err == cudaErrorInvalidClusterSize || err == cudaErrorLaunchOutOfResources ||
                  err == cudaErrorInvalidValue)) {
      (void)cudaGetLastError();
      C /= 2;
      c_cap.store(C);
      continue;
    }
    DMRG2_CUDA(err);
  }
  DMRG2_CHECK_LAUNCH();
}

void tridiag_eigvals(const double* d, const double* e, int n, int K, double* lam, cudaStream_t s) {
  // 64 points per round (6 bits), about 9 rounds: the counts are issue-bound, and fewer points
  // per round cost fewer counts in all
  tridiag_bisect_kernel<<<K, 64, sizeof(double) * 2 * n, s>>>(d, e, n, K, lam);
  DMRG2_CHECK_LAUNCH();
}

void tridiag_eigvecs(const double* d, const double* e, int n, int K, const double* lam,
                     const SvdOut* tr, double* Z, double* scratch, double gtol_rel, cudaStream_t s) {
  (void)scratch;
  static std::atomic<unsigned long long> attr{0};
  set_smem_attr_once(attr, (const void*)tridiag_invit_kernel, 220 * 1024);
  const size_t per = sizeof(double) * 6 * (size_t)n;
  int vpb = (int)std::min<size_t>(8, (220 * 1024 - sizeof(double) * 2 * (size_t)n) / per);
  if (vpb < 1) throw std::runtime_error("inverse iteration: matrix order too large");
  const size_t smem = sizeof(double) * 2 * (size_t)n + per * vpb;
  tridiag_invit_kernel<<<(K + vpb - 1) / vpb, vpb, smem, s>>>(d, e, n, K, lam, tr, Z, gtol_rel);
  DMRG2_CHECK_LAUNCH();
}

void group_mgs(double* Z, int n, int K, const double* lam, const SvdOut* tr, double gtol_rel,
               cudaStream_t s) {
  if ((size_t)K * sizeof(double) > (size_t)GS_SMEM) throw std::runtime_error("group_mgs: order too large");
  static std::atomic<unsigned long long> attr{0};
  set_smem_attr_once(attr, (const void*)group_cgs_kernel, GS_SMEM);
  group_cgs_kernel<<<std::max(1, std::min(K, 148)), GS_THREADS, GS_SMEM, s>>>(Z, n, K, lam, tr, gtol_rel);
  DMRG2_CHECK_LAUNCH();
}

template <typename T>
__global__ void copy_real_cols_kernel(const double* Z, ll tot, T* Zg) {
  for (ll t = (ll)blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += (ll)gridDim.x * blockDim.x)
    Zg[t] = ST<T>::make(Z[t], 0.0);
}
template <typename T>
static void copy_real_cols(const double* Z, int n, int K, T* Zg, cudaStream_t s) {
  copy_real_cols_kernel<T><<<1, 256, 0, s>>>(Z, (ll)n * K, Zg);
  DMRG2_CHECK_LAUNCH();
}

// slab width (columns per CTA) and reflector block size of the back-transform
template <typename T>
static void aq_plan(int n, int K, int& cols, int& nb) {
  const size_t cap = 220 * 1024 / sizeof(T);
  const size_t rows = cap / (size_t)n;  // rows of n elements that fit: the column slab + two reflector blocks
  // the narrowest slab that still fills one wave of CTAs (2 columns: K = 256 -> 128 CTAs)
  cols = (K + 1) / 2 <= 160 ? 2 : (K + 3) / 4 <= 160 ? 4 : AQ_COLS;
  nb = (int)std::min<size_t>(AQ_MAXNB, rows > (size_t)cols ? (rows - cols) / 2 : 0);
  if (nb < 1) throw std::runtime_error("apply_q: matrix order too large");
}

template <typename T>
void wy_build(const T* R, ll ld, const T* tau, int n, int K, T* Tb, cudaStream_t s) {
  if (n < 2) return;
  int cols, nb;
  aq_plan<T>(n, K, cols, nb);
  const int nblk = (n - 1 + nb - 1) / nb;
  wy_build_kernel<T><<<nblk, 256, 0, s>>>(R, ld, tau, n, nb, Tb);
  DMRG2_CHECK_LAUNCH();
}

template <typename T>
void apply_q(const T* R, ll ld, const T* tau, int n, const double* Z, int K, const SvdOut* tr, T* Zg,
             T* Tb, cudaStream_t s, bool wy_ready) {
  if (n < 2) {  // Q = I
    copy_real_cols(Z, n, K, Zg, s);
    return;
  }
  int cols, nb;
  aq_plan<T>(n, K, cols, nb);
  const size_t smem = sizeof(T) * (size_t)n * (cols + 2 * nb);
  if (!wy_ready) wy_build<T>(R, ld, tau, n, K, Tb, s);
  auto launch = [&](auto kern, int c, std::atomic<unsigned long long>& attr) {
    set_smem_attr_once(attr, (const void*)kern, 220 * 1024);
    kern<<<(K + c - 1) / c, AQ_THREADS, smem, s>>>(R, ld, Tb, n, nb, Z, K, tr, Zg);
  };
  static std::atomic<unsigned long long> attr2{0}, attr4{0}, attr8{0};
  if (cols == 2) launch(apply_q_kernel<T, 2>, 2, attr2);
  else if (cols == 4) launch(apply_q_kernel<T, 4>, 4, attr4);
  else launch(apply_q_kernel<T, AQ_COLS>, AQ_COLS, attr8);
  DMRG2_CHECK_LAUNCH();
}

void ns_check(const double* S, int K, SvdOut* out, double tol, double* part, unsigned* counter,
              cudaStream_t s) {
  ns_check_kernel<<<32, 256, 0, s>>>(S, K, out, tol, part, counter);
  DMRG2_CHECK_LAUNCH();
}

void eig_truncate(const double* d, const double* lam, int n, int K, int chi_max, double cutoff,
                  bool relative, SvdOut* out, cudaStream_t s, double floor_rel) {
  eig_truncate_kernel<<<1, 256, 0, s>>>(d, lam, n, K, chi_max, cutoff, relative ? 1 : 0, floor_rel, out);
  DMRG2_CHECK_LAUNCH();
}

// out[r][j] = conj(in[r][j]) (j < k), in has leading dimension ldi
template <typename T>
__global__ void copy_cols_conj_kernel(const T* __restrict__ in, ll ldi, int rows, int k, T* __restrict__ out) {
  const ll tot = (ll)rows * k;
  for (ll t = (ll)blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += (ll)gridDim.x * blockDim.x) {
    ll r = t / k;
    int j = (int)(t % k);
    out[t] = ST<T>::conj(in[r * ldi + j]);
  }
}
// out[j][r] = conj(in[r][j]) (j < k)
template <typename T>
__global__ void transpose_conj_kernel(const T* __restrict__ in, ll ldi, int rows, int k, T* __restrict__ out) {
  const ll tot = (ll)rows * k;
  for (ll t = (ll)blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += (ll)gridDim.x * blockDim.x) {
    int j = (int)(t / rows);
    ll r = t % rows;
    out[t] = ST<T>::conj(in[r * ldi + j]);
  }
}
static int eg_grid(ll tot) {
  ll g = (tot + 255) / 256;
  if (g > 148 * 8) g = 148 * 8;
  return (int)(g < 1 ? 1 : g);
}
template <typename T>
void copy_cols_conj(const T* in, ll ldi, int rows, int k, T* out, cudaStream_t s) {
  copy_cols_conj_kernel<T><<<eg_grid((ll)rows * k), 256, 0, s>>>(in, ldi, rows, k, out);
  DMRG2_CHECK_LAUNCH();
}
template <typename T>
void transpose_conj(const T* in, ll ldi, int rows, int k, T* out, cudaStream_t s) {
  transpose_conj_kernel<T><<<eg_grid((ll)rows * k), 256, 0, s>>>(in, ldi, rows, k, out);
  DMRG2_CHECK_LAUNCH();
}
template void copy_cols_conj<double>(const double*, ll, int, int, double*, cudaStream_t);
template void copy_cols_conj<zc>(const zc*, ll, int, int, zc*, cudaStream_t);
template void transpose_conj<double>(const double*, ll, int, int, double*, cudaStream_t);
template void transpose_conj<zc>(const zc*, ll, int, int, zc*, cudaStream_t);

template void hetrd_cluster<double>(double*, int, ll, double*, double*, double*, cudaStream_t);
template void hetrd_cluster<zc>(zc*, int, ll, double*, double*, zc*, cudaStream_t);
template void apply_q<double>(const double*, ll, const double*, int, const double*, int,
                              const SvdOut*, double*, double*, cudaStream_t, bool);
template void apply_q<zc>(const zc*, ll, const zc*, int, const double*, int, const SvdOut*, zc*, zc*,
                          cudaStream_t, bool);
template void wy_build<double>(const double*, ll, const double*, int, int, double*, cudaStream_t);
template void wy_build<zc>(const zc*, ll, const zc*, int, int, zc*, cudaStream_t);

}  // namespace dmrg2
