// Split-BF16 GEMM on tcgen05 tensor cores (see umma.cuh).
//
// Kernel structure (one 128 x 128 output tile per CTA, 4 warps):
//   * the operands are first split into three BF16 pieces each by a separate
//     kernel, written K-major and zero-padded to the tile grid (M, N to 128,
//     K to 64), so the GEMM kernel has no edge cases;
//   * per K tile of 64, every thread copies 16-byte chunks of the six pieces
//     into shared memory with cp.async, in the canonical no-swizzle K-major
//     UMMA layout: 8-row x 16-byte core matrices, consecutive along K at a
//     leading-byte offset of 128 B and consecutive along M/N at a stride-byte
//     offset of 1024 B;
//   * one thread issues the tcgen05.mma instructions (M = 128, N = 128,
//     K = 16, BF16 inputs, FP32 accumulator in tensor memory): six piece
//     products per K step, four K steps per tile, then tcgen05.commit arrives
//     on an mbarrier that every thread waits on (bounded) before the shared
//     tile is refilled;
//   * the epilogue reads the accumulator with tcgen05.ld (warp w owns TMEM
//     lanes 32w..32w+31 = tile rows) and writes alpha acc + beta C in FP64.
// Shared memory is written through the generic proxy and read by the tensor
// core through the async proxy: fence.proxy.async.shared::cta orders the two.
#include <cuda_bf16.h>

#include "umma.cuh"

namespace dmrg2 {

void SplitScratch::reserve(size_t b, cudaStream_t s) {
  if (!err) {
    err = (int*)dev_alloc(sizeof(int));
    DMRG2_CUDA(cudaMemset(err, 0, sizeof(int)));
  }
  if (b <= bytes) return;
  if (p) {
    DMRG2_CUDA(cudaStreamSynchronize(s));  // kernels queued on s may still read the old pieces
    dev_free(p);
  }
  p = nullptr;
  bytes = 0;
  p = dev_alloc(b);
  bytes = b;
}

void SplitScratch::release() {
  if (p) dev_free(p);
  if (err) dev_free(err);
  p = nullptr;
  err = nullptr;
  bytes = 0;
}

namespace {

constexpr int UM_BM = 128, UM_BN = 128, UM_BK = 64;
constexpr int UM_THREADS = 128;
constexpr int UM_PIECE_BYTES = UM_BM * UM_BK * 2;  // one 128 x 64 BF16 tile (16 KB)
constexpr int UM_SMEM = 6 * UM_PIECE_BYTES;        // three A pieces + three B pieces
constexpr int UM_SPIN = 1 << 22;                   // mbarrier polls before giving up
constexpr int UM_SPIN_TEST = 1 << 10;              // the same under the unsignalled-wait test hook

ll round_up(ll x, ll m) { return (x + m - 1) / m * m; }

// ---------------------------------------------------------------- descriptors
// instruction descriptor, kind::f16: FP32 accumulator (bits 4-5 = 1), BF16 A and B
// (bits 7-9, 10-12 = 1), both K-major (bits 15, 16 = 0), N >> 3 at bits 17-22,
// M >> 4 at bits 24-28
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// shared-memory matrix descriptor, no swizzle: start address >> 4 at bits 0-13,
// leading-byte offset >> 4 at bits 16-29, stride-byte offset >> 4 at bits 32-45,
// descriptor version 1 at bits 46-47, base offset 0, layout type 0 (no swizzle)
__device__ inline uint64_t umma_sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ inline uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ inline bool mbar_wait(uint32_t bar, uint32_t parity, int* err, int spin) {
  for (int it = 0; it < spin; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  if (err) atomicExch(err, 1);  // err: the device error flag, or null (no report)
  return false;
}

// ---------------------------------------------------------------- split kernels
// piece q of x: q = 0: bf16(x); 1: bf16(x - p0); 2: bf16(x - p0 - p1)
__device__ inline void split3(double x, __nv_bfloat16& a, __nv_bfloat16& b, __nv_bfloat16& c) {
  a = __double2bfloat16(x);
  const double r1 = x - (double)__bfloat162float(a);
  b = __double2bfloat16(r1);
  const double r2 = r1 - (double)__bfloat162float(b);
  c = __double2bfloat16(r2);
}

template <typename T>
__device__ inline T load_op(const T* X, ll ld, int trans, int r, int c) {
  // element (r, c) of op(X): N/C read X[r][c]... T/C read X[c][r]; C/conj conjugate
  const T v = (trans == 1 || trans == 2) ? X[(ll)c * ld + r] : X[(ll)r * ld + c];
  return (trans == 2 || trans == 3) ? ST<T>::conj(v) : v;
}

// A' (Mp x Kp, K-major): real: op(A); complex: [[Ar, -Ai], [Ai, Ar]]
template <typename T>
__global__ void split_a_kernel(const T* __restrict__ A, ll lda, ll sA, int ta, int M, int K, int Mp, int Kp,
                               int nb, __nv_bfloat16* __restrict__ out, const int* skip) {
  if (skip && *((volatile const int*)skip)) return;
  const ll per = (ll)Mp * Kp, tot = per * nb;
  const ll piece = tot;  // elements per piece array (all batches)
  for (ll t = (ll)blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += (ll)gridDim.x * blockDim.x) {
    const int b = (int)(t / per);
    const ll rem = t - (ll)b * per;
    const int i = (int)(rem / Kp), k = (int)(rem % Kp);
    double x = 0.0;
    if (!ST<T>::cplx) {
      if (i < M && k < K) x = ST<T>::re(load_op(A + (ll)b * sA, lda, ta, i, k));
    } else if (i < 2 * M && k < 2 * K) {
      const int r = i >= M, c = k >= K;
      const T z = load_op(A + (ll)b * sA, lda, ta, i - r * M, k - c * K);
      x = (r == c) ? ST<T>::re(z) : (r ? ST<T>::im(z) : -ST<T>::im(z));
    }
    split3(x, out[t], out[piece + t], out[2 * piece + t]);
  }
}

// B' (Np x Kp, K-major, row n holds column n of op(B)): real: op(B)^T; complex: [Br; Bi]^T
template <typename T>
__global__ void split_b_kernel(const T* __restrict__ B, ll ldb, ll sB, int tb, int K, int N, int Np, int Kp,
                               int nb, __nv_bfloat16* __restrict__ out, const int* skip) {
  if (skip && *((volatile const int*)skip)) return;
  const ll per = (ll)Np * Kp, tot = per * nb;
  const ll piece = tot;
  for (ll t = (ll)blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += (ll)gridDim.x * blockDim.x) {
    const int b = (int)(t / per);
    const ll rem = t - (ll)b * per;
    const int n = (int)(rem / Kp), k = (int)(rem % Kp);
    double x = 0.0;
    const int Kr = ST<T>::cplx ? 2 * K : K;
    if (n < N && k < Kr) {
      const int c = k >= K;
      const T z = load_op(B + (ll)b * sB, ldb, tb, k - c * K, n);
      x = c ? ST<T>::im(z) : ST<T>::re(z);
    }
    split3(x, out[t], out[piece + t], out[2 * piece + t]);
  }
}

// ---------------------------------------------------------------- GEMM kernel
template <typename T>
__global__ void __launch_bounds__(UM_THREADS, 1)
    umma_bf16x3_kernel(const __nv_bfloat16* __restrict__ Ap, const __nv_bfloat16* __restrict__ Bp, int Mp,
                       int Np, int Kp, int nbA, int nbB, int M, int N, double alpha, double beta,
                       T* __restrict__ C, ll ldc, ll sC, int* __restrict__ err, const int* skip,
                       int unsignalled) {
  if (skip && *((volatile const int*)skip)) return;  // uniform: before any TMEM allocation
  extern __shared__ __align__(1024) unsigned char usm[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tmem_slot;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int b = blockIdx.z;
  const int m0 = blockIdx.y * UM_BM, n0 = blockIdx.x * UM_BN;
  const ll pieceA = (ll)nbA * Mp * Kp, pieceB = (ll)nbB * Np * Kp;
  const __nv_bfloat16* A0 = Ap + (ll)(nbA > 1 ? b : 0) * Mp * Kp + (ll)m0 * Kp;
  const __nv_bfloat16* B0 = Bp + (ll)(nbB > 1 ? b : 0) * Np * Kp + (ll)n0 * Kp;
  const uint32_t sbase = smem_u32(usm);
  const uint32_t sbar = smem_u32(&bar);

  if (warp == 0) {
    const uint32_t slot = smem_u32(&tmem_slot);
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot), "r"(128));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(sbar), "r"(1) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;

  const int nk = Kp / UM_BK;
  const uint32_t idesc = umma_idesc_bf16(UM_BM, UM_BN);
  const int spin = unsignalled ? UM_SPIN_TEST : UM_SPIN;
  bool ok = true;
  int kt_issued = -1;  // last K tile whose MMAs and commit were issued (thread 0)
  int kt = 0;
  for (; kt < nk && ok; ++kt) {
    // six pieces x 128 rows x 8 chunks of 16 bytes
    for (int q = tid; q < 6 * UM_BM * 8; q += UM_THREADS) {
      const int piece = q / (UM_BM * 8);
      const int rc = q - piece * (UM_BM * 8);
      const int r = rc >> 3, c = rc & 7;
      const __nv_bfloat16* src = piece < 3 ? A0 + piece * pieceA + (ll)r * Kp + (ll)kt * UM_BK + c * 8
                                           : B0 + (piece - 3) * pieceB + (ll)r * Kp + (ll)kt * UM_BK + c * 8;
      const uint32_t dst = sbase + piece * UM_PIECE_BYTES + (r >> 3) * 1024 + c * 128 + (r & 7) * 16;
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0 && !unsignalled) {
      kt_issued = kt;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      constexpr int pa[6] = {0, 0, 1, 1, 0, 2};
      constexpr int pb[6] = {0, 1, 0, 1, 2, 0};
#pragma unroll
      for (int ks = 0; ks < UM_BK / 16; ++ks) {
#pragma unroll
        for (int pp = 0; pp < 6; ++pp) {
          const uint64_t da = umma_sdesc(sbase + pa[pp] * UM_PIECE_BYTES + ks * 256, 128, 1024);
          const uint64_t db = umma_sdesc(sbase + (3 + pb[pp]) * UM_PIECE_BYTES + ks * 256, 128, 1024);
          const uint32_t acc = (kt > 0 || ks > 0 || pp > 0) ? 1u : 0u;
          asm volatile(
              "{\n\t.reg .pred p;\n\t"
              "setp.ne.b32 p, %4, 0;\n\t"
              "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
              ::"r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc));
        }
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(sbar)
                   : "memory");
    }
    // uniform in the CTA (a barrier also orders the tile's consumption before its refill)
    ok = __syncthreads_and(mbar_wait(sbar, (uint32_t)(kt & 1), err, spin)) != 0;
  }
  if (!ok) {
    // timed out: let the MMAs of the last issued tile finish (bounded) before the
    // accumulator is released; the result is not read
    if (tid == 0 && kt_issued == kt - 1) (void)mbar_wait(sbar, (uint32_t)(kt_issued & 1), nullptr, UM_SPIN);
    __syncthreads();
  }
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  // epilogue: warp w reads TMEM lanes 32w + lane (tile row), 128 FP32 columns
  const int row = m0 + warp * 32 + lane;
  const int Mr = ST<T>::cplx ? 2 * M : M;
  const bool live = ok && row < Mr;
  const int part = ST<T>::cplx ? (row >= M) : 0;
  const int m = row - part * M;
  double* Cd = reinterpret_cast<double*>(C + (ll)b * sC);
  const int ew = ST<T>::cplx ? 2 : 1;
#pragma unroll 1
  for (int col = 0; col < UM_BN && ok; col += 8) {
    uint32_t v[8];
    const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)col;
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    if (live) {
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int n = n0 + col + j;
        if (n < N) {
          double* dst = Cd + ((ll)m * ldc + n) * ew + part;
          const double acc = (double)__uint_as_float(v[j]);
          *dst = (beta != 0.0) ? alpha * acc + beta * *dst : alpha * acc;
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128));
  }
}

}  // namespace

template <typename T>
void gemm_bf16x3(int ta, int tb, int M, int N, int K, T alpha, const T* A, ll lda, ll sA, const T* B,
                 ll ldb, ll sB, T beta, T* C, ll ldc, ll sC, int nbatch, SplitScratch& ws, cudaStream_t s,
                 const int* skip) {
  if (M < 1 || N < 1 || K < 1 || nbatch < 1) return;
  if (ST<T>::im(alpha) != 0.0 || ST<T>::im(beta) != 0.0)
    throw std::invalid_argument("gemm_bf16x3: alpha and beta must be real");
  const bool cplx = ST<T>::cplx;
  const ll Mp = round_up(cplx ? 2LL * M : M, UM_BM), Np = round_up(N, UM_BN);
  const ll Kp = round_up(cplx ? 2LL * K : K, UM_BK);
  if (Mp / UM_BM > 65535 || nbatch > 65535) throw std::invalid_argument("gemm_bf16x3: grid too large");
  const int nbA = sA == 0 ? 1 : nbatch, nbB = sB == 0 ? 1 : nbatch;  // shared operands split once
  const size_t need = sizeof(__nv_bfloat16) * 3 * ((size_t)nbA * Mp + (size_t)nbB * Np) * (size_t)Kp;
  ws.reserve(need, s);
  __nv_bfloat16* Ap = (__nv_bfloat16*)ws.p;
  __nv_bfloat16* Bp = Ap + 3 * (size_t)nbA * Mp * Kp;
  const int grid = 148 * 8;
  split_a_kernel<T><<<grid, 256, 0, s>>>(A, lda, sA, ta, M, K, (int)Mp, (int)Kp, nbA, Ap, skip);
  DMRG2_CHECK_LAUNCH();
  split_b_kernel<T><<<grid, 256, 0, s>>>(B, ldb, sB, tb, K, N, (int)Np, (int)Kp, nbB, Bp, skip);
  DMRG2_CHECK_LAUNCH();
  static std::atomic<unsigned long long> attr{0};
  set_smem_attr_once(attr, (const void*)umma_bf16x3_kernel<T>, UM_SMEM);
  dim3 g((unsigned)(Np / UM_BN), (unsigned)(Mp / UM_BM), (unsigned)nbatch);
  umma_bf16x3_kernel<T><<<g, UM_THREADS, UM_SMEM, s>>>(Ap, Bp, (int)Mp, (int)Np, (int)Kp, nbA, nbB, M, N,
                                                      ST<T>::re(alpha), ST<T>::re(beta), C, ldc, sC, ws.err,
                                                      skip, test_unsignalled_waits() ? 1 : 0);
  DMRG2_CHECK_LAUNCH();
}

template void gemm_bf16x3<double>(int, int, int, int, int, double, const double*, ll, ll, const double*, ll,
                                  ll, double, double*, ll, ll, int, SplitScratch&, cudaStream_t, const int*);
template void gemm_bf16x3<zc>(int, int, int, int, int, zc, const zc*, ll, ll, const zc*, ll, ll, zc, zc*, ll,
                              ll, int, SplitScratch&, cudaStream_t, const int*);

}  // namespace dmrg2
