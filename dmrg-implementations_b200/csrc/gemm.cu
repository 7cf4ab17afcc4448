// Host launcher and instantiations of the DMMA GEMM.
#include "gemm.cuh"

namespace dmrg2 {

long long& launch_counter() {
  static long long c = 0;
  return c;
}

template <typename T, bool TA, bool TB, bool CA>
static void launch_impl(const Gemm<T>& d, cudaStream_t st) {
  using G = GemmTile<T>;
  using S = GemmSmem<T, TA, TB>;
  static bool attr_set = false;  // per instantiation; set once per process
  if (!attr_set) {
    DMRG2_CUDA(cudaFuncSetAttribute(gemm_kernel<T, TA, TB, CA>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::BYTES));
    attr_set = true;
  }
  GemmArgs a;
  a.M = d.M; a.N = d.N; a.K = d.K;
  a.A = d.A; a.lda = d.lda; a.sA1 = d.sA1; a.sA2 = d.sA2;
  a.B = d.B; a.ldb = d.ldb; a.sB1 = d.sB1; a.sB2 = d.sB2;
  a.C = d.C; a.ldc = d.ldc; a.sC1 = d.sC1; a.sC2 = d.sC2;
  a.nb2 = d.nb2;
  a.alpha_re = ST<T>::re(d.alpha); a.alpha_im = ST<T>::im(d.alpha);
  a.beta_re = ST<T>::re(d.beta); a.beta_im = ST<T>::im(d.beta);
  a.skip = d.skip;
  dim3 grid(ceil_div(d.N, G::BN), ceil_div(d.M, G::BM), d.nb1 * d.nb2);
  gemm_kernel<T, TA, TB, CA><<<grid, G::THREADS, S::BYTES, st>>>(a);
  DMRG2_CHECK_LAUNCH();
}

template <typename T>
void launch_gemm(const Gemm<T>& d, cudaStream_t st) {
  if (d.M <= 0 || d.N <= 0 || d.nb1 * d.nb2 <= 0) return;
  if (d.nb1 * d.nb2 > 65535) throw std::runtime_error("gemm: batch count exceeds 65535");
  if (ceil_div(d.M, GemmTile<T>::BM) > 65535) throw std::runtime_error("gemm: M too large");
  const bool ca = ST<T>::cplx && d.ca;
  if (!d.ta && !d.tb && !ca) return launch_impl<T, false, false, false>(d, st);
  if (!d.ta && d.tb && !ca) return launch_impl<T, false, true, false>(d, st);
  if (d.ta && !d.tb && !ca) return launch_impl<T, true, false, false>(d, st);
  if (d.ta && d.tb && !ca) return launch_impl<T, true, true, false>(d, st);
  if constexpr (ST<T>::cplx) {
    if (!d.ta && !d.tb) return launch_impl<T, false, false, true>(d, st);
    if (!d.ta && d.tb) return launch_impl<T, false, true, true>(d, st);
    if (d.ta && !d.tb) return launch_impl<T, true, false, true>(d, st);
    return launch_impl<T, true, true, true>(d, st);
  }
}

template void launch_gemm<double>(const Gemm<double>&, cudaStream_t);
template void launch_gemm<zc>(const Gemm<zc>&, cudaStream_t);

}  // namespace dmrg2
