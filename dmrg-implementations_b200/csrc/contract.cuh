// Tensor-network contractions of the two-site sweep, expressed as strided
// batched DMMA GEMMs (see gemm.cuh).
//
// Layouts (row-major, fastest index last):
//   MPS site  A[a][s][b]          (chi_l, d, chi_r)
//   theta     T[a][s][r][e]       (chi_l, d, d, chi_r)
//   left env  L[a][w][c]          (bra, mpo, ket)
//   right env R[f][n][e]          (bra, mpo, ket)
//   MPO       W[wl][wr][s][t]     (mpo_l, mpo_r, s_in, s_out); applied operator O[t][s]
#pragma once

#include <vector>

#include "common.cuh"
#include "gemm.cuh"
#include "umma.cuh"

namespace dmrg2 {

// H_eff matvec (reference: apply_heff_two_site, dmrg2_gpu_impl.h:607-780)
//   step 1: X[a][w][s][r][e] = sum_c L[a][w][c] theta[c][s][r][e]      (Dl batches)
//   step 2: Y[a][p][q][n][e] = sum_{w,s,r} WWt[(p,q,n)][(w,s,r)] X[a][w][s][r][e]  (cL batches)
//   step 3: out[a][p][q][f]  = sum_{n,e} Y[a][p][q][n][e] R[f][n][e]  (one GEMM, K = Dr*cR)
//
// wsp, when given, is the nonzero form of WWt (wwt_sparse_block below): step 2 then sums
// only the nonzero entries, in the same column order, so the result is the same.
template <typename T>
void heff_apply(const T* Lenv, const T* Renv, const T* WWt, const T* in, T* out, T* X, T* Y, int cL,
                int cR, int d, int Dl, int Dr, const int* skip, cudaStream_t s, const T* wsp = nullptr);

// The fused two-site MPO of a bond as the engine stores it, one block: the dense Kout x Kin
// matrix WWt, then its nonzeros row by row (Kout x Kin slots for values), then, as ints, the
// Kout + 1 row starts and the Kout x Kin slots for column indices (ascending in each row).
// The fused Heisenberg MPO (D = 5, d = 2) has 30 nonzeros of 400.
inline ll wwt_block_elems(int Kin, int Kout, size_t elem_bytes) {
  const ll kk = (ll)Kin * Kout;
  return 2 * kk + (((ll)Kout + 1 + kk) * (ll)sizeof(int) + (ll)elem_bytes - 1) / (ll)elem_bytes;
}
// appends the nonzero form to a dense WWt (Kout x Kin) in place; returns the nonzero count
template <typename T>
int wwt_sparse_block(std::vector<T>& w, int Kin, int Kout);

// The same matvec in the precision form: steps 1 and 3 as split-BF16 GEMMs on the
// tcgen05 tensor cores (FP32 accumulation), step 2 in FP64.
template <typename T>
void heff_apply_split(const T* Lenv, const T* Renv, const T* WWt, const T* in, T* out, T* X, T* Y, int cL,
                      int cR, int d, int Dl, int Dr, SplitScratch& ws, const int* skip, cudaStream_t s);

// Single-site H_eff (reference: apply_heff, gpu-rocm/dmrg-gpu/src/dmrg_gpu_impl.h):
//   out[a][t][f] = sum L[a][w][c] A[c][s][e] W[w][w'][s][t] R[f][w'][e], with
//   WmixL[(t,w')][(w,s)] = W[w][w'][s][t] (the left-environment mixing matrix)
template <typename T>
void heff1_apply(const T* Lenv, const T* Renv, const T* WmixL, const T* in, T* out, T* X, T* Y, int cL, int cR,
                 int d, int Dl, int Dr, const int* skip, cudaStream_t s);
double heff1_flops(int cL, int cR, int d, int Dl, int Dr, bool cplx);

// algorithmic real flops of one heff_apply
double heff_flops(int cL, int cR, int d, int Dl, int Dr, bool cplx);
double env_flops(int chi_in, int chi_out, int d, int Dl, int Dr, bool cplx);

// Left environment (reference: update_left_env, dmrg2_gpu_impl.h:787-860)
//   L'[a'][w'][c'] = sum conj(A[a][t][a']) L[a][w][c] W[w][w'][s][t] A[c][s][c']
template <typename T>
void env_left(const T* Lenv, const T* A, const T* WmixL, T* Lnew, T* X, T* Y, int cL, int cO, int d,
              int Dl, int Dr, cudaStream_t s);

// Right environment (reference: update_right_env, dmrg2_gpu_impl.h:867-934)
//   R'[a'][w'][c'] = sum conj(B[a'][t][a]) R[a][w][c] W[w'][w][s][t] B[c'][s][c]
template <typename T>
void env_right(const T* Renv, const T* B, const T* WmixR, T* Rnew, T* X, T* Y, int cI, int cO,
               int d, int Dl, int Dr, cudaStream_t s);

// theta = A_i . A_{i+1} (reference: form_theta_two_site, dmrg2_gpu_impl.h:583-600)
template <typename T>
// theta = A B; ws (ws_elems elements, optional) lets a GEMM with few output tiles split K
void theta_form(const T* A, const T* B, T* theta, int cL, int cM, int cR, int d, cudaStream_t s, T* ws = nullptr,
                ll ws_elems = 0);

// host-side MPO preprocessing (reference: set_mpo / precompute_fused_mpo, dmrg2_gpu_impl.h:436-576)
template <typename T>
void build_wwt(const T* WL, const T* WR, int Dl, int Dm, int Dr, int d, std::vector<T>& out);
template <typename T>
void build_wmix_left(const T* W, int Dl, int Dr, int d, std::vector<T>& out);
template <typename T>
void build_wmix_right(const T* W, int Dl, int Dr, int d, std::vector<T>& out);

}  // namespace dmrg2
