// Host driver of one Lanczos ground-state solve on the device.
//
// The host enqueues Krylov iterations ahead of the device and polls the
// device-side `done` flag through a small pinned ring with a lookahead of
// POLL_LOOK iterations, so the GPU never idles on the host and at most
// POLL_LOOK iterations of no-op launches are issued after convergence.
#pragma once

#include <algorithm>
#include <functional>
#include <stdexcept>
#include <vector>

#include "common.cuh"
#include "kernels.cuh"

namespace dmrg2 {

template <typename T>
struct LanczosWork {
  static constexpr int POLL_RING = 8;
  static constexpr int POLL_LOOK = 2;
  T* krylov = nullptr;  // kcap vectors of length >= n
  T* w = nullptr;       // work vector
  int kcap = 0;
  LanczosDev* st = nullptr;
  RedScratch red;
  int* h_flags = nullptr;
  LanczosDev* h_st = nullptr;
  std::vector<cudaEvent_t> ev_poll, ev_mv;
  std::vector<void*> owned;

  void init(int kcap_, ll nmax) {
    kcap = std::min(kcap_, KRYLOV_CAP);
    krylov = (T*)alloc(sizeof(T) * (size_t)kcap * std::max<ll>(nmax, 1));
    w = (T*)alloc(sizeof(T) * (size_t)std::max<ll>(nmax, 1));
    st = (LanczosDev*)alloc(sizeof(LanczosDev));
    red.nblk = vec_blocks(nmax);
    red.part = (double*)alloc(sizeof(double) * (size_t)red.nblk * 2 * (KRYLOV_CAP + 2));
    red.counter = (unsigned*)alloc(sizeof(unsigned) * 4);
    DMRG2_CUDA(cudaMemset(red.counter, 0, sizeof(unsigned) * 4));
    DMRG2_CUDA(cudaMemset(st, 0, sizeof(LanczosDev)));
    h_flags = (int*)host_pinned(sizeof(int) * POLL_RING);
    h_st = (LanczosDev*)host_pinned(sizeof(LanczosDev));
    ev_poll.resize(POLL_RING);
    for (auto& e : ev_poll) DMRG2_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    ev_mv.resize(2 * KRYLOV_CAP);
    for (auto& e : ev_mv) DMRG2_CUDA(cudaEventCreate(&e));
  }
  void* alloc(size_t b) {
    void* p = nullptr;
    p = dev_alloc(b);
    owned.push_back(p);
    return p;
  }
  size_t bytes(ll nmax) const {
    return sizeof(T) * ((size_t)kcap + 1) * (size_t)nmax + sizeof(LanczosDev) +
           sizeof(double) * (size_t)red.nblk * 2 * (KRYLOV_CAP + 2);
  }
  void release() {
    for (void* p : owned) dev_free(p);
    owned.clear();
    if (h_flags) host_unpin(h_flags);
    if (h_st) host_unpin(h_st);
    h_flags = nullptr;
    h_st = nullptr;
    for (auto e : ev_poll) cudaEventDestroy(e);
    for (auto e : ev_mv) cudaEventDestroy(e);
    ev_poll.clear();
    ev_mv.clear();
  }
};

struct LanczosResult {
  double energy = 0.0;
  int iters = 0;         // Krylov vectors built (all passes)
  int matvecs = 0;
  int converged = 0;
  double matvec_s = 0.0;  // device time of the matvecs
};

// matvec(in, out, skip_flag) enqueues out = H in on stream s, doing nothing when
// *skip_flag != 0 on the device. theta: start vector on entry, normalised Ritz
// vector on exit.
template <typename T>
LanczosResult lanczos_solve(LanczosWork<T>& W, T* theta, ll n, int krylov_max, double tol,
                            int max_restarts, unsigned seed,
                            const std::function<void(const T*, T*, const int*)>& matvec,
                            cudaStream_t s) {
  LanczosResult res;
  const int kmax = (int)std::min<ll>(std::min(krylov_max, W.kcap), n);
  if (kmax < 1) throw std::runtime_error("lanczos: empty problem");
  for (int rs = 0; rs <= max_restarts; ++rs) {
    lz_start(theta, W.krylov, n, W.st, W.red, seed + 104729u * (unsigned)rs, tol, kmax, s);
    int issued = 0;
    for (int j = 0; j < kmax; ++j) {
      if (j >= LanczosWork<T>::POLL_LOOK) {
        int jj = j - LanczosWork<T>::POLL_LOOK;
        DMRG2_CUDA(cudaEventSynchronize(W.ev_poll[jj % LanczosWork<T>::POLL_RING]));
        if (W.h_flags[jj % LanczosWork<T>::POLL_RING]) break;
      }
      T* vj = W.krylov + (ll)j * n;
      DMRG2_CUDA(cudaEventRecord(W.ev_mv[2 * j], s));
      matvec(vj, W.w, &W.st->done);
      DMRG2_CUDA(cudaEventRecord(W.ev_mv[2 * j + 1], s));
      lz_dots(W.krylov, j + 1, n, W.w, W.st, W.red, s);
      lz_update_dots(W.krylov, j + 1, n, W.w, W.st, W.red, s);
      lz_update_norm_check(W.krylov, j + 1, n, W.w, W.st, W.red, j, kmax, s);
      if (j + 1 < kmax) lz_normalize_next(W.krylov + (ll)(j + 1) * n, W.w, n, W.st, s);
      DMRG2_CUDA(cudaMemcpyAsync(&W.h_flags[j % LanczosWork<T>::POLL_RING], &W.st->done,
                                 sizeof(int), cudaMemcpyDeviceToHost, s));
      DMRG2_CUDA(cudaEventRecord(W.ev_poll[j % LanczosWork<T>::POLL_RING], s));
      issued = j + 1;
    }
    DMRG2_CUDA(cudaMemcpyAsync(W.h_st, W.st, sizeof(LanczosDev), cudaMemcpyDeviceToHost, s));
    DMRG2_CUDA(cudaStreamSynchronize(s));
    if (!W.h_st->done || W.h_st->n_iter < 1) throw std::runtime_error("Lanczos did not terminate");
    const int used = std::min(issued, W.h_st->n_iter);
    for (int j = 0; j < used; ++j) {
      float ms = 0.f;
      DMRG2_CUDA(cudaEventElapsedTime(&ms, W.ev_mv[2 * j], W.ev_mv[2 * j + 1]));
      res.matvec_s += ms * 1e-3;
    }
    res.matvecs += used;
    res.iters += W.h_st->n_iter;
    res.energy = W.h_st->e_cur;
    lz_ritz(W.krylov, n, theta, W.st, W.red, s);
    res.converged = W.h_st->converged;
    if (res.converged) break;
  }
  return res;
}

}  // namespace dmrg2
