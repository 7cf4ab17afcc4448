// Host driver of one Lanczos ground-state solve on the device.
//
// Two forms, the same arithmetic:
//  - host-driven: the host enqueues Krylov iterations ahead of the device and polls the
//    device-side `done` flag through a small pinned ring with a lookahead of POLL_LOOK
//    iterations, so the GPU never idles on the host and at most POLL_LOOK iterations of
//    no-op launches are issued after convergence;
//  - device-looped: one CUDA graph per matvec identity (operator shapes and the fixed
//    buffers it reads and writes) holds the whole solve: the start (norms, reset, first
//    vector), a conditional WHILE node whose body is one Krylov step (matvec, the three
//    vector passes, the normalisation, and a one-thread kernel that advances the index
//    and ends the loop on convergence or after kmax bodies), then the Ritz vector and a
//    copy of the solver state to pinned host memory. The host copies in a seed, launches
//    the graph once per restart and waits once; no flags cross to the host between steps
//    and no no-op steps are issued. A call site opts in by passing a key; solves run
//    host-driven until a key is met the second time, when the solve is followed by the
//    capture (graphs.cuh holds the cache).
#pragma once

#include <algorithm>
#include <array>
#include <cstring>
#include <functional>
#include <stdexcept>
#include <vector>

#include "common.cuh"
#include "graphs.cuh"
#include "kernels.cuh"

namespace dmrg2 {

// identifies a matvec for the graph cache: operator shapes and device pointers, chosen by
// the caller (unused entries 0); the solve adds n, kmax, the tolerance and its buffers
using LzKey = std::array<long long, 11>;

// a converged chi=256 sweep of 100 sites meets ~100 distinct (cL, cR) bond shapes (bonds
// below the cap keep what the cutoff leaves); a graph is a few kilobytes
constexpr int LZ_GRAPH_CAP = 1024;

template <typename T>
struct LanczosWork {
  static constexpr int POLL_RING = 8;
  static constexpr int POLL_LOOK = 2;
  T* krylov = nullptr;  // kcap vectors of length >= n
  T* w = nullptr;       // work vector
  T* cur = nullptr;     // the device-looped matvec's input (a copy of the current Krylov vector)
  GraphCache graphs;    // device-looped solves, by key
  int kcap = 0;
  LanczosDev* st = nullptr;
  RedScratch red;
  int* h_flags = nullptr;
  LanczosDev* h_st = nullptr;
  unsigned* h_seed = nullptr;  // the device-looped solve's seed, copied to st->seed_in
  std::vector<cudaEvent_t> ev_poll, ev_mv;
  std::vector<void*> owned;

  void init(int kcap_, ll nmax) {
    graphs.cap = LZ_GRAPH_CAP;
    graphs.name = "lanczos";
    kcap = std::min(kcap_, KRYLOV_CAP);
    krylov = (T*)alloc(sizeof(T) * (size_t)kcap * std::max<ll>(nmax, 1));
    w = (T*)alloc(sizeof(T) * (size_t)std::max<ll>(nmax, 1));
    cur = (T*)alloc(sizeof(T) * (size_t)std::max<ll>(nmax, 1));
    st = (LanczosDev*)alloc(sizeof(LanczosDev));
    red.nblk = vec_blocks(nmax);
    red.part = (double*)alloc(sizeof(double) * (size_t)red.nblk * 2 * (KRYLOV_CAP + 2));
    red.counter = (unsigned*)alloc(sizeof(unsigned) * 4);
    DMRG2_CUDA(cudaMemset(red.counter, 0, sizeof(unsigned) * 4));
    DMRG2_CUDA(cudaMemset(st, 0, sizeof(LanczosDev)));
    h_flags = (int*)host_pinned(sizeof(int) * POLL_RING);
    h_st = (LanczosDev*)host_pinned(sizeof(LanczosDev));
    h_seed = (unsigned*)host_pinned(sizeof(unsigned));
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
    return sizeof(T) * ((size_t)kcap + 2) * (size_t)nmax + sizeof(LanczosDev) +
           sizeof(double) * (size_t)red.nblk * 2 * (KRYLOV_CAP + 2);
  }
  void release() {
    graphs.clear();
    for (void* p : owned) dev_free(p);
    owned.clear();
    if (h_flags) host_unpin(h_flags);
    if (h_st) host_unpin(h_st);
    if (h_seed) host_unpin(h_seed);
    h_flags = nullptr;
    h_st = nullptr;
    h_seed = nullptr;
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
  int device_loops = 0;   // restarts run as the device-looped graph
};

// Captures one solve of W's buffers and this matvec into G (nothing runs): the start
// (norms, reset with the seed read from st->seed_in, first vector), the WHILE node over
// the Krylov steps, the Ritz vector and the copy of the solver state to W.h_st.
template <typename T>
void lz_build_graph(LanczosWork<T>& W, GraphEntry& G, T* theta, ll n, int kmax, double tol,
                    const std::function<void(const T*, T*, const int*)>& matvec, cudaStream_t s) {
  DMRG2_CUDA(cudaGraphCreate(&G.g, 0));
  G.fixed = capture_to_graph(s, G.g, [&]() {
    lz_start(theta, W.krylov, n, W.st, W.red, 0u, tol, kmax, s, W.cur, &W.st->seed_in);
  });
  const cudaGraphNode_t start = graph_leaf(G.g);
  cudaGraphConditionalHandle h;
  DMRG2_CUDA(cudaGraphConditionalHandleCreate(&h, G.g, 1, cudaGraphCondAssignDefault));
  cudaGraphNodeParams p{};
  p.type = cudaGraphNodeTypeConditional;
  p.conditional.handle = h;
  p.conditional.type = cudaGraphCondTypeWhile;
  p.conditional.size = 1;
  cudaGraphNode_t loop;
  DMRG2_CUDA(cudaGraphAddNode(&loop, G.g, &start, 1, &p));
  G.launches = capture_to_graph(s, p.conditional.phGraph_out[0], [&]() {
    matvec(W.cur, W.w, &W.st->done);
    lz_step_dev(W.krylov, n, W.w, W.cur, W.st, W.red, kmax, s);
    lz_loop_next(W.st, h, kmax, s);
  });
  G.fixed += capture_to_graph(
      s, G.g,
      [&]() {
        lz_ritz(W.krylov, n, theta, W.st, W.red, s);
        DMRG2_CUDA(cudaMemcpyAsync(W.h_st, W.st, sizeof(LanczosDev), cudaMemcpyDeviceToHost, s));
      },
      &loop);
  graph_instantiate(W.graphs, G);
}

// matvec(in, out, skip_flag) enqueues out = H in on stream s, doing nothing when
// *skip_flag != 0 on the device. theta: start vector on entry, normalised Ritz
// vector on exit. With a key: the device-looped form, cached in W.graphs (the key must
// identify everything the matvec reads and writes besides in and out).
template <typename T>
LanczosResult lanczos_solve(LanczosWork<T>& W, T* theta, ll n, int krylov_max, double tol,
                            int max_restarts, unsigned seed,
                            const std::function<void(const T*, T*, const int*)>& matvec,
                            cudaStream_t s, const LzKey* key = nullptr) {
  LanczosResult res;
  const int kmax = (int)std::min<ll>(std::min(krylov_max, W.kcap), n);
  if (kmax < 1) throw std::runtime_error("lanczos: empty problem");
  GraphEntry* G = nullptr;
  bool build = false;
  if (key && graphs_enabled()) {
    GraphKey k{};
    std::copy(key->begin(), key->end(), k.begin());
    double tol_key = tol;
    long long tol_bits = 0;
    std::memcpy(&tol_bits, &tol_key, sizeof(tol_bits));
    k[11] = n;
    k[12] = kmax;
    k[13] = tol_bits;
    k[14] = (ll)theta;
    k[15] = (ll)&W;
    G = W.graphs.find(k);
    if (!G && W.graphs.seen_before(k)) {
      G = W.graphs.slot(k);
      build = true;
    }
  }
  for (int rs = 0; rs <= max_restarts; ++rs) {
    if (G && G->ex) {
      // the pinned seed is read by this copy before the host writes it again (the wait below)
      *W.h_seed = seed + 104729u * (unsigned)rs;
      DMRG2_CUDA(cudaMemcpyAsync(&W.st->seed_in, W.h_seed, sizeof(unsigned), cudaMemcpyHostToDevice, s));
      DMRG2_CUDA(cudaGraphLaunch(G->ex, s));
      W.graphs.replays += 1;
      DMRG2_CUDA(cudaStreamSynchronize(s));
      if (!W.h_st->done || W.h_st->n_iter < 1) throw std::runtime_error("Lanczos did not terminate");
      const int bodies = W.h_st->guard;
      launch_counter() += bodies * G->launches + G->fixed;
      thread_launches() += bodies * G->launches + G->fixed;
      res.matvecs += bodies;
      res.iters += W.h_st->n_iter;
      res.energy = W.h_st->e_cur;
      res.matvec_s += (double)W.h_st->mv_ns * 1e-9;
      res.converged = W.h_st->converged;
      res.device_loops += 1;
      if (res.converged) break;
      continue;
    }
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
  if (build) {
    try {
      const auto t0 = std::chrono::steady_clock::now();
      lz_build_graph(W, *G, theta, n, kmax, tol, matvec, s);
      W.graphs.builds += 1;
      W.graphs.build_s += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    } catch (const std::exception& e) {
      G->reset();
      graphs_disable(e.what());
    }
  }
  return res;
}

}  // namespace dmrg2
