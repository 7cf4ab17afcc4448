// Cached CUDA graphs of the per-bond launch sequences.
//
// A sequence that the host would otherwise launch kernel by kernel (a Lanczos solve, a
// warm-started split) is captured once into a graph and replayed with one launch while
// its key (shapes and the device buffers it reads and writes) stays the same. Replays do
// the same arithmetic in the same order as the launches they stand for, so results are
// bitwise the same with graphs on or off.
#pragma once

#include <array>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <functional>
#include <stdexcept>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "common.cuh"

namespace dmrg2 {

using GraphKey = std::array<long long, 16>;

inline std::atomic<bool>& graphs_broken() {
  static std::atomic<bool> b{false};
  return b;
}

// on unless DMRG2_GRAPHS=0, or while GEMMs are being tuned (the tuner times candidates,
// which a capture cannot hold), or after a capture failed in this process
inline bool graphs_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("DMRG2_GRAPHS");
    return !(e && e[0] == '0') && !tune_enabled();
  }();
  return on && !graphs_broken().load();
}

// the launch sequences stay correct without graphs: use them from now on, and say why once
inline void graphs_disable(const char* why) {
  cudaGetLastError();
  if (!graphs_broken().exchange(true)) std::fprintf(stderr, "dmrg2: CUDA graphs disabled (capture failed: %s)\n", why);
}

struct GraphEntry {
  GraphKey key{};
  cudaGraph_t g = nullptr;
  cudaGraphExec_t ex = nullptr;
  long long launches = 0;  // kernels one replay runs (per loop body for a looped graph)
  long long fixed = 0;     // a looped graph's kernels outside the loop
  unsigned long long last_use = 0;
  void reset() {
    if (ex) cudaGraphExecDestroy(ex);
    if (g) cudaGraphDestroy(g);
    ex = nullptr;
    g = nullptr;
    launches = 0;
    fixed = 0;
  }
};

// DMRG2_GRAPH_STATS=1: each cache prints its builds, replays and build time when cleared
inline bool graph_stats() {
  static const bool on = [] {
    const char* e = std::getenv("DMRG2_GRAPH_STATS");
    return e && e[0] == '1';
  }();
  return on;
}

struct GraphKeyHash {
  size_t operator()(const GraphKey& k) const {
    unsigned long long h = 1469598103934665603ull;
    for (long long v : k) h = (h ^ (unsigned long long)v) * 1099511628211ull;
    return (size_t)h;
  }
};

// At most `cap` graphs; the least recently used goes first.
struct GraphCache {
  std::vector<GraphEntry> e;
  std::unordered_map<GraphKey, size_t, GraphKeyHash> index;
  std::unordered_set<GraphKey, GraphKeyHash> seen;
  unsigned long long uses = 0;
  int cap = 256;
  const char* name = "graphs";
  long long builds = 0, replays = 0;
  double build_s = 0.0;  // host time spent capturing and instantiating
  double inst_s = 0.0;   // of which in cudaGraphInstantiate

  GraphEntry* find(const GraphKey& k) {
    auto it = index.find(k);
    if (it == index.end() || !e[it->second].ex) return nullptr;
    GraphEntry* g = &e[it->second];
    g->last_use = ++uses;
    return g;
  }
  // A key is captured on its second sighting: a capture costs about as much host time as
  // a few replays save, so keys that occur once (shapes passed through while the bond
  // dimensions grow) are not captured.
  bool seen_before(const GraphKey& k) {
    if (seen.count(k)) return true;
    if (seen.size() >= 8192) seen.clear();
    seen.insert(k);
    return false;
  }
  // an empty entry carrying key k (evicting the least recently used one when full)
  GraphEntry* slot(const GraphKey& k) {
    size_t i;
    auto it = index.find(k);
    if (it != index.end()) {
      i = it->second;
      e[i].reset();
    } else if ((int)e.size() < cap) {
      e.emplace_back();
      i = e.size() - 1;
    } else {
      i = 0;
      for (size_t j = 1; j < e.size(); ++j)
        if (e[j].last_use < e[i].last_use) i = j;
      index.erase(e[i].key);
      e[i].reset();
    }
    e[i].key = k;
    e[i].last_use = ++uses;
    index[k] = i;
    return &e[i];
  }
  void clear() {
    if (graph_stats() && (builds || replays))
      std::fprintf(stderr, "[graphs] %s: %lld builds (%.3f s, %.3f s instantiating), %lld replays, %zu cached\n",
                   name, builds, build_s, inst_s, replays, e.size());
    for (auto& g : e) g.reset();
    e.clear();
    index.clear();
    seen.clear();
    builds = replays = 0;
    build_s = inst_s = 0.0;
  }
};

// Records what fn() enqueues on s into graph g (nothing runs; s may still hold queued
// work) and returns the number of kernels recorded. The launch counters drop them
// again: each replay adds what it runs.
// With dep, the recorded work follows that node of g.
inline long long capture_to_graph(cudaStream_t s, cudaGraph_t g, const std::function<void()>& fn,
                                  const cudaGraphNode_t* dep = nullptr) {
  const long long t0 = thread_launches();
  auto undo = [&]() {
    const long long nb = thread_launches() - t0;
    thread_launches() -= nb;
    launch_counter() -= nb;
    return nb;
  };
  DMRG2_CUDA(cudaStreamBeginCaptureToGraph(s, g, dep, nullptr, dep ? 1 : 0, cudaStreamCaptureModeThreadLocal));
  try {
    fn();
  } catch (...) {
    cudaGraph_t t = nullptr;
    cudaStreamEndCapture(s, &t);
    undo();
    throw;
  }
  cudaGraph_t t = nullptr;
  const cudaError_t err = cudaStreamEndCapture(s, &t);
  const long long nb = undo();
  DMRG2_CUDA(err);
  return nb;
}

// the one node of g that no other node depends on (g was recorded from one stream)
inline cudaGraphNode_t graph_leaf(cudaGraph_t g) {
  size_t n = 0;
  DMRG2_CUDA(cudaGraphGetNodes(g, nullptr, &n));
  std::vector<cudaGraphNode_t> nodes(n);
  DMRG2_CUDA(cudaGraphGetNodes(g, nodes.data(), &n));
  cudaGraphNode_t leaf = nullptr;
  int leaves = 0;
  for (auto v : nodes) {
    size_t nd = 0;
    DMRG2_CUDA(cudaGraphNodeGetDependentNodes(v, nullptr, &nd));
    if (nd == 0) {
      leaf = v;
      ++leaves;
    }
  }
  if (leaves != 1) throw std::runtime_error("graph_leaf: the recorded work does not end in one node");
  return leaf;
}

// cudaGraphInstantiate, timed into the cache's statistics
inline void graph_instantiate(GraphCache& c, GraphEntry& G) {
  const auto t0 = std::chrono::steady_clock::now();
  DMRG2_CUDA(cudaGraphInstantiate(&G.ex, G.g, 0));
  c.inst_s += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// a replay of G on s: counts its kernels as launched
inline void graph_replay(const GraphEntry& G, cudaStream_t s, long long bodies = 1) {
  DMRG2_CUDA(cudaGraphLaunch(G.ex, s));
  launch_counter() += bodies * G.launches;
  thread_launches() += bodies * G.launches;
}

}  // namespace dmrg2
