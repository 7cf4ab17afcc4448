// Two-site DMRG sweep engine.
//
// Mirrors the algorithm of the reference driver (gpu-rocm/dmrg2-gpu/src/dmrg2_gpu_impl.h):
// build environments (941-964), then per sweep a left-to-right and a
// right-to-left half sweep (1366-1413); each bond forms theta (583-600), finds
// the ground state of H_eff with Lanczos (971-1160), splits it by a truncated
// SVD (1167-1343) and updates one environment (787-934). The sweep energy is
// the eigenvalue of the last bond optimised and the run stops at |dE| < tol
// (1440-1447).
//
// Differences by design (all device-resident, no library calls):
//  * any MPS can be loaded (set_mps); it is right-canonicalised on the device
//    before the environments are built, so first-sweep energies are variational;
//  * per-sweep chi schedule, cutoff, Krylov cap and restarts;
//  * per-sweep energy, truncation error (discarded weight) and timings.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <functional>
#include <memory>
#include <random>
#include <thread>
#include <type_traits>

#include "contract.cuh"
#include "engine.h"
#include "lanczos_driver.cuh"
#include "rsvd.cuh"
#include "truncate.cuh"
#include "truncate_c.cuh"

namespace dmrg2 {

namespace {
// the warm-started subspace split goes with the density-matrix route; its Cholesky factor
// has order k (real data) or 2k (complex data, on the real embedding), at most CHOL_MAX
bool warm_capable(const EngineConfig& c) {
  return c.truncation == 0 && c.svd_method == 0 && !c.single_site &&
         (c.complex ? 2 * c.chi_max : c.chi_max) <= CHOL_MAX;
}
// the randomised split is an option of two-site sweeps with the density-matrix split
bool rsvd_capable(const EngineConfig& c) {
  return c.truncation == 2 && c.svd_method == 0 && !c.single_site;
}

ll ipow_cap(int d, int e, ll cap) {
  ll v = 1;
  for (int i = 0; i < e; ++i) {
    v *= d;
    if (v >= cap) return cap;
  }
  return v;
}
}  // namespace

// the lane the calling host thread works on, per engine (see Engine::LaneScope)
thread_local const void* tl_lane_engine = nullptr;
thread_local void* tl_lane = nullptr;

template <typename T>
class Engine final : public EngineBase {
 public:
  explicit Engine(const EngineConfig& c) : cfg_(c) {
    if (cfg_.L < 2) throw std::runtime_error("L must be >= 2");
    if (cfg_.d < 1) throw std::runtime_error("d must be >= 1");
    if (cfg_.chi_max < 1) throw std::runtime_error("chi_max must be >= 1");
    if (cfg_.krylov_max < 2) cfg_.krylov_max = 2;
    if (cfg_.single_site && (cfg_.svd_method != 0 || cfg_.precision != 0))
      throw std::invalid_argument("single-site sweeps use the density-matrix truncation and FP64 matvecs");
    L_ = cfg_.L;
    d_ = cfg_.d;
    reset_split_history();
    lanes_.emplace_back(new Lane());
    DMRG2_CUDA(cudaStreamCreateWithFlags(&lanes_[0]->st, cudaStreamNonBlocking));
    cap_.resize(L_ + 1);
    for (int i = 0; i <= L_; ++i) cap_[i] = (int)ipow_cap(d_, std::min(i, L_ - i), cfg_.chi_max);
    dims_.assign(L_ + 1, 1);
    mps_.assign(L_, nullptr);
    {  // every MPS slot in one allocation, 256-byte aligned slices
      std::vector<size_t> off(L_);
      size_t tot = 0;
      for (int i = 0; i < L_; ++i) {
        off[i] = tot;
        tot += round256(sizeof(T) * (size_t)std::max<ll>((ll)cap_[i] * d_ * cap_[i + 1], 1));
      }
      void* p = nullptr;
      p = dev_alloc(tot);
      allocs_.push_back(p);
      for (int i = 0; i < L_; ++i) {
        mps_[i] = (T*)((char*)p + off[i]);
        bytes_ += sizeof(T) * (size_t)std::max<ll>((ll)cap_[i] * d_ * cap_[i + 1], 1);
      }
    }
    nmax_ = 1;
    for (int i = 0; i + 1 < L_; ++i) nmax_ = std::max(nmax_, (ll)cap_[i] * d_ * d_ * cap_[i + 2]);
    qmax_ = 1;
    for (int i = 0; i + 1 < L_; ++i) {
      ll m = (ll)cap_[i] * d_, n = (ll)d_ * cap_[i + 2];
      qmax_ = std::max(qmax_, std::max(m, n));
    }
    for (int i = 0; i < L_; ++i) qmax_ = std::max(qmax_, (ll)d_ * cap_[i + 1]);
    init_lane(*lanes_[0], true);
    canon_flags_ = (int*)dalloc_bytes(sizeof(int) * (size_t)(L_ + 1));
    h_flags_ = (int*)host_pinned(sizeof(int) * (size_t)(L_ + 1));
    DMRG2_CUDA(cudaEventCreate(&ev_s0_));
    DMRG2_CUDA(cudaEventCreate(&ev_s1_));
  }

  ~Engine() override {
    cudaStreamSynchronize(ln().st);
    free_tmp();
    free_mpo();
    for (void* p : allocs_) dev_free(p);
    host_unpin(h_flags_);
    cudaEventDestroy(ev_s0_);
    cudaEventDestroy(ev_s1_);
    for (auto& l : lanes_) release_lane(*l);
  }

  EngineConfig& config() override { return cfg_; }
  double energy() const override { return energy_; }
  double env_build_s() const override { return env_build_s_; }
  const std::vector<int>& bond_dims() const override { return dims_; }
  size_t device_bytes() const override { return bytes_ + bytes_mpo_; }

  // --------------------------------------------------------------------------
  void set_mpo(const std::vector<const void*>& W, const std::vector<int>& Dl,
               const std::vector<int>& Dr) override {
    if ((int)W.size() != L_ || (int)Dl.size() != L_ || (int)Dr.size() != L_)
      throw std::runtime_error("set_mpo: expected L tensors and bond dims");
    if (Dl[0] != 1 || Dr[L_ - 1] != 1)
      throw std::runtime_error("set_mpo: boundary MPO bonds must be 1 (Dl[0] = Dr[L-1] = 1)");
    for (int i = 0; i + 1 < L_; ++i)
      if (Dr[i] != Dl[i + 1]) throw std::runtime_error("set_mpo: Dr[i] != Dl[i+1]");
    for (int i = 0; i < L_; ++i)
      if (Dl[i] < 1 || Dr[i] < 1 || Dl[i] > 4096 || Dr[i] > 4096)
        throw std::runtime_error("set_mpo: bad MPO bond dimension");
    DMRG2_CUDA(cudaStreamSynchronize(ln().st));
    free_mpo();
    Dl_ = Dl;
    Dr_ = Dr;
    Db_.assign(L_ + 1, 1);
    for (int i = 0; i < L_; ++i) Db_[i] = Dl[i];
    Db_[L_] = Dr[L_ - 1];
    hW_.assign(L_, {});
    for (int i = 0; i < L_; ++i) {
      size_t n = (size_t)Dl[i] * Dr[i] * d_ * d_;
      hW_[i].resize(n);
      std::memcpy(hW_[i].data(), W[i], n * sizeof(T));
    }
    // host images of the mixing matrices and fused two-site MPOs
    std::vector<std::vector<T>> hml(L_), hmr(L_), hww(L_ - 1);
    for (int i = 0; i < L_; ++i) {
      build_wmix_left(hW_[i].data(), Dl[i], Dr[i], d_, hml[i]);
      build_wmix_right(hW_[i].data(), Dl[i], Dr[i], d_, hmr[i]);
    }
    for (int i = 0; i + 1 < L_; ++i) build_wwt(hW_[i].data(), hW_[i + 1].data(), Dl[i], Dr[i], Dr[i + 1], d_, hww[i]);
    // each bond's fused MPO also in its nonzero form; the mixing step uses it where at
    // most half the entries are nonzero (DMRG2_MIX_DENSE=1: always the dense form)
    static const bool mix_dense = [] {
      const char* e = std::getenv("DMRG2_MIX_DENSE");
      return e && e[0] == '1';
    }();
    wwt_sparse_.assign(L_ - 1, 0);
    for (int i = 0; i + 1 < L_; ++i) {
      const int Kin = Dl[i] * d_ * d_, Kout = d_ * d_ * Dr[i + 1];
      const int nnz = wwt_sparse_block(hww[i], Kin, Kout);
      wwt_sparse_[i] = (!mix_dense && 2 * (ll)nnz <= (ll)Kin * Kout && Kin <= 32 && Kout <= 32) ? 1 : 0;
    }
    // contraction scratch
    ll xs = 1;
    const ll dd = (ll)d_ * d_;
    for (int i = 0; i + 1 < L_; ++i) {
      ll cL = cap_[i], cR = cap_[i + 2];
      xs = std::max(xs, cL * Db_[i] * dd * cR);
      xs = std::max(xs, cL * dd * Db_[i + 2] * cR);
    }
    for (int i = 0; i < L_; ++i) {
      ll a = cap_[i], b = cap_[i + 1];
      xs = std::max(xs, a * Dl[i] * d_ * b);
      xs = std::max(xs, a * d_ * Dr[i] * b);
      xs = std::max(xs, b * Dr[i] * d_ * a);
      xs = std::max(xs, (ll)d_ * b * Dl[i] * a);
    }
    // one device allocation for every MPO-dependent buffer, carved in 256-byte aligned
    // slices; the uploaded matrices form its prefix and cross to the device in one copy
    auto el = [](ll n) { return sizeof(T) * (size_t)std::max<ll>(n, 1); };
    size_t up = 0;
    for (auto& h : hml) up += round256(el((ll)h.size()));
    for (auto& h : hmr) up += round256(el((ll)h.size()));
    for (auto& h : hww) up += round256(el((ll)h.size()));
    ll opn = 1, opw = 1;  // staged operator slots
    for (int i = 0; i <= L_; ++i) opn = std::max(opn, (ll)cap_[i] * cap_[i] * Db_[i]);
    for (auto& h : hww) opw = std::max(opw, (ll)h.size());
    for (auto& h : hml) opw = std::max(opw, (ll)h.size());
    size_t total = up + 2 * round256(el(xs)) + 2 * round256(el(opn)) + round256(el(opw));
    for (int i = 0; i <= L_; ++i) total += 2 * round256(el((ll)cap_[i] * cap_[i] * Db_[i]));
    mpo_slab_ = dev_alloc(total);
    std::vector<char> stage(up);
    size_t off = 0;
    auto carve = [&](ll n) {
      T* p = (T*)((char*)mpo_slab_ + off);
      off += round256(el(n));
      bytes_mpo_ += el(n);
      return p;
    };
    auto put = [&](const std::vector<T>& h) {
      if (!h.empty()) std::memcpy(stage.data() + off, h.data(), sizeof(T) * h.size());
      return carve((ll)h.size());
    };
    wml_.assign(L_, nullptr);
    wmr_.assign(L_, nullptr);
    wwt_.assign(L_ - 1, nullptr);
    for (int i = 0; i < L_; ++i) {
      wml_[i] = put(hml[i]);
      wmr_[i] = put(hmr[i]);
    }
    for (int i = 0; i + 1 < L_; ++i) wwt_[i] = put(hww[i]);
    DMRG2_CUDA(cudaMemcpy(mpo_slab_, stage.data(), up, cudaMemcpyHostToDevice));
    lenv_.assign(L_ + 1, nullptr);
    renv_.assign(L_ + 1, nullptr);
    for (int i = 0; i <= L_; ++i) {
      ll n = (ll)cap_[i] * cap_[i] * Db_[i];
      lenv_[i] = carve(n);
      renv_[i] = carve(n);
    }
    lanes_[0]->X = carve(xs);
    lanes_[0]->Y = carve(xs);
    lanes_[0]->opL = carve(opn);
    lanes_[0]->opR = carve(opn);
    lanes_[0]->opW = carve(opw);
    xs_ = xs;
    opn_ = opn;
    opw_ = opw;
    mpo_set_ = true;
    envs_valid_ = false;
  }

  void set_mps(const std::vector<const void*>& A, const std::vector<int>& dims) override {
    if ((int)A.size() != L_ || (int)dims.size() != L_ + 1)
      throw std::runtime_error("set_mps: expected L tensors and L+1 bond dims");
    if (dims[0] != 1 || dims[L_] != 1) throw std::runtime_error("set_mps: boundary bonds must be 1");
    for (int i = 0; i <= L_; ++i)
      if (dims[i] < 1 || dims[i] > cap_[i])
        throw std::runtime_error("set_mps: bond " + std::to_string(i) + " dimension " +
                                 std::to_string(dims[i]) + " exceeds min(chi_max, d^min(i,L-i)) = " +
                                 std::to_string(cap_[i]));
    DMRG2_CUDA(cudaStreamSynchronize(ln().st));
    dims_ = dims;
    for (int i = 0; i < L_; ++i) {
      size_t n = (size_t)dims[i] * d_ * dims[i + 1];
      DMRG2_CUDA(cudaMemcpy(mps_[i], A[i], n * sizeof(T), cudaMemcpyHostToDevice));
    }
    mps_set_ = true;
    canonical_ = false;
    envs_valid_ = false;
    reset_split_history();
  }

  void get_mps(std::vector<void*>& out) override {
    DMRG2_CUDA(cudaStreamSynchronize(ln().st));
    for (int i = 0; i < L_; ++i) {
      size_t n = (size_t)dims_[i] * d_ * dims_[i + 1];
      DMRG2_CUDA(cudaMemcpy(out[i], mps_[i], n * sizeof(T), cudaMemcpyDeviceToHost));
    }
  }

  // --------------------------------------------------------------------------
  std::vector<SweepStats> run(const std::vector<int>& schedule) override {
    if (!mpo_set_) throw std::runtime_error("run: MPO not set");
    if (!mps_set_) throw std::runtime_error("run: MPS not set");
    for (int c : schedule)
      if (c < 1 || c > cfg_.chi_max) throw std::runtime_error("run: schedule chi outside [1, chi_max]");
    auto t0 = std::chrono::steady_clock::now();
    right_canonicalize();
    reset_split_history();
    build_right_envs();
    DMRG2_CUDA(cudaStreamSynchronize(ln().st));
    env_build_s_ = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();

    envs_valid_ = true;
    return sweeps(schedule, true);
  }

  std::vector<SweepStats> resume(const std::vector<int>& schedule) override {
    if (!envs_valid_) throw std::logic_error("resume: no previous run on this MPS/MPO");
    for (int c : schedule)
      if (c < 1 || c > cfg_.chi_max) throw std::runtime_error("resume: schedule chi outside [1, chi_max]");
    return sweeps(schedule, false);
  }

  // ---------------------------------------------------------------- parallel sweep
  // Segmented sweeps with boundary merges (the reference's PDMRGGPU, gpu-rocm/pdmrg-gpu/
  // src/pdmrg_gpu_impl.h:2320-2725; Stoudenmire and White, New J. Phys. 15, 2013). The
  // chain is cut into P segments (partition_chain, :582-601). After full-chain warm-up
  // sweeps, each local iteration runs: even segments left-to-right and odd ones
  // right-to-left, concurrently (one host thread and one lane, i.e. stream and scratch,
  // per segment); then every even boundary is merged; then the segments sweep back the
  // other way and the odd boundaries are merged. A merge optimises theta = psi_L diag(V)
  // psi_R over the boundary bond, with V = 1/S from the last merge there (ones at first),
  // splits it with the Jacobi SVD (the small singular values enter V with relative
  // accuracy), stores V = 1/max(S, 1e-12), keeps U on the left site and S Vh on the right
  // one, and rebuilds both boundary environments from the orthonormal factors U and Vh.
  // The energy is the last merge's eigenvalue; the outer loop stops once it changes by less
  // than tol. Warm-up, recalibration and polish sweeps are full-chain two-site sweeps.
  // At the end V is put back into the boundaries that were swept from both sides after
  // their last merge (psi = psi_L V psi_R) and the MPS is right-canonicalised, so get_mps
  // and expect_local see one normalised state.
  std::vector<SweepStats> pdmrg(const PdmrgOptions& o) override {
    if (!mpo_set_) throw std::runtime_error("pdmrg: MPO not set");
    if (!mps_set_) throw std::runtime_error("pdmrg: MPS not set");
    if (cfg_.single_site) throw std::invalid_argument("pdmrg: the parallel sweep is two-site");
    const int P = o.n_segments;
    const int chi = o.chi > 0 ? o.chi : cfg_.chi_max;
    if (chi > cfg_.chi_max) throw std::invalid_argument("pdmrg: chi above chi_max");
    if (P < 2 || 2 * P > L_) throw std::invalid_argument("pdmrg: n_segments must lie in 2..L/2");
    if (o.n_outer < 1 || o.n_local < 1 || o.n_warmup < 0 || o.n_polish < 0 || o.n_recal < 0)
      throw std::invalid_argument("pdmrg: bad iteration counts");
    // the left-to-right half of a full sweep builds the left environments the segments
    // start from (the right ones come from the canonical form below)
    if (o.n_warmup < 1) throw std::invalid_argument("pdmrg: at least one warm-up sweep is needed");
    int device = 0;
    DMRG2_CUDA(cudaGetDevice(&device));
    std::vector<SweepStats> out;
    auto t0 = std::chrono::steady_clock::now();
    right_canonicalize();
    reset_split_history();
    build_right_envs();
    DMRG2_CUDA(cudaStreamSynchronize(ln().st));
    env_build_s_ = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    envs_valid_ = true;
    auto full_sweeps = [&](int n, int phase) {
      if (n <= 0) return;
      for (SweepStats& st : sweeps(std::vector<int>((size_t)n, chi), false)) {
        st.phase = phase;
        out.push_back(st);
      }
    };
    full_sweeps(o.n_warmup, 1);
    // segments: the first L % P take one site more (partition_chain)
    std::vector<int> first(P), last(P);
    for (int k = 0, pos = 0; k < P; ++k) {
      const int len = L_ / P + (k < L_ % P ? 1 : 0);
      first[k] = pos;
      last[k] = pos + len - 1;
      pos += len;
    }
    // lanes 1..P, the boundary vectors V on the device; both freed on every exit
    struct Cleanup {
      Engine* e;
      std::vector<double*> v;
      ~Cleanup() {
        while (e->lanes_.size() > 1) {  // synchronises each lane's stream first
          e->release_lane(*e->lanes_.back());
          e->lanes_.pop_back();
        }
        cudaStreamSynchronize(e->ln().st);
        for (double* p : v) dev_free(p);
      }
    } cleanup{this, {}};
    while ((int)lanes_.size() < P + 1) {
      lanes_.emplace_back(new Lane());
      init_lane(*lanes_.back(), false);
    }
    std::vector<double*>& V = cleanup.v;
    V.assign((size_t)(P - 1), nullptr);
    const std::vector<double> ones((size_t)cfg_.chi_max, 1.0);
    auto reset_v = [&]() {
      for (double* p : V) DMRG2_CUDA(cudaMemcpy(p, ones.data(), sizeof(double) * ones.size(), cudaMemcpyHostToDevice));
    };
    for (auto& p : V) p = (double*)dev_alloc(sizeof(double) * ones.size());
    reset_v();
    // runs job(k, stats) for k < n on lanes 1..n, one host thread each, and waits
    auto parallel = [&](int n, const std::function<void(int, SweepStats&)>& job) {
      std::vector<SweepStats> st((size_t)n);
      std::vector<std::exception_ptr> ex((size_t)n);
      std::vector<std::thread> th;
      for (int k = 0; k < n; ++k)
        th.emplace_back([&, k] {
          try {
            DMRG2_CUDA(cudaSetDevice(device));
            LaneScope scope(this, lanes_[(size_t)k + 1].get());
            job(k, st[(size_t)k]);
            DMRG2_CUDA(cudaStreamSynchronize(ln().st));
          } catch (...) {
            ex[(size_t)k] = std::current_exception();
          }
        });
      for (auto& t : th) t.join();
      for (auto& e : ex)
        if (e) std::rethrow_exception(e);
      return st;
    };
    // psi = psi_L V psi_R at the boundaries swept from both sides since their last merge
    std::vector<char> needs_v((size_t)(P - 1), 0);
    auto settle = [&]() {
      for (int b = 0; b + 1 < P; ++b)
        if (needs_v[(size_t)b]) {
          const int bs = last[b];
          row_scale<T>(mps_[bs + 1], V[(size_t)b], dims_[bs + 1], (ll)d_ * dims_[bs + 2], mps_[bs + 1], false,
                       ln().st);
          needs_v[(size_t)b] = 0;
        }
      DMRG2_CUDA(cudaStreamSynchronize(ln().st));
    };
    auto half_sweep = [&](int parity, SweepStats& acc) {
      // parity 0: even segments left-to-right, odd right-to-left; parity 1 the reverse
      for (const SweepStats& st : parallel(P, [&](int k, SweepStats& ss) {
             const char dir = ((k & 1) == parity) ? 'R' : 'L';
             if (dir == 'R')
               for (int i = first[k]; i < last[k]; ++i) optimize_bond(i, 'R', chi, ss);
             else
               for (int i = last[k] - 1; i >= first[k]; --i) optimize_bond(i, 'L', chi, ss);
           }))
        add_stats(acc, st);
      for (int b = 0; b + 1 < P; ++b) needs_v[(size_t)b] = 1;  // both neighbours moved
    };
    auto merge = [&](int parity, SweepStats& acc) {
      std::vector<int> act;
      for (int b = parity; b + 1 < P; b += 2) act.push_back(b);
      if (act.empty()) return;
      std::vector<double> e(act.size());
      auto st = parallel((int)act.size(), [&](int j, SweepStats& ss) {
        e[(size_t)j] = merge_boundary(last[act[(size_t)j]], V[(size_t)act[(size_t)j]], chi, ss);
      });
      for (const SweepStats& x : st) add_stats(acc, x);
      for (int b : act) needs_v[(size_t)b] = 0;
      energy_ = e.back();
    };
    double e_prev = energy_;
    bool converged = false;
    for (int outer = 0; outer < o.n_outer; ++outer) {
      SweepStats so;
      so.phase = 2;
      so.sweep = outer;
      so.chi_max = chi;
      auto ts = std::chrono::steady_clock::now();
      double e_local = energy_;
      for (int loc = 0; loc < o.n_local; ++loc) {
        half_sweep(0, so);
        merge(0, so);
        half_sweep(1, so);
        merge(1, so);
        if (std::fabs(energy_ - e_local) < cfg_.tol && loc > 0) break;
        e_local = energy_;
      }
      so.wall_s = so.device_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - ts).count();
      so.energy = energy_;
      so.max_bond = *std::max_element(dims_.begin(), dims_.end());
      out.push_back(so);
      const double dE = std::fabs(energy_ - e_prev);
      e_prev = energy_;
      if (dE < cfg_.tol) {
        converged = true;
        break;
      }
      if (o.n_recal > 0 && (outer + 1) % o.n_recal == 0 && outer + 1 < o.n_outer) {
        settle();
        right_canonicalize();
        build_right_envs();
        full_sweeps(1, 3);
        e_prev = energy_;
        reset_v();
      }
    }
    settle();
    if (o.n_polish > 0 && !converged) {
      right_canonicalize();
      build_right_envs();
      full_sweeps(o.n_polish, 4);
    }
    right_canonicalize();
    DMRG2_CUDA(cudaStreamSynchronize(ln().st));
    envs_valid_ = false;  // environments of the segmented state; run() rebuilds them
    return out;
  }

  // one boundary merge on the calling thread's lane (see pdmrg); returns the eigenvalue
  double merge_boundary(int bs, double* V, int chi, SweepStats& ss) {
    Lane& l = ln();
    const int cL = dims_[bs], cM = dims_[bs + 1], cR = dims_[bs + 2];
    const ll m = (ll)cL * d_, nc = (ll)d_ * cR;
    row_scale<T>(mps_[bs + 1], V, cM, nc, l.svdX, false, l.st);  // diag(V) psi_R
    theta_form(mps_[bs], l.svdX, l.theta, cL, cM, cR, d_, l.st, l.X, xs_);
    const double e = lanczos(bs, m * nc, ss);
    DMRG2_CUDA(cudaEventRecord(l.ev_c, l.st));
    DMRG2_CUDA(cudaMemcpyAsync(l.svdX, l.theta, sizeof(T) * (size_t)(m * nc), cudaMemcpyDeviceToDevice, l.st));
    set_identity(l.svdQ, (int)m, l.st);
    svd_jacobi(l.svdX, l.svdQ, (int)m, nc, l.jctl, cfg_.jacobi_max_sweeps, jacobi_tol(nc), nullptr, l.st);
    svd_sort_truncate(l.svdX, (int)m, nc, l.sigma, l.perm, l.svdout, chi, cfg_.cutoff, false, l.jctl, l.st);
    DMRG2_CUDA(cudaEventRecord(l.ev_d, l.st));
    const SvdOut so = read_svd();
    const int k = so.k;
    svd_gather(l.svdX, l.svdQ, l.perm, (int)m, nc, k, 0, mps_[bs], mps_[bs + 1], l.st);  // U, S Vh
    dims_[bs + 1] = k;
    gather_sigma(l.sigma, l.perm, k, V, l.st);                   // V <- S
    row_scale<T>(mps_[bs + 1], V, k, nc, l.svdQ, true, l.st);   // Vh = diag(1/S) S Vh
    inv_clip(V, k, 1e-12, l.st);                                 // V <- 1 / max(S, 1e-12)
    env_left(lenv_[bs], mps_[bs], wml_[bs], lenv_[bs + 1], l.X, l.Y, cL, k, d_, Dl_[bs], Dr_[bs], l.st);
    env_right(renv_[bs + 2], l.svdQ, wmr_[bs + 1], renv_[bs + 1], l.X, l.Y, cR, k, d_, Dl_[bs + 1], Dr_[bs + 1],
              l.st);
    float ms = 0.f;
    DMRG2_CUDA(cudaEventElapsedTime(&ms, l.ev_c, l.ev_d));
    ss.svd_s += ms * 1e-3;
    ss.jacobi_sweeps_max = std::max(ss.jacobi_sweeps_max, so.jacobi_sweeps);
    ss.trunc_err_max = std::max(ss.trunc_err_max, so.trunc_err);
    ss.trunc_err_sum += so.trunc_err;
    te_ref_[bs] = so.trunc_err;
    short_age_[bs] = 0;
    return e;
  }

  static void add_stats(SweepStats& a, const SweepStats& b) {
    a.trunc_err_max = std::max(a.trunc_err_max, b.trunc_err_max);
    a.trunc_err_sum += b.trunc_err_sum;
    a.matvecs += b.matvecs;
    a.heff_s += b.heff_s;
    a.heff_flops += b.heff_flops;
    a.lanczos_iters += b.lanczos_iters;
    a.lanczos_unconverged += b.lanczos_unconverged;
    a.svd_s += b.svd_s;
    a.jacobi_sweeps_max = std::max(a.jacobi_sweeps_max, b.jacobi_sweeps_max);
    a.lowprec_matvecs += b.lowprec_matvecs;
    a.warm_splits += b.warm_splits;
    a.warm_fallbacks += b.warm_fallbacks;
    a.eig_fallbacks += b.eig_fallbacks;
    a.warm_short += b.warm_short;
    a.rsvd_splits += b.rsvd_splits;
    a.rsvd_fallbacks += b.rsvd_fallbacks;
    a.device_loops += b.device_loops;
  }

  std::vector<SweepStats> sweeps(const std::vector<int>& schedule, bool stop_rule) {
    std::vector<SweepStats> out;
    double e_prev = energy_;
    for (size_t sw = 0; sw < schedule.size(); ++sw) {
      SweepStats ss;
      ss.sweep = (int)sw;
      ss.chi_max = schedule[sw];
      auto ts = std::chrono::steady_clock::now();
      DMRG2_CUDA(cudaEventRecord(ev_s0_, ln().st));
      double e = 0.0;
      if (cfg_.single_site) {
        e = sweep1(schedule[sw], ss);
      } else {
        for (int i = 0; i + 1 < L_; ++i) e = optimize_bond(i, 'R', schedule[sw], ss);
        for (int i = L_ - 2; i >= 0; --i) e = optimize_bond(i, 'L', schedule[sw], ss);
      }
      DMRG2_CUDA(cudaEventRecord(ev_s1_, ln().st));
      DMRG2_CUDA(cudaStreamSynchronize(ln().st));
      float ms = 0.f;
      DMRG2_CUDA(cudaEventElapsedTime(&ms, ev_s0_, ev_s1_));
      ss.device_s = ms * 1e-3;
      ss.wall_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - ts).count();
      ss.energy = e;
      ss.max_bond = *std::max_element(dims_.begin(), dims_.end());
      energy_ = e;
      prev_sweep_chi_ = schedule[sw];
      out.push_back(ss);
      if (stop_rule && (int)sw + 1 >= cfg_.min_sweeps && std::fabs(e - e_prev) < cfg_.tol) break;
      e_prev = e;
    }
    canonical_ = true;
    return out;
  }

  // <O_i> for all sites; valid on a right-canonical MPS with its norm on site 0
  void expect_local(const void* op, std::vector<double>& re, std::vector<double>& im) override {
    if (!mps_set_) throw std::runtime_error("expect_local: MPS not set");
    if (!mpo_set_) throw std::runtime_error("expect_local: MPO not set (scratch buffers)");
    if (!canonical_) right_canonicalize();
    const ll cm = cfg_.chi_max;
    T* E = dalloc_tmp(cm * cm);
    T* E2 = dalloc_tmp(cm * cm);
    T* F = dalloc_tmp(cm * cm);
    T* opd = dalloc_tmp((ll)d_ * d_);
    T* idd = dalloc_tmp((ll)d_ * d_);
    double* res = (double*)dalloc_tmp_bytes(sizeof(double) * 2 * (L_ + 1));
    std::vector<T> hid((size_t)d_ * d_, ST<T>::zero());
    for (int i = 0; i < d_; ++i) hid[(size_t)i * d_ + i] = ST<T>::one();
    DMRG2_CUDA(cudaMemcpyAsync(opd, op, sizeof(T) * d_ * d_, cudaMemcpyHostToDevice, ln().st));
    DMRG2_CUDA(cudaMemcpyAsync(idd, hid.data(), sizeof(T) * d_ * d_, cudaMemcpyHostToDevice, ln().st));
    T one = ST<T>::one();
    DMRG2_CUDA(cudaMemcpyAsync(E, &one, sizeof(T), cudaMemcpyHostToDevice, ln().st));
    for (int i = 0; i < L_; ++i) {
      int a = dims_[i], b = dims_[i + 1];
      env_left(E, mps_[i], opd, F, ln().X, ln().Y, a, b, d_, 1, 1, ln().st);
      trace_real(F, b, b, res + 2 * i, res + 2 * i + 1, ln().st);
      env_left(E, mps_[i], idd, E2, ln().X, ln().Y, a, b, d_, 1, 1, ln().st);
      if (i == 0) trace_real(E2, b, b, res + 2 * L_, res + 2 * L_ + 1, ln().st);
      std::swap(E, E2);
    }
    std::vector<double> h(2 * (L_ + 1));
    DMRG2_CUDA(cudaMemcpyAsync(h.data(), res, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, ln().st));
    DMRG2_CUDA(cudaStreamSynchronize(ln().st));
    free_tmp();
    double nrm = h[2 * L_];
    re.resize(L_);
    im.resize(L_);
    for (int i = 0; i < L_; ++i) {
      re[i] = h[2 * i] / nrm;
      im[i] = h[2 * i + 1] / nrm;
    }
  }

 private:
  // ---------------------------------------------------------------- memory
  T* dalloc(ll n) { return (T*)dalloc_bytes(sizeof(T) * (size_t)std::max<ll>(n, 1)); }
  void* dalloc_bytes(size_t b) {
    void* p = nullptr;
    p = dev_alloc(b);
    allocs_.push_back(p);
    bytes_ += b;
    return p;
  }
  static size_t round256(size_t b) { return (b + 255) & ~(size_t)255; }
  T* dalloc_tmp(ll n) { return (T*)dalloc_tmp_bytes(sizeof(T) * (size_t)std::max<ll>(n, 1)); }
  void* dalloc_tmp_bytes(size_t b) {
    void* p = nullptr;
    p = dev_alloc(b);
    tmp_allocs_.push_back(p);
    return p;
  }
  void free_tmp() {
    for (void* p : tmp_allocs_) dev_free(p);
    tmp_allocs_.clear();
  }
  void free_mpo() {
    if (mpo_slab_) dev_free(mpo_slab_);
    mpo_slab_ = nullptr;
    bytes_mpo_ = 0;
  }

  // rotation threshold on |<x_p,x_q>| / (|x_p||x_q|): len * eps, as LAPACK's
  // one-sided Jacobi (dgesvj) uses; below that the computed inner products are noise
  double jacobi_tol(ll len) const { return 2.2e-16 * std::max<double>(16.0, (double)len); }

  // ---------------------------------------------------------------- setup
  // Highest site whose tensor is not a right isometry (A A^H = 1 to 1e-12), with every
  // site above it one; 0 when sites 1..L-1 all are. Such sites (an MPS read back after
  // a right-to-left half-sweep, a checkpoint) need no decomposition: A A^H = 1 makes the
  // density matrix a projector, whose degenerate spectrum would only be rotated.
  int first_non_isometry() {
    for (int i = L_ - 1; i >= 1; --i) {
      const int cl = dims_[i], nc = d_ * dims_[i + 1];
      Gemm<T> g;  // conj(A A^H) = conj(A) A^T
      g.ca = true; g.tb = true;
      g.M = cl; g.N = cl; g.K = nc;
      g.A = mps_[i]; g.lda = nc;
      g.B = mps_[i]; g.ldb = nc;
      g.C = ln().theta; g.ldc = cl;
      launch_gemm(g, ln().st);
      identity_check(ln().theta, cl, 1e-12, canon_flags_ + i, ln().st);
    }
    DMRG2_CUDA(cudaMemcpyAsync(h_flags_, canon_flags_, sizeof(int) * (size_t)(L_ + 1), cudaMemcpyDeviceToHost, ln().st));
    DMRG2_CUDA(cudaStreamSynchronize(ln().st));
    for (int i = L_ - 1; i >= 1; --i)
      if (!h_flags_[i]) return i;
    return 0;
  }

  void right_canonicalize() {
    envs_valid_ = false;
    const int first = first_non_isometry();
    for (int i = first; i >= 1; --i) {
      const int cl = dims_[i], cr = dims_[i + 1];
      const int nc = d_ * cr;
      const int chi = std::min(cfg_.chi_max, cap_[i]);
      int k = 0;
      bool jacobi = (cfg_.svd_method == 1);
      if (!jacobi) {
        try {
          SvdOut o = eig_split(ln().ew, mps_[i], cl, nc, 'L', chi, 1e-14, true, ln().tmp, mps_[i], ln().st);
          k = o.k;
          scale_inplace(ln().tmp, (ll)cl * k, &ln().ew.out->sigma_max2, ln().st);
        } catch (const NumericError&) {
          jacobi = true;  // eigenvectors not orthonormal: the Jacobi SVD splits this site
        }
      }
      if (jacobi) {
        transpose(mps_[i], ln().svdX, cl, nc, ln().st);
        norm2(ln().svdX, (ll)cl * nc, ln().dscal, ln().red, ln().st);
        set_identity(ln().svdQ, nc, ln().st);
        svd_jacobi(ln().svdX, ln().svdQ, nc, (ll)cl, ln().jctl, cfg_.jacobi_max_sweeps, jacobi_tol(cl), ln().dscal, ln().st);
        svd_sort_truncate(ln().svdX, nc, (ll)cl, ln().sigma, ln().perm, ln().svdout, chi, 1e-14, true, ln().jctl, ln().st);
        k = read_svd().k;
        svd_gather(ln().svdX, ln().svdQ, ln().perm, nc, (ll)cl, k, 1, ln().tmp, mps_[i], ln().st);
        scale_inplace(ln().tmp, (ll)cl * k, &ln().svdout->sigma_max2, ln().st);
      }
      {  // A[i-1] <- A[i-1] . (U S / sigma_max)
        Gemm<T> g;
        g.M = dims_[i - 1] * d_; g.N = k; g.K = cl;
        g.A = mps_[i - 1]; g.lda = cl;
        g.B = ln().tmp; g.ldb = k;
        g.C = ln().theta; g.ldc = k;
        launch_gemm(g, ln().st);
      }
      DMRG2_CUDA(cudaMemcpyAsync(mps_[i - 1], ln().theta, sizeof(T) * (size_t)dims_[i - 1] * d_ * k,
                                 cudaMemcpyDeviceToDevice, ln().st));
      dims_[i] = k;
    }
    const ll n0 = (ll)d_ * dims_[1];
    norm2(mps_[0], n0, ln().dscal, ln().red, ln().st);
    scale_inplace(mps_[0], n0, ln().dscal, ln().st);
    canonical_ = true;
  }

  void build_right_envs() {
    T one = ST<T>::one();
    DMRG2_CUDA(cudaMemcpyAsync(lenv_[0], &one, sizeof(T), cudaMemcpyHostToDevice, ln().st));
    DMRG2_CUDA(cudaMemcpyAsync(renv_[L_], &one, sizeof(T), cudaMemcpyHostToDevice, ln().st));
    const int lowest = cfg_.single_site ? 1 : 2;  // single-site sweeps start with R[1]
    for (int i = L_ - 1; i >= lowest; --i)
      env_right(renv_[i + 1], mps_[i], wmr_[i], renv_[i], ln().X, ln().Y, dims_[i + 1], dims_[i], d_, Dl_[i],
                Dr_[i], ln().st);
  }

  SvdOut read_svd() {
    DMRG2_CUDA(cudaMemcpyAsync(ln().h_svd, ln().svdout, sizeof(SvdOut), cudaMemcpyDeviceToHost, ln().st));
    DMRG2_CUDA(cudaStreamSynchronize(ln().st));
    if (ln().h_svd->jacobi_err) throw std::runtime_error("Jacobi SVD barrier timed out");
    return *ln().h_svd;
  }

  // copies n elements of a bond's operator into a lane slot (on the lane's stream)
  const T* stage_op(T* slot, const T* src, ll n) {
    DMRG2_CUDA(cudaMemcpyAsync(slot, src, sizeof(T) * (size_t)n, cudaMemcpyDeviceToDevice, ln().st));
    return slot;
  }

  // ---------------------------------------------------------------- sweep
  double optimize_bond(int i, char dir, int chi, SweepStats& ss) {
    const int cL = dims_[i], cM = dims_[i + 1], cR = dims_[i + 2];
    const ll n = (ll)cL * d_ * d_ * cR;
    theta_form(mps_[i], mps_[i + 1], ln().theta, cL, cM, cR, d_, ln().st, ln().X, xs_);
    double e = lanczos(i, n, ss);
    svd_split(i, dir, chi, ss);
    if (dir == 'R')
      env_left(lenv_[i], mps_[i], wml_[i], lenv_[i + 1], ln().X, ln().Y, dims_[i], dims_[i + 1], d_, Dl_[i],
               Dr_[i], ln().st);
    else
      env_right(renv_[i + 2], mps_[i + 1], wmr_[i + 1], renv_[i + 1], ln().X, ln().Y, dims_[i + 2],
                dims_[i + 1], d_, Dl_[i + 1], Dr_[i + 1], ln().st);
    return e;
  }

  double lanczos(int i, ll n, SweepStats& ss) {
    const int cL = dims_[i], cR = dims_[i + 2];
    const int Dl = Db_[i], Dr = Db_[i + 2];
    const double fl = heff_flops(cL, cR, d_, Dl, Dr, ST<T>::cplx);
    const ll kk = (ll)Dl * d_ * d_ * d_ * d_ * Dr;  // entries of the dense fused MPO
    const bool sparse = wwt_sparse_[i] != 0;
    auto mv = [&](const T* in, T* out, const int* skip) {
      heff_apply(lenv_[i], renv_[i + 2], wwt_[i], in, out, ln().X, ln().Y, cL, cR, d_, Dl, Dr, skip, ln().st,
                 sparse ? wwt_[i] + kk : nullptr);
    };
    LanczosResult r;
    if (cfg_.precision == 1) {
      // precision form: converge on the split-BF16 operator (FP32-level accuracy), then
      // refine the Ritz vector with FP64 matvecs; the energy is the FP64 one. With graphs
      // both solves run device-looped on the staged operator (the split's scratch pointer
      // is part of the key: it moves when a larger shape grows it).
      const bool graph = cfg_.graphs && graphs_enabled();
      const ll dd = (ll)d_ * d_;
      const T* sL = graph ? stage_op(ln().opL, lenv_[i], (ll)cL * Dl * cL) : lenv_[i];
      const T* sR = graph ? stage_op(ln().opR, renv_[i + 2], (ll)cR * Dr * cR) : renv_[i + 2];
      const T* sW = graph ? stage_op(ln().opW, wwt_[i], wwt_block_elems(Dl * (int)dd, (int)dd * Dr, sizeof(T)))
                          : wwt_[i];
      auto mv_lp = [&](const T* in, T* out, const int* skip) {
        heff_apply_split(sL, sR, sW, in, out, ln().X, ln().Y, cL, cR, d_, Dl, Dr, ln().split, skip, ln().st);
      };
      auto mv_hp = [&](const T* in, T* out, const int* skip) {
        heff_apply(sL, sR, sW, in, out, ln().X, ln().Y, cL, cR, d_, Dl, Dr, skip, ln().st, sparse ? sW + kk : nullptr);
      };
      const LzKey key_lp{4, cL, cR, Dl, Dr, d_, (ll)sL, (ll)sR, (ll)sW, (ll)ln().X, (ll)ln().split.p};
      const LzKey key_hp{sparse ? 3 : 2, cL, cR, Dl, Dr, d_, (ll)sL, (ll)sR, (ll)sW, (ll)ln().X, (ll)ln().Y};
      LanczosResult lp = lanczos_solve<T>(ln().lw, ln().theta, n, cfg_.krylov_max, std::max(cfg_.lanczos_tol, 1e-9),
                                          cfg_.max_restarts, cfg_.seed + 7919u * (unsigned)i, mv_lp, ln().st,
                                          graph ? &key_lp : nullptr);
      r = lanczos_solve<T>(ln().lw, ln().theta, n, std::min(cfg_.krylov_max, 16), cfg_.lanczos_tol, 1,
                           cfg_.seed + 7919u * (unsigned)i + 1u, mv_hp, ln().st, graph ? &key_hp : nullptr);
      ss.lowprec_matvecs += lp.matvecs;
      r.matvecs += lp.matvecs;
      r.iters += lp.iters;
      r.matvec_s += lp.matvec_s;
    } else if (cfg_.graphs && graphs_enabled()) {
      // the device-looped solve: the bond's operator is staged into the lane's fixed slots,
      // so the cached graph of this shape serves it
      const ll dd = (ll)d_ * d_;
      const T *sL = stage_op(ln().opL, lenv_[i], (ll)cL * Dl * cL), *sR = stage_op(ln().opR, renv_[i + 2], (ll)cR * Dr * cR),
              *sW = stage_op(ln().opW, wwt_[i], wwt_block_elems(Dl * (int)dd, (int)dd * Dr, sizeof(T)));
      auto mvs = [&](const T* in, T* out, const int* skip) {
        heff_apply(sL, sR, sW, in, out, ln().X, ln().Y, cL, cR, d_, Dl, Dr, skip, ln().st, sparse ? sW + kk : nullptr);
      };
      const LzKey key{sparse ? 3 : 2, cL, cR, Dl, Dr, d_, (ll)sL, (ll)sR, (ll)sW, (ll)ln().X, (ll)ln().Y};
      r = lanczos_solve<T>(ln().lw, ln().theta, n, cfg_.krylov_max, cfg_.lanczos_tol, cfg_.max_restarts,
                           cfg_.seed + 7919u * (unsigned)i, mvs, ln().st, &key);
    } else {
      r = lanczos_solve<T>(ln().lw, ln().theta, n, cfg_.krylov_max, cfg_.lanczos_tol, cfg_.max_restarts,
                           cfg_.seed + 7919u * (unsigned)i, mv, ln().st);
    }
    ss.heff_s += r.matvec_s;
    ss.matvecs += r.matvecs;
    ss.heff_flops += fl * r.matvecs;
    ss.lanczos_iters += r.iters;
    ss.device_loops += r.device_loops;
    if (!r.converged) ss.lanczos_unconverged += 1;
    return r.energy;
  }

  // ---------------------------------------------------------------- single-site sweep
  // (reference: DMRGGPU::sweep_left_to_right / sweep_right_to_left, optimize_site and
  // svd_and_update_mps, gpu-rocm/dmrg-gpu/src/dmrg_gpu_impl.h:1119-1450): every site is
  // optimised with the one-site H_eff; left to right, A[i] = U and S Vh moves into A[i+1];
  // right to left, A[i] = Vh and U S moves into A[i-1]; the end sites are optimised
  // without a split. Bond dimensions can only stay or shrink.
  double sweep1(int chi, SweepStats& ss) {
    double e = 0.0;
    for (int i = 0; i + 1 < L_; ++i) {
      e = lanczos1(i, ss);
      split1(i, 'R', chi, ss);
      env_left(lenv_[i], mps_[i], wml_[i], lenv_[i + 1], ln().X, ln().Y, dims_[i], dims_[i + 1], d_, Dl_[i], Dr_[i], ln().st);
    }
    e = lanczos1(L_ - 1, ss);
    DMRG2_CUDA(cudaMemcpyAsync(mps_[L_ - 1], ln().theta, sizeof(T) * (size_t)dims_[L_ - 1] * d_ * dims_[L_],
                               cudaMemcpyDeviceToDevice, ln().st));
    for (int i = L_ - 1; i >= 1; --i) {
      e = lanczos1(i, ss);
      split1(i, 'L', chi, ss);
      env_right(renv_[i + 1], mps_[i], wmr_[i], renv_[i], ln().X, ln().Y, dims_[i + 1], dims_[i], d_, Dl_[i], Dr_[i], ln().st);
    }
    e = lanczos1(0, ss);
    DMRG2_CUDA(cudaMemcpyAsync(mps_[0], ln().theta, sizeof(T) * (size_t)dims_[0] * d_ * dims_[1],
                               cudaMemcpyDeviceToDevice, ln().st));
    return e;
  }

  double lanczos1(int i, SweepStats& ss) {
    const int cL = dims_[i], cR = dims_[i + 1];
    const int Dl = Db_[i], Dr = Db_[i + 1];
    const ll n = (ll)cL * d_ * cR;
    DMRG2_CUDA(cudaMemcpyAsync(ln().theta, mps_[i], sizeof(T) * (size_t)n, cudaMemcpyDeviceToDevice, ln().st));
    const bool graph = cfg_.graphs && graphs_enabled();  // staged operator, cached graph per shape
    const T* sL = graph ? stage_op(ln().opL, lenv_[i], (ll)cL * Dl * cL) : lenv_[i];
    const T* sR = graph ? stage_op(ln().opR, renv_[i + 1], (ll)cR * Dr * cR) : renv_[i + 1];
    const T* sW = graph ? stage_op(ln().opW, wml_[i], (ll)d_ * Dr * Dl * d_) : wml_[i];
    auto mv = [&](const T* in, T* out, const int* skip) {
      heff1_apply(sL, sR, sW, in, out, ln().X, ln().Y, cL, cR, d_, Dl, Dr, skip, ln().st);
    };
    const LzKey key{1, cL, cR, Dl, Dr, d_, (ll)sL, (ll)sR, (ll)sW, (ll)ln().X, (ll)ln().Y};
    LanczosResult r = lanczos_solve<T>(ln().lw, ln().theta, n, cfg_.krylov_max, cfg_.lanczos_tol, cfg_.max_restarts,
                                       cfg_.seed + 7919u * (unsigned)i, mv, ln().st, graph ? &key : nullptr);
    ss.heff_s += r.matvec_s;
    ss.matvecs += r.matvecs;
    ss.heff_flops += heff1_flops(cL, cR, d_, Dl, Dr, ST<T>::cplx) * r.matvecs;
    ss.lanczos_iters += r.iters;
    ss.device_loops += r.device_loops;
    if (!r.converged) ss.lanczos_unconverged += 1;
    return r.energy;
  }

  void split1(int i, char dir, int chi, SweepStats& ss) {
    const int cL = dims_[i], cR = dims_[i + 1];
    DMRG2_CUDA(cudaEventRecord(ln().ev_c, ln().st));
    SvdOut o;
    if (dir == 'R') {  // theta (cL d) x cR: A[i] = U, then A[i+1] <- (S Vh) A[i+1]
      o = eig_split(ln().ew, ln().theta, cL * d_, cR, 'R', chi, cfg_.cutoff, false, mps_[i], ln().tmp, ln().st);
      const int k = o.k, cR2 = dims_[i + 2];
      Gemm<T> g;
      g.M = k; g.N = d_ * cR2; g.K = cR;
      g.A = ln().tmp; g.lda = cR;
      g.B = mps_[i + 1]; g.ldb = (ll)d_ * cR2;
      g.C = ln().svdX; g.ldc = (ll)d_ * cR2;
      launch_gemm(g, ln().st);
      DMRG2_CUDA(cudaMemcpyAsync(mps_[i + 1], ln().svdX, sizeof(T) * (size_t)k * d_ * cR2, cudaMemcpyDeviceToDevice,
                                 ln().st));
      dims_[i + 1] = k;
    } else {  // theta cL x (d cR): A[i] = Vh, then A[i-1] <- A[i-1] (U S)
      o = eig_split(ln().ew, ln().theta, cL, d_ * cR, 'L', chi, cfg_.cutoff, false, ln().tmp, mps_[i], ln().st);
      const int k = o.k, cL2 = dims_[i - 1];
      Gemm<T> g;
      g.M = cL2 * d_; g.N = k; g.K = cL;
      g.A = mps_[i - 1]; g.lda = cL;
      g.B = ln().tmp; g.ldb = k;
      g.C = ln().svdX; g.ldc = k;
      launch_gemm(g, ln().st);
      DMRG2_CUDA(cudaMemcpyAsync(mps_[i - 1], ln().svdX, sizeof(T) * (size_t)cL2 * d_ * k, cudaMemcpyDeviceToDevice,
                                 ln().st));
      dims_[i] = k;
    }
    DMRG2_CUDA(cudaEventRecord(ln().ev_d, ln().st));
    DMRG2_CUDA(cudaEventSynchronize(ln().ev_d));
    float ms = 0.f;
    DMRG2_CUDA(cudaEventElapsedTime(&ms, ln().ev_c, ln().ev_d));
    ss.svd_s += ms * 1e-3;
    ss.trunc_err_max = std::max(ss.trunc_err_max, o.trunc_err);
    ss.trunc_err_sum += o.trunc_err;
  }

  void reset_split_history() {
    prev_sweep_chi_ = 0;
    te_ref_.assign((size_t)std::max(L_ - 1, 0), -1.0);
    short_age_.assign((size_t)std::max(L_ - 1, 0), 0);
  }

  // the warm-started split applies on a sweep that repeats the previous sweep's bond cap
  // (not in the first sweep at a new cap, where the state still moves far); it keeps the
  // bond's dimension k (the factor next to theta is an orthonormal basis of a
  // k-dimensional kept space)
  bool warm_split_applies(int i, int chi, ll m, ll nc) const {
    const int k = dims_[i + 1];
    const int kmax = ST<T>::cplx ? ln().wstc.kmax : ln().wst.kmax;  // 0 where the split is not built
    return prev_sweep_chi_ == chi && k <= chi && k <= kmax && std::min(m, nc) > k;
  }
  // |theta|^2 of the last warm split
  double warm_fro2() const { return ST<T>::cplx ? ln().wstc.h_buf[1] : ln().wst.h_buf[1]; }

  // A bond below the cap keeps its dimension only while the weight the warm split
  // discards could all lie below the exact split's threshold (cutoff^2, or the density
  // matrix's rounding floor 16 eps |theta|^2): otherwise some discarded Schmidt value
  // may be above it, the exact split would keep more states, and it runs instead (this
  // is how a bond dimension grows back).
  bool warm_split_keeps_rank(int k, int chi, ll m, ll nc, double te, double fro2) const {
    if (k >= chi) return true;
    const double thr = std::max(cfg_.cutoff * cfg_.cutoff, EIG_NOISE_FLOOR * fro2);
    return te <= (double)(std::min(m, nc) - k) * thr;
  }

  // One power half-step from the warm factor is kept when its discarded weight is within
  // WARM_SHORT_SLACK of the weight the last full split of this bond (three half-steps,
  // or the exact split) discarded, plus the rounding floor of |theta|^2 - |kept|^2; a
  // short split can therefore never discard more than that reference, which only full
  // splits set. At most WARM_SHORT_RUN short splits of a bond follow one full split.
  static constexpr double WARM_SHORT_SLACK = 1e-3;
  static constexpr int WARM_SHORT_RUN = 3;
  bool warm_short_accepts(int i, double te, double fro2) const {
    return te <= te_ref_[i] * (1.0 + WARM_SHORT_SLACK) + 64.0 * 2.220446049250313e-16 * fro2;
  }

  void svd_split(int i, char dir, int chi, SweepStats& ss) {
    const int cL = dims_[i], cR = dims_[i + 2];
    const ll m = (ll)cL * d_, nc = (ll)d_ * cR;
    DMRG2_CUDA(cudaEventRecord(ln().ev_c, ln().st));
    {
      if (warm_split_applies(i, chi, m, nc)) {
        double te = 0.0;
        const T* warm = (dir == 'R') ? mps_[i + 1] : mps_[i];
        const int k = dims_[i + 1];
        auto split = [&](WstMode mode) {
          bool done;
          if constexpr (ST<T>::cplx)
            done = wst_split_c(ln().wstc, ln().red, ln().theta, (int)m, (int)nc, dir, k, warm, mps_[i], mps_[i + 1], te,
                               ln().st, mode, ln().ev_d);
          else
            done = wst_split(ln().wst, ln().red, ln().theta, (int)m, (int)nc, dir, k, warm, mps_[i], mps_[i + 1], te,
                             ln().st, mode, cfg_.graphs, ln().ev_d);
          return done && warm_split_keeps_rank(k, chi, m, nc, te, warm_fro2());
        };
        bool ok = false, short_kept = false;
        if (te_ref_[i] >= 0.0 && short_age_[i] < WARM_SHORT_RUN) {
          if (split(WST_SHORT)) {
            const double te_short = te;
            short_kept = warm_short_accepts(i, te, warm_fro2());
            ok = short_kept;
            if (!short_kept || wst_debug()) {
              ok = split(WST_RESUME);  // the two remaining half-steps on the same theta
              if (wst_debug())
                std::fprintf(stderr, "[warm short] bond %d %c k=%d te_short=%.6e te_full=%.6e te_ref=%.6e kept=%d\n",
                             i, dir, k, te_short, te, te_ref_[i], (int)short_kept);
              short_kept = short_kept && !wst_debug();
            }
          }
        } else {
          ok = split(WST_FULL);
        }
        if (ok) {
          // ev_d was recorded by the last wst_split call, which waited for the stream
          float ms = 0.f;
          DMRG2_CUDA(cudaEventElapsedTime(&ms, ln().ev_c, ln().ev_d));
          ss.svd_s += ms * 1e-3;
          ss.warm_splits += 1;
          if (short_kept) {
            ss.warm_short += 1;
            short_age_[i] += 1;
          } else {
            te_ref_[i] = te;
            short_age_[i] = 0;
          }
          ss.trunc_err_max = std::max(ss.trunc_err_max, te);
          ss.trunc_err_sum += te;
          return;  // dims_[i + 1] unchanged
        }
        ss.warm_fallbacks += 1;
      }
    }
    if (ln().rsvd.rmax > 0 && rsvd_applies(ln().rsvd, (int)m, (int)nc, dir, chi)) {
      // randomised split (truncation mode 2): a fresh test matrix per call
      SvdOut o;
      const unsigned long long seed = ((unsigned long long)cfg_.seed << 32) ^ (unsigned long long)(++rsvd_calls_);
      bool ok = false;
      try {
        ok = rsvd_split(ln().rsvd, ln().ew, ln().red, ln().theta, (int)m, (int)nc, dir, chi, cfg_.cutoff, seed, mps_[i],
                        mps_[i + 1], o, ln().st);
      } catch (const NumericError&) {
        ok = false;  // the small split's eigenvectors: the exact split below decides
      }
      if (ok) {
        DMRG2_CUDA(cudaEventRecord(ln().ev_d, ln().st));
        DMRG2_CUDA(cudaEventSynchronize(ln().ev_d));
        float ms = 0.f;
        DMRG2_CUDA(cudaEventElapsedTime(&ms, ln().ev_c, ln().ev_d));
        ss.svd_s += ms * 1e-3;
        ss.rsvd_splits += 1;
        dims_[i + 1] = o.k;
        ss.trunc_err_max = std::max(ss.trunc_err_max, o.trunc_err);
        ss.trunc_err_sum += o.trunc_err;
        te_ref_[i] = o.trunc_err;
        short_age_[i] = 0;
        return;
      }
      ss.rsvd_fallbacks += 1;
    }
    SvdOut o;
    bool jacobi = (cfg_.svd_method == 1);
    if (!jacobi) {
      try {
        o = eig_split(ln().ew, ln().theta, (int)m, (int)nc, dir, chi, cfg_.cutoff, false, mps_[i], mps_[i + 1], ln().st);
        DMRG2_CUDA(cudaEventRecord(ln().ev_d, ln().st));
        DMRG2_CUDA(cudaEventSynchronize(ln().ev_d));
      } catch (const NumericError&) {
        // the eigenvectors of this density matrix could not be made orthonormal: split the
        // bond with the one-sided Jacobi SVD of theta instead (theta is unchanged)
        jacobi = true;
        ss.eig_fallbacks += 1;
      }
    }
    if (jacobi) {
      int nvec;
      ll len;
      if (dir == 'R') {
        nvec = (int)m;
        len = nc;
        DMRG2_CUDA(cudaMemcpyAsync(ln().svdX, ln().theta, sizeof(T) * m * nc, cudaMemcpyDeviceToDevice, ln().st));
      } else {
        nvec = (int)nc;
        len = m;
        transpose(ln().theta, ln().svdX, m, nc, ln().st);
      }
      set_identity(ln().svdQ, nvec, ln().st);
      svd_jacobi(ln().svdX, ln().svdQ, nvec, len, ln().jctl, cfg_.jacobi_max_sweeps, jacobi_tol(len), nullptr, ln().st);
      svd_sort_truncate(ln().svdX, nvec, len, ln().sigma, ln().perm, ln().svdout, chi, cfg_.cutoff, false, ln().jctl, ln().st);
      DMRG2_CUDA(cudaEventRecord(ln().ev_d, ln().st));
      o = read_svd();
      svd_gather(ln().svdX, ln().svdQ, ln().perm, nvec, len, o.k, dir == 'R' ? 0 : 1, mps_[i], mps_[i + 1], ln().st);
    }
    float ms = 0.f;
    DMRG2_CUDA(cudaEventElapsedTime(&ms, ln().ev_c, ln().ev_d));
    ss.svd_s += ms * 1e-3;
    ss.jacobi_sweeps_max = std::max(ss.jacobi_sweeps_max, o.jacobi_sweeps);
    dims_[i + 1] = o.k;
    ss.trunc_err_max = std::max(ss.trunc_err_max, o.trunc_err);
    ss.trunc_err_sum += o.trunc_err;
    te_ref_[i] = o.trunc_err;
    short_age_[i] = 0;
  }

  // ---------------------------------------------------------------- lanes
  // Scratch of one stream of bond work: a bond (theta, Lanczos, split, environment update)
  // runs on the lane its host thread selected (LaneScope), lane 0 by default. Segment
  // sweeps of the parallel sweep run on lanes 1..P concurrently; the bonds they touch are
  // disjoint.
  struct Lane {
    cudaStream_t st = nullptr;
    T *theta = nullptr, *X = nullptr, *Y = nullptr, *svdX = nullptr, *svdQ = nullptr, *tmp = nullptr;
    // the bond's operator (left and right environments, fused or single-site MPO) staged
    // into fixed slots, so one cached device-looped Lanczos graph serves every bond of a shape
    T *opL = nullptr, *opR = nullptr, *opW = nullptr;
    LanczosWork<T> lw;
    EigWork<T> ew;
    WstWork wst;     // warm-started subspace split (real data)
    WstWorkC wstc;   // the same for complex data
    RsvdWork<T> rsvd;  // randomised split (truncation mode 2)
    double* sigma = nullptr;
    int* perm = nullptr;
    SvdOut* svdout = nullptr;
    JacobiCtl* jctl = nullptr;
    double* dscal = nullptr;
    RedScratch red;
    SvdOut* h_svd = nullptr;
    SplitScratch split;  // BF16 pieces of the precision-form matvec
    cudaEvent_t ev_c = nullptr, ev_d = nullptr;
    std::vector<void*> owned;  // device buffers of lanes other than 0
  };
  Lane& ln() const {
    return (tl_lane_engine == this) ? *static_cast<Lane*>(tl_lane) : *lanes_[0];
  }
  // selects lane l for the bond work of the calling thread while in scope
  struct LaneScope {
    LaneScope(const void* eng, Lane* l) {
      tl_lane_engine = eng;
      tl_lane = l;
    }
    ~LaneScope() {
      tl_lane_engine = nullptr;
      tl_lane = nullptr;
    }
  };
  void init_lane(Lane& l, bool primary) {
    if (!l.st) DMRG2_CUDA(cudaStreamCreateWithFlags(&l.st, cudaStreamNonBlocking));
    auto al = [&](size_t b) -> void* {
      b = std::max<size_t>(b, sizeof(T));
      if (primary) return dalloc_bytes(b);
      void* p = nullptr;
      p = dev_alloc(b);
      l.owned.push_back(p);
      return p;
    };
    l.theta = (T*)al(sizeof(T) * (size_t)nmax_);
    l.svdX = (T*)al(sizeof(T) * (size_t)nmax_);
    l.svdQ = (T*)al(sizeof(T) * (size_t)(qmax_ * qmax_));
    l.tmp = (T*)al(sizeof(T) * (size_t)cfg_.chi_max * cfg_.chi_max);
    l.lw.init(cfg_.krylov_max, nmax_);
    l.ew.init((int)qmax_, cfg_.chi_max);
    if (primary) bytes_ += l.lw.bytes(nmax_) + l.ew.bytes;
    if (warm_capable(cfg_)) {
      if constexpr (ST<T>::cplx) {
        l.wstc.init((int)qmax_, cfg_.chi_max);
        if (primary) bytes_ += l.wstc.bytes;
      } else {
        l.wst.init((int)qmax_, cfg_.chi_max);
        if (primary) bytes_ += l.wst.bytes;
      }
    }
    if (rsvd_capable(cfg_)) {
      l.rsvd.init((int)qmax_, cfg_.chi_max + RSVD_OVERSAMPLE);
      if (primary) bytes_ += l.rsvd.bytes;
    }
    l.sigma = (double*)al(sizeof(double) * (size_t)qmax_);
    l.perm = (int*)al(sizeof(int) * (size_t)qmax_);
    l.svdout = (SvdOut*)al(sizeof(SvdOut));
    l.jctl = (JacobiCtl*)al(sizeof(JacobiCtl));
    l.dscal = (double*)al(sizeof(double) * 16);
    l.red.nblk = vec_blocks(nmax_);
    l.red.part = (double*)al(sizeof(double) * (size_t)l.red.nblk * 2 * (KRYLOV_CAP + 2));
    l.red.counter = (unsigned*)al(sizeof(unsigned) * 4);
    DMRG2_CUDA(cudaMemset(l.red.counter, 0, sizeof(unsigned) * 4));
    l.h_svd = (SvdOut*)host_pinned(sizeof(SvdOut));
    DMRG2_CUDA(cudaEventCreate(&l.ev_c));
    DMRG2_CUDA(cudaEventCreate(&l.ev_d));
    if (!primary && mpo_set_) {  // lane 0's X, Y are carved from the MPO slab
      l.X = (T*)al(sizeof(T) * (size_t)xs_);
      l.Y = (T*)al(sizeof(T) * (size_t)xs_);
      l.opL = (T*)al(sizeof(T) * (size_t)opn_);
      l.opR = (T*)al(sizeof(T) * (size_t)opn_);
      l.opW = (T*)al(sizeof(T) * (size_t)opw_);
    }
  }
  void release_lane(Lane& l) {
    if (l.st) cudaStreamSynchronize(l.st);
    l.split.release();
    l.lw.release();
    l.ew.release();
    l.wst.release();
    l.wstc.release();
    l.rsvd.release();
    for (void* p : l.owned) dev_free(p);
    l.owned.clear();
    if (l.h_svd) host_unpin(l.h_svd);
    l.h_svd = nullptr;
    if (l.ev_c) cudaEventDestroy(l.ev_c);
    if (l.ev_d) cudaEventDestroy(l.ev_d);
    l.ev_c = l.ev_d = nullptr;
    if (l.st) cudaStreamDestroy(l.st);
    l.st = nullptr;
  }

  // ---------------------------------------------------------------- state
  EngineConfig cfg_;
  int L_ = 0, d_ = 0;
  std::vector<int> cap_, dims_, Dl_, Dr_, Db_;
  std::vector<std::vector<T>> hW_;
  std::vector<T*> mps_, lenv_, renv_, wwt_, wml_, wmr_;
  std::vector<int> wwt_sparse_;  // bond uses the nonzero form of its fused MPO
  std::atomic<unsigned long long> rsvd_calls_{0};
  int prev_sweep_chi_ = 0;      // bond cap of the last completed sweep (0: none since the last set-up)
  std::vector<double> te_ref_;  // per bond: weight discarded by its last full split (< 0: none yet)
  std::vector<int> short_age_;  // per bond: short warm splits since that full split
  int* canon_flags_ = nullptr;
  int* h_flags_ = nullptr;
  cudaEvent_t ev_s0_ = nullptr, ev_s1_ = nullptr;
  std::vector<std::unique_ptr<Lane>> lanes_;  // lane 0: the engine's own stream and scratch
  bool envs_valid_ = false;
  std::vector<void*> allocs_, tmp_allocs_;
  void* mpo_slab_ = nullptr;  // every MPO-dependent buffer (mixing matrices, environments, scratch)
  size_t bytes_ = 0, bytes_mpo_ = 0;
  ll nmax_ = 0, qmax_ = 0;
  ll xs_ = 0;  // elements of each contraction scratch buffer ln().X, ln().Y
  ll opn_ = 0, opw_ = 0;  // elements of the staged operator slots (environments, MPO)
  bool mpo_set_ = false, mps_set_ = false, canonical_ = false;
  double energy_ = 0.0, env_build_s_ = 0.0;
};

size_t engine_footprint(const EngineConfig& c, const std::vector<int>& Dl, const std::vector<int>& Dr) {
  const int L = c.L, d = c.d;
  if (L < 2 || (int)Dl.size() != L || (int)Dr.size() != L) throw std::invalid_argument("footprint: bad shapes");
  const size_t sb = c.complex ? 16 : 8;
  const ll chi = c.chi_max;
  std::vector<ll> cap(L + 1);
  for (int i = 0; i <= L; ++i) cap[i] = ipow_cap(d, std::min(i, L - i), chi);
  auto el = [&](ll n) { return sb * (size_t)std::max<ll>(n, 1); };
  size_t b = 0;
  // constructor
  for (int i = 0; i < L; ++i) b += el(cap[i] * d * cap[i + 1]);
  ll nmax = 1, qmax = 1;
  for (int i = 0; i + 1 < L; ++i) {
    nmax = std::max(nmax, cap[i] * d * d * cap[i + 2]);
    qmax = std::max(qmax, std::max(cap[i] * d, (ll)d * cap[i + 2]));
  }
  for (int i = 0; i < L; ++i) qmax = std::max(qmax, (ll)d * cap[i + 1]);
  b += 2 * el(nmax) + el(qmax * qmax) + el(chi * chi);
  const int kcap = std::min(std::max(c.krylov_max, 2), KRYLOV_CAP);
  const ll nblk = vec_blocks(nmax);
  b += sb * ((size_t)kcap + 2) * (size_t)nmax + sizeof(LanczosDev) + sizeof(double) * (size_t)nblk * 2 * (KRYLOV_CAP + 2);
  {
    const size_t nn = (size_t)qmax, kk = (size_t)std::max<ll>(std::min<ll>(chi, qmax), 1);
    b += sb * nn * nn + 2 * sizeof(double) * nn + sb * nn + sizeof(double) * kk + 2 * sizeof(double) * nn * kk +
         sizeof(double) * kk * kk + sizeof(double) * 5 * nn * kk + sb * nn * kk + sb * 256 * (nn + 1) +
         sizeof(double) * 64 + sizeof(unsigned) * 4 + sizeof(SvdOut);
  }
  if (warm_capable(c)) b += c.complex ? wstc_bytes(qmax, chi) : wst_bytes(qmax, chi);
  if (rsvd_capable(c))
    b += c.complex ? RsvdWork<zc>::bytes_for(qmax, chi + RSVD_OVERSAMPLE)
                   : RsvdWork<double>::bytes_for(qmax, chi + RSVD_OVERSAMPLE);
  b += sizeof(double) * (size_t)qmax + sizeof(int) * (size_t)qmax + sizeof(SvdOut) + sizeof(JacobiCtl) +
       sizeof(double) * 16 + sizeof(double) * (size_t)nblk * 2 * (KRYLOV_CAP + 2) + sizeof(unsigned) * 4 +
       sizeof(int) * (size_t)(L + 1);
  // set_mpo
  for (int i = 0; i < L; ++i) b += 2 * el((ll)d * Dr[i] * Dl[i] * d);
  for (int i = 0; i + 1 < L; ++i) b += el(wwt_block_elems(Dl[i] * d * d, d * d * Dr[i + 1], sb));
  std::vector<ll> Db(L + 1, 1);
  for (int i = 0; i < L; ++i) Db[i] = Dl[i];
  Db[L] = Dr[L - 1];
  ll opn = 1, opw = 1;
  for (int i = 0; i <= L; ++i) {
    b += 2 * el(cap[i] * cap[i] * Db[i]);
    opn = std::max(opn, cap[i] * cap[i] * Db[i]);
  }
  for (int i = 0; i < L; ++i) opw = std::max(opw, (ll)d * Dr[i] * Dl[i] * d);
  for (int i = 0; i + 1 < L; ++i) opw = std::max(opw, wwt_block_elems(Dl[i] * d * d, d * d * Dr[i + 1], sb));
  b += 2 * el(opn) + el(opw);
  ll xs = 1;
  const ll dd = (ll)d * d;
  for (int i = 0; i + 1 < L; ++i) {
    xs = std::max(xs, cap[i] * Db[i] * dd * cap[i + 2]);
    xs = std::max(xs, cap[i] * dd * Db[i + 2] * cap[i + 2]);
  }
  for (int i = 0; i < L; ++i) {
    const ll a = cap[i], bb = cap[i + 1];
    xs = std::max(xs, a * Dl[i] * d * bb);
    xs = std::max(xs, a * d * Dr[i] * bb);
    xs = std::max(xs, bb * Dr[i] * d * a);
    xs = std::max(xs, (ll)d * bb * Dl[i] * a);
  }
  b += 2 * el(xs);
  return b;
}

std::unique_ptr<EngineBase> make_engine(const EngineConfig& cfg) {
  if (cfg.complex) return std::unique_ptr<EngineBase>(new Engine<zc>(cfg));
  return std::unique_ptr<EngineBase>(new Engine<double>(cfg));
}

}  // namespace dmrg2
