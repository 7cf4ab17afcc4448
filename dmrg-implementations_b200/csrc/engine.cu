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
#include <chrono>
#include <cstring>
#include <random>
#include <type_traits>

#include "contract.cuh"
#include "engine.h"
#include "lanczos_driver.cuh"
#include "rsvd.cuh"
#include "truncate.cuh"

namespace dmrg2 {

namespace {
// the warm-started subspace split is built for real data, the density-matrix route and
// bond caps of at most 512
bool warm_capable(const EngineConfig& c) {
  return !c.complex && c.truncation == 0 && c.svd_method == 0 && !c.single_site && c.chi_max <= CHOL_MAX;
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
    DMRG2_CUDA(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
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
      DMRG2_CUDA(cudaMalloc(&p, tot));
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
    theta_ = dalloc(nmax_);
    svdX_ = dalloc(nmax_);
    svdQ_ = dalloc(qmax_ * qmax_);
    tmp_ = dalloc((ll)cfg_.chi_max * cfg_.chi_max);
    lw_.init(cfg_.krylov_max, nmax_);
    bytes_ += lw_.bytes(nmax_);
    ew_.init((int)qmax_, cfg_.chi_max);
    bytes_ += ew_.bytes;
    if (warm_capable(cfg_)) {
      wst_.init((int)qmax_, cfg_.chi_max);
      bytes_ += wst_.bytes;
    }
    if (rsvd_capable(cfg_)) {
      rsvd_.init((int)qmax_, cfg_.chi_max + RSVD_OVERSAMPLE);
      bytes_ += rsvd_.bytes;
    }
    sigma_ = (double*)dalloc_bytes(sizeof(double) * qmax_);
    perm_ = (int*)dalloc_bytes(sizeof(int) * qmax_);
    svdout_ = (SvdOut*)dalloc_bytes(sizeof(SvdOut));
    jctl_ = (JacobiCtl*)dalloc_bytes(sizeof(JacobiCtl));
    dscal_ = (double*)dalloc_bytes(sizeof(double) * 16);
    red_.nblk = vec_blocks(nmax_);
    red_.part = (double*)dalloc_bytes(sizeof(double) * (size_t)red_.nblk * 2 * (KRYLOV_CAP + 2));
    red_.counter = (unsigned*)dalloc_bytes(sizeof(unsigned) * 4);
    DMRG2_CUDA(cudaMemset(red_.counter, 0, sizeof(unsigned) * 4));
    DMRG2_CUDA(cudaMallocHost(&h_svd_, sizeof(SvdOut)));
    canon_flags_ = (int*)dalloc_bytes(sizeof(int) * (size_t)(L_ + 1));
    DMRG2_CUDA(cudaMallocHost(&h_flags_, sizeof(int) * (size_t)(L_ + 1)));
    DMRG2_CUDA(cudaEventCreate(&ev_c_));
    DMRG2_CUDA(cudaEventCreate(&ev_d_));
    DMRG2_CUDA(cudaEventCreate(&ev_s0_));
    DMRG2_CUDA(cudaEventCreate(&ev_s1_));
  }

  ~Engine() override {
    cudaStreamSynchronize(st_);
    free_tmp();
    free_mpo();
    for (void* p : allocs_) cudaFree(p);
    cudaFreeHost(h_svd_);
    cudaFreeHost(h_flags_);
    split_.release();
    lw_.release();
    ew_.release();
    wst_.release();
    rsvd_.release();
    cudaEventDestroy(ev_c_);
    cudaEventDestroy(ev_d_);
    cudaEventDestroy(ev_s0_);
    cudaEventDestroy(ev_s1_);
    cudaStreamDestroy(st_);
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
    DMRG2_CUDA(cudaStreamSynchronize(st_));
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
    size_t total = up + 2 * round256(el(xs));
    for (int i = 0; i <= L_; ++i) total += 2 * round256(el((ll)cap_[i] * cap_[i] * Db_[i]));
    DMRG2_CUDA(cudaMalloc(&mpo_slab_, total));
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
    X_ = carve(xs);
    Y_ = carve(xs);
    xs_ = xs;
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
    DMRG2_CUDA(cudaStreamSynchronize(st_));
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
    DMRG2_CUDA(cudaStreamSynchronize(st_));
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
    DMRG2_CUDA(cudaStreamSynchronize(st_));
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

  std::vector<SweepStats> sweeps(const std::vector<int>& schedule, bool stop_rule) {
    std::vector<SweepStats> out;
    double e_prev = energy_;
    for (size_t sw = 0; sw < schedule.size(); ++sw) {
      SweepStats ss;
      ss.sweep = (int)sw;
      ss.chi_max = schedule[sw];
      auto ts = std::chrono::steady_clock::now();
      DMRG2_CUDA(cudaEventRecord(ev_s0_, st_));
      double e = 0.0;
      if (cfg_.single_site) {
        e = sweep1(schedule[sw], ss);
      } else {
        for (int i = 0; i + 1 < L_; ++i) e = optimize_bond(i, 'R', schedule[sw], ss);
        for (int i = L_ - 2; i >= 0; --i) e = optimize_bond(i, 'L', schedule[sw], ss);
      }
      DMRG2_CUDA(cudaEventRecord(ev_s1_, st_));
      DMRG2_CUDA(cudaStreamSynchronize(st_));
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
    DMRG2_CUDA(cudaMemcpyAsync(opd, op, sizeof(T) * d_ * d_, cudaMemcpyHostToDevice, st_));
    DMRG2_CUDA(cudaMemcpyAsync(idd, hid.data(), sizeof(T) * d_ * d_, cudaMemcpyHostToDevice, st_));
    T one = ST<T>::one();
    DMRG2_CUDA(cudaMemcpyAsync(E, &one, sizeof(T), cudaMemcpyHostToDevice, st_));
    for (int i = 0; i < L_; ++i) {
      int a = dims_[i], b = dims_[i + 1];
      env_left(E, mps_[i], opd, F, X_, Y_, a, b, d_, 1, 1, st_);
      trace_real(F, b, b, res + 2 * i, res + 2 * i + 1, st_);
      env_left(E, mps_[i], idd, E2, X_, Y_, a, b, d_, 1, 1, st_);
      if (i == 0) trace_real(E2, b, b, res + 2 * L_, res + 2 * L_ + 1, st_);
      std::swap(E, E2);
    }
    std::vector<double> h(2 * (L_ + 1));
    DMRG2_CUDA(cudaMemcpyAsync(h.data(), res, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, st_));
    DMRG2_CUDA(cudaStreamSynchronize(st_));
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
    DMRG2_CUDA(cudaMalloc(&p, b));
    allocs_.push_back(p);
    bytes_ += b;
    return p;
  }
  static size_t round256(size_t b) { return (b + 255) & ~(size_t)255; }
  T* dalloc_tmp(ll n) { return (T*)dalloc_tmp_bytes(sizeof(T) * (size_t)std::max<ll>(n, 1)); }
  void* dalloc_tmp_bytes(size_t b) {
    void* p = nullptr;
    DMRG2_CUDA(cudaMalloc(&p, b));
    tmp_allocs_.push_back(p);
    return p;
  }
  void free_tmp() {
    for (void* p : tmp_allocs_) cudaFree(p);
    tmp_allocs_.clear();
  }
  void free_mpo() {
    if (mpo_slab_) cudaFree(mpo_slab_);
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
      g.C = theta_; g.ldc = cl;
      launch_gemm(g, st_);
      identity_check(theta_, cl, 1e-12, canon_flags_ + i, st_);
    }
    DMRG2_CUDA(cudaMemcpyAsync(h_flags_, canon_flags_, sizeof(int) * (size_t)(L_ + 1), cudaMemcpyDeviceToHost, st_));
    DMRG2_CUDA(cudaStreamSynchronize(st_));
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
          SvdOut o = eig_split(ew_, mps_[i], cl, nc, 'L', chi, 1e-14, true, tmp_, mps_[i], st_);
          k = o.k;
          scale_inplace(tmp_, (ll)cl * k, &ew_.out->sigma_max2, st_);
        } catch (const NumericError&) {
          jacobi = true;  // eigenvectors not orthonormal: the Jacobi SVD splits this site
        }
      }
      if (jacobi) {
        transpose(mps_[i], svdX_, cl, nc, st_);
        norm2(svdX_, (ll)cl * nc, dscal_, red_, st_);
        set_identity(svdQ_, nc, st_);
        svd_jacobi(svdX_, svdQ_, nc, (ll)cl, jctl_, cfg_.jacobi_max_sweeps, jacobi_tol(cl), dscal_, st_);
        svd_sort_truncate(svdX_, nc, (ll)cl, sigma_, perm_, svdout_, chi, 1e-14, true, jctl_, st_);
        k = read_svd().k;
        svd_gather(svdX_, svdQ_, perm_, nc, (ll)cl, k, 1, tmp_, mps_[i], st_);
        scale_inplace(tmp_, (ll)cl * k, &svdout_->sigma_max2, st_);
      }
      {  // A[i-1] <- A[i-1] . (U S / sigma_max)
        Gemm<T> g;
        g.M = dims_[i - 1] * d_; g.N = k; g.K = cl;
        g.A = mps_[i - 1]; g.lda = cl;
        g.B = tmp_; g.ldb = k;
        g.C = theta_; g.ldc = k;
        launch_gemm(g, st_);
      }
      DMRG2_CUDA(cudaMemcpyAsync(mps_[i - 1], theta_, sizeof(T) * (size_t)dims_[i - 1] * d_ * k,
                                 cudaMemcpyDeviceToDevice, st_));
      dims_[i] = k;
    }
    const ll n0 = (ll)d_ * dims_[1];
    norm2(mps_[0], n0, dscal_, red_, st_);
    scale_inplace(mps_[0], n0, dscal_, st_);
    canonical_ = true;
  }

  void build_right_envs() {
    T one = ST<T>::one();
    DMRG2_CUDA(cudaMemcpyAsync(lenv_[0], &one, sizeof(T), cudaMemcpyHostToDevice, st_));
    DMRG2_CUDA(cudaMemcpyAsync(renv_[L_], &one, sizeof(T), cudaMemcpyHostToDevice, st_));
    const int lowest = cfg_.single_site ? 1 : 2;  // single-site sweeps start with R[1]
    for (int i = L_ - 1; i >= lowest; --i)
      env_right(renv_[i + 1], mps_[i], wmr_[i], renv_[i], X_, Y_, dims_[i + 1], dims_[i], d_, Dl_[i],
                Dr_[i], st_);
  }

  SvdOut read_svd() {
    DMRG2_CUDA(cudaMemcpyAsync(h_svd_, svdout_, sizeof(SvdOut), cudaMemcpyDeviceToHost, st_));
    DMRG2_CUDA(cudaStreamSynchronize(st_));
    if (h_svd_->jacobi_err) throw std::runtime_error("Jacobi SVD barrier timed out");
    return *h_svd_;
  }

  // ---------------------------------------------------------------- sweep
  double optimize_bond(int i, char dir, int chi, SweepStats& ss) {
    const int cL = dims_[i], cM = dims_[i + 1], cR = dims_[i + 2];
    const ll n = (ll)cL * d_ * d_ * cR;
    theta_form(mps_[i], mps_[i + 1], theta_, cL, cM, cR, d_, st_, X_, xs_);
    double e = lanczos(i, n, ss);
    svd_split(i, dir, chi, ss);
    if (dir == 'R')
      env_left(lenv_[i], mps_[i], wml_[i], lenv_[i + 1], X_, Y_, dims_[i], dims_[i + 1], d_, Dl_[i],
               Dr_[i], st_);
    else
      env_right(renv_[i + 2], mps_[i + 1], wmr_[i + 1], renv_[i + 1], X_, Y_, dims_[i + 2],
                dims_[i + 1], d_, Dl_[i + 1], Dr_[i + 1], st_);
    return e;
  }

  double lanczos(int i, ll n, SweepStats& ss) {
    const int cL = dims_[i], cR = dims_[i + 2];
    const int Dl = Db_[i], Dr = Db_[i + 2];
    const double fl = heff_flops(cL, cR, d_, Dl, Dr, ST<T>::cplx);
    auto mv = [&](const T* in, T* out, const int* skip) {
      heff_apply(lenv_[i], renv_[i + 2], wwt_[i], in, out, X_, Y_, cL, cR, d_, Dl, Dr, skip, st_);
    };
    LanczosResult r;
    if (cfg_.precision == 1) {
      // precision form: converge on the split-BF16 operator (FP32-level accuracy), then
      // refine the Ritz vector with FP64 matvecs; the energy is the FP64 one
      auto mv_lp = [&](const T* in, T* out, const int* skip) {
        heff_apply_split(lenv_[i], renv_[i + 2], wwt_[i], in, out, X_, Y_, cL, cR, d_, Dl, Dr, split_, skip, st_);
      };
      LanczosResult lp = lanczos_solve<T>(lw_, theta_, n, cfg_.krylov_max, std::max(cfg_.lanczos_tol, 1e-9),
                                          cfg_.max_restarts, cfg_.seed + 7919u * (unsigned)i, mv_lp, st_);
      r = lanczos_solve<T>(lw_, theta_, n, std::min(cfg_.krylov_max, 16), cfg_.lanczos_tol, 1,
                           cfg_.seed + 7919u * (unsigned)i + 1u, mv, st_);
      ss.lowprec_matvecs += lp.matvecs;
      r.matvecs += lp.matvecs;
      r.iters += lp.iters;
      r.matvec_s += lp.matvec_s;
    } else {
      r = lanczos_solve<T>(lw_, theta_, n, cfg_.krylov_max, cfg_.lanczos_tol, cfg_.max_restarts,
                           cfg_.seed + 7919u * (unsigned)i, mv, st_);
    }
    ss.heff_s += r.matvec_s;
    ss.matvecs += r.matvecs;
    ss.heff_flops += fl * r.matvecs;
    ss.lanczos_iters += r.iters;
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
      env_left(lenv_[i], mps_[i], wml_[i], lenv_[i + 1], X_, Y_, dims_[i], dims_[i + 1], d_, Dl_[i], Dr_[i], st_);
    }
    e = lanczos1(L_ - 1, ss);
    DMRG2_CUDA(cudaMemcpyAsync(mps_[L_ - 1], theta_, sizeof(T) * (size_t)dims_[L_ - 1] * d_ * dims_[L_],
                               cudaMemcpyDeviceToDevice, st_));
    for (int i = L_ - 1; i >= 1; --i) {
      e = lanczos1(i, ss);
      split1(i, 'L', chi, ss);
      env_right(renv_[i + 1], mps_[i], wmr_[i], renv_[i], X_, Y_, dims_[i + 1], dims_[i], d_, Dl_[i], Dr_[i], st_);
    }
    e = lanczos1(0, ss);
    DMRG2_CUDA(cudaMemcpyAsync(mps_[0], theta_, sizeof(T) * (size_t)dims_[0] * d_ * dims_[1],
                               cudaMemcpyDeviceToDevice, st_));
    return e;
  }

  double lanczos1(int i, SweepStats& ss) {
    const int cL = dims_[i], cR = dims_[i + 1];
    const int Dl = Db_[i], Dr = Db_[i + 1];
    const ll n = (ll)cL * d_ * cR;
    DMRG2_CUDA(cudaMemcpyAsync(theta_, mps_[i], sizeof(T) * (size_t)n, cudaMemcpyDeviceToDevice, st_));
    auto mv = [&](const T* in, T* out, const int* skip) {
      heff1_apply(lenv_[i], renv_[i + 1], wml_[i], in, out, X_, Y_, cL, cR, d_, Dl, Dr, skip, st_);
    };
    LanczosResult r = lanczos_solve<T>(lw_, theta_, n, cfg_.krylov_max, cfg_.lanczos_tol, cfg_.max_restarts,
                                       cfg_.seed + 7919u * (unsigned)i, mv, st_);
    ss.heff_s += r.matvec_s;
    ss.matvecs += r.matvecs;
    ss.heff_flops += heff1_flops(cL, cR, d_, Dl, Dr, ST<T>::cplx) * r.matvecs;
    ss.lanczos_iters += r.iters;
    if (!r.converged) ss.lanczos_unconverged += 1;
    return r.energy;
  }

  void split1(int i, char dir, int chi, SweepStats& ss) {
    const int cL = dims_[i], cR = dims_[i + 1];
    DMRG2_CUDA(cudaEventRecord(ev_c_, st_));
    SvdOut o;
    if (dir == 'R') {  // theta (cL d) x cR: A[i] = U, then A[i+1] <- (S Vh) A[i+1]
      o = eig_split(ew_, theta_, cL * d_, cR, 'R', chi, cfg_.cutoff, false, mps_[i], tmp_, st_);
      const int k = o.k, cR2 = dims_[i + 2];
      Gemm<T> g;
      g.M = k; g.N = d_ * cR2; g.K = cR;
      g.A = tmp_; g.lda = cR;
      g.B = mps_[i + 1]; g.ldb = (ll)d_ * cR2;
      g.C = svdX_; g.ldc = (ll)d_ * cR2;
      launch_gemm(g, st_);
      DMRG2_CUDA(cudaMemcpyAsync(mps_[i + 1], svdX_, sizeof(T) * (size_t)k * d_ * cR2, cudaMemcpyDeviceToDevice,
                                 st_));
      dims_[i + 1] = k;
    } else {  // theta cL x (d cR): A[i] = Vh, then A[i-1] <- A[i-1] (U S)
      o = eig_split(ew_, theta_, cL, d_ * cR, 'L', chi, cfg_.cutoff, false, tmp_, mps_[i], st_);
      const int k = o.k, cL2 = dims_[i - 1];
      Gemm<T> g;
      g.M = cL2 * d_; g.N = k; g.K = cL;
      g.A = mps_[i - 1]; g.lda = cL;
      g.B = tmp_; g.ldb = k;
      g.C = svdX_; g.ldc = k;
      launch_gemm(g, st_);
      DMRG2_CUDA(cudaMemcpyAsync(mps_[i - 1], svdX_, sizeof(T) * (size_t)cL2 * d_ * k, cudaMemcpyDeviceToDevice,
                                 st_));
      dims_[i] = k;
    }
    DMRG2_CUDA(cudaEventRecord(ev_d_, st_));
    DMRG2_CUDA(cudaEventSynchronize(ev_d_));
    float ms = 0.f;
    DMRG2_CUDA(cudaEventElapsedTime(&ms, ev_c_, ev_d_));
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
    return prev_sweep_chi_ == chi && k <= chi && k <= wst_.kmax && std::min(m, nc) > k;
  }

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
    DMRG2_CUDA(cudaEventRecord(ev_c_, st_));
    if constexpr (std::is_same<T, double>::value) {
      if (warm_split_applies(i, chi, m, nc)) {
        double te = 0.0;
        const double* warm = (dir == 'R') ? mps_[i + 1] : mps_[i];
        const int k = dims_[i + 1];
        auto split = [&](WstMode mode) {
          return wst_split(wst_, red_, theta_, (int)m, (int)nc, dir, k, warm, mps_[i], mps_[i + 1], te, st_, mode) &&
                 warm_split_keeps_rank(k, chi, m, nc, te, wst_.h_buf[1]);
        };
        bool ok = false, short_kept = false;
        if (te_ref_[i] >= 0.0 && short_age_[i] < WARM_SHORT_RUN) {
          if (split(WST_SHORT)) {
            const double te_short = te;
            short_kept = warm_short_accepts(i, te, wst_.h_buf[1]);
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
          DMRG2_CUDA(cudaEventRecord(ev_d_, st_));
          DMRG2_CUDA(cudaEventSynchronize(ev_d_));
          float ms = 0.f;
          DMRG2_CUDA(cudaEventElapsedTime(&ms, ev_c_, ev_d_));
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
    if (rsvd_.rmax > 0 && rsvd_applies(rsvd_, (int)m, (int)nc, dir, chi)) {
      // randomised split (truncation mode 2): a fresh test matrix per call
      SvdOut o;
      const unsigned long long seed = ((unsigned long long)cfg_.seed << 32) ^ (unsigned long long)(++rsvd_calls_);
      bool ok = false;
      try {
        ok = rsvd_split(rsvd_, ew_, red_, theta_, (int)m, (int)nc, dir, chi, cfg_.cutoff, seed, mps_[i],
                        mps_[i + 1], o, st_);
      } catch (const NumericError&) {
        ok = false;  // the small split's eigenvectors: the exact split below decides
      }
      if (ok) {
        DMRG2_CUDA(cudaEventRecord(ev_d_, st_));
        DMRG2_CUDA(cudaEventSynchronize(ev_d_));
        float ms = 0.f;
        DMRG2_CUDA(cudaEventElapsedTime(&ms, ev_c_, ev_d_));
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
        o = eig_split(ew_, theta_, (int)m, (int)nc, dir, chi, cfg_.cutoff, false, mps_[i], mps_[i + 1], st_);
        DMRG2_CUDA(cudaEventRecord(ev_d_, st_));
        DMRG2_CUDA(cudaEventSynchronize(ev_d_));
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
        DMRG2_CUDA(cudaMemcpyAsync(svdX_, theta_, sizeof(T) * m * nc, cudaMemcpyDeviceToDevice, st_));
      } else {
        nvec = (int)nc;
        len = m;
        transpose(theta_, svdX_, m, nc, st_);
      }
      set_identity(svdQ_, nvec, st_);
      svd_jacobi(svdX_, svdQ_, nvec, len, jctl_, cfg_.jacobi_max_sweeps, jacobi_tol(len), nullptr, st_);
      svd_sort_truncate(svdX_, nvec, len, sigma_, perm_, svdout_, chi, cfg_.cutoff, false, jctl_, st_);
      DMRG2_CUDA(cudaEventRecord(ev_d_, st_));
      o = read_svd();
      svd_gather(svdX_, svdQ_, perm_, nvec, len, o.k, dir == 'R' ? 0 : 1, mps_[i], mps_[i + 1], st_);
    }
    float ms = 0.f;
    DMRG2_CUDA(cudaEventElapsedTime(&ms, ev_c_, ev_d_));
    ss.svd_s += ms * 1e-3;
    ss.jacobi_sweeps_max = std::max(ss.jacobi_sweeps_max, o.jacobi_sweeps);
    dims_[i + 1] = o.k;
    ss.trunc_err_max = std::max(ss.trunc_err_max, o.trunc_err);
    ss.trunc_err_sum += o.trunc_err;
    te_ref_[i] = o.trunc_err;
    short_age_[i] = 0;
  }

  // ---------------------------------------------------------------- state
  EngineConfig cfg_;
  int L_ = 0, d_ = 0;
  cudaStream_t st_ = nullptr;
  std::vector<int> cap_, dims_, Dl_, Dr_, Db_;
  std::vector<std::vector<T>> hW_;
  std::vector<T*> mps_, lenv_, renv_, wwt_, wml_, wmr_;
  T *theta_ = nullptr, *X_ = nullptr, *Y_ = nullptr, *svdX_ = nullptr,
    *svdQ_ = nullptr, *tmp_ = nullptr;
  LanczosWork<T> lw_;
  EigWork<T> ew_;
  WstWork wst_;                 // warm-started subspace split (real data)
  RsvdWork<T> rsvd_;            // randomised split (truncation mode 2)
  unsigned long long rsvd_calls_ = 0;
  int prev_sweep_chi_ = 0;      // bond cap of the last completed sweep (0: none since the last set-up)
  std::vector<double> te_ref_;  // per bond: weight discarded by its last full split (< 0: none yet)
  std::vector<int> short_age_;  // per bond: short warm splits since that full split
  double* sigma_ = nullptr;
  int* perm_ = nullptr;
  SvdOut* svdout_ = nullptr;
  JacobiCtl* jctl_ = nullptr;
  double* dscal_ = nullptr;
  RedScratch red_;
  SvdOut* h_svd_ = nullptr;
  SplitScratch split_;  // BF16 pieces of the precision-form matvec
  int* canon_flags_ = nullptr;
  int* h_flags_ = nullptr;
  cudaEvent_t ev_c_ = nullptr, ev_d_ = nullptr, ev_s0_ = nullptr, ev_s1_ = nullptr;
  bool envs_valid_ = false;
  std::vector<void*> allocs_, tmp_allocs_;
  void* mpo_slab_ = nullptr;  // every MPO-dependent buffer (mixing matrices, environments, scratch)
  size_t bytes_ = 0, bytes_mpo_ = 0;
  ll nmax_ = 0, qmax_ = 0;
  ll xs_ = 0;  // elements of each contraction scratch buffer X_, Y_
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
  b += sb * ((size_t)kcap + 1) * (size_t)nmax + sizeof(LanczosDev) + sizeof(double) * (size_t)nblk * 2 * (KRYLOV_CAP + 2);
  {
    const size_t nn = (size_t)qmax, kk = (size_t)std::max<ll>(std::min<ll>(chi, qmax), 1);
    b += sb * nn * nn + 2 * sizeof(double) * nn + sb * nn + sizeof(double) * kk + 2 * sizeof(double) * nn * kk +
         sizeof(double) * kk * kk + sizeof(double) * 5 * nn * kk + sb * nn * kk + sb * 256 * (nn + 1) +
         sizeof(double) * 64 + sizeof(unsigned) * 4 + sizeof(SvdOut);
  }
  if (warm_capable(c)) b += wst_bytes(qmax, chi);
  if (rsvd_capable(c))
    b += c.complex ? RsvdWork<zc>::bytes_for(qmax, chi + RSVD_OVERSAMPLE)
                   : RsvdWork<double>::bytes_for(qmax, chi + RSVD_OVERSAMPLE);
  b += sizeof(double) * (size_t)qmax + sizeof(int) * (size_t)qmax + sizeof(SvdOut) + sizeof(JacobiCtl) +
       sizeof(double) * 16 + sizeof(double) * (size_t)nblk * 2 * (KRYLOV_CAP + 2) + sizeof(unsigned) * 4 +
       sizeof(int) * (size_t)(L + 1);
  // set_mpo
  for (int i = 0; i < L; ++i) b += 2 * el((ll)d * Dr[i] * Dl[i] * d);
  for (int i = 0; i + 1 < L; ++i) b += el((ll)d * d * Dr[i + 1] * Dl[i] * d * d);
  std::vector<ll> Db(L + 1, 1);
  for (int i = 0; i < L; ++i) Db[i] = Dl[i];
  Db[L] = Dr[L - 1];
  for (int i = 0; i <= L; ++i) b += 2 * el(cap[i] * cap[i] * Db[i]);
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
