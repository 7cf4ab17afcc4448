// extern "C" boundary of the engine (declared in include/dmrg2_b200.h).
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <functional>
#include <map>
#include <mutex>
#include <thread>
#include <memory>
#include <random>
#include <string>
#include <vector>

#include "../../include/dmrg2_b200.h"
#include "contract.cuh"
#include "engine.h"
#include "kernels.cuh"
#include "lanczos_driver.cuh"
#include "noalloc.cuh"
#include "truncate.cuh"
#include "umma.cuh"

using namespace dmrg2;

struct dmrg2_handle {
  std::unique_ptr<EngineBase> eng;
  EngineConfig cfg;
  int dtype = DMRG2_F64;
  std::string err;
};

namespace {

thread_local std::string g_err;

size_t scalar_bytes(int dtype) { return dtype == DMRG2_C128 ? 16 : 8; }

template <typename F>
int guarded(dmrg2_handle* h, F&& f) {
  try {
    f();
    return DMRG2_OK;
  } catch (const CudaError& e) {
    (h ? h->err : g_err) = e.what();
    (void)cudaGetLastError();  // clear a non-sticky error so the next call starts clean
    return DMRG2_ERR_CUDA;
  } catch (const NumericError& e) {
    (h ? h->err : g_err) = e.what();
    return DMRG2_ERR_NUMERIC;
  } catch (const std::invalid_argument& e) {
    (h ? h->err : g_err) = e.what();
    return DMRG2_ERR_ARG;
  } catch (const std::logic_error& e) {
    (h ? h->err : g_err) = e.what();
    return DMRG2_ERR_STATE;
  } catch (const std::runtime_error& e) {
    std::string m = e.what();
    (h ? h->err : g_err) = m;
    if (m.find("timed out") != std::string::npos || m.find("terminate") != std::string::npos)
      return DMRG2_ERR_NUMERIC;
    return DMRG2_ERR_ARG;
  } catch (const std::exception& e) {
    (h ? h->err : g_err) = e.what();
    return DMRG2_ERR_INTERNAL;
  }
}

struct DBuf {
  void* p = nullptr;
  DBuf() = default;
  explicit DBuf(size_t b) { p = dev_alloc(b ? b : 16); }
  DBuf(const void* host, size_t b) : DBuf(b) {
    if (host && b) DMRG2_CUDA(cudaMemcpy(p, host, b, cudaMemcpyHostToDevice));
  }
  ~DBuf() {
    if (p) dev_free(p);
  }
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  template <typename T>
  T* as() const { return (T*)p; }
};

// reference column-major MPS  ->  row-major (a, s, b)
void mps_ref_to_row(const char* src, char* dst, int cl, int d, int cr, size_t sb) {
  for (int a = 0; a < cl; ++a)
    for (int s = 0; s < d; ++s)
      for (int b = 0; b < cr; ++b)
        std::memcpy(dst + (((size_t)a * d + s) * cr + b) * sb,
                    src + ((size_t)a + (size_t)s * cl + (size_t)b * cl * d) * sb, sb);
}
void mps_row_to_ref(const char* src, char* dst, int cl, int d, int cr, size_t sb) {
  for (int a = 0; a < cl; ++a)
    for (int s = 0; s < d; ++s)
      for (int b = 0; b < cr; ++b)
        std::memcpy(dst + ((size_t)a + (size_t)s * cl + (size_t)b * cl * d) * sb,
                    src + (((size_t)a * d + s) * cr + b) * sb, sb);
}

std::vector<int> reference_bond_dims(int L, int d, int chi) {
  std::vector<int> b(L + 1, 1);
  for (int i = 1; i < L; ++i) {
    long long v = 1;
    for (int k = 0; k < std::min(i, L - i) && v < chi; ++k) v *= d;
    b[i] = (int)std::min<long long>(v, chi);
  }
  return b;
}

template <typename T>
void do_op_heff(int cL, int cR, int d, int Dl, int Dm, int Dr, const void* L, const void* R,
                const void* WL, const void* WR, const void* theta, void* out) {
  const size_t sb = sizeof(T);
  const ll dd = (ll)d * d;
  std::vector<T> wwt;
  build_wwt((const T*)WL, (const T*)WR, Dl, Dm, Dr, d, wwt);
  const ll n = (ll)cL * dd * cR;
  DBuf dL(L, sb * cL * Dl * cL), dR(R, sb * cR * Dr * cR), dW(wwt.data(), sb * wwt.size());
  DBuf din(theta, sb * n), dout(sb * n);
  const ll xs = std::max((ll)cL * Dl * dd * cR, (ll)cL * dd * Dr * cR);
  DBuf X(sb * xs), Y(sb * xs);
  heff_apply(dL.as<T>(), dR.as<T>(), dW.as<T>(), din.as<T>(), dout.as<T>(), X.as<T>(), Y.as<T>(),
             cL, cR, d, Dl, Dr, nullptr, 0);
  DMRG2_CUDA(cudaMemcpy(out, dout.p, sb * n, cudaMemcpyDeviceToHost));
}

template <typename T>
void do_op_env_left(int cL, int cO, int d, int Dl, int Dr, const void* L, const void* A,
                    const void* W, void* out) {
  const size_t sb = sizeof(T);
  std::vector<T> wm;
  build_wmix_left((const T*)W, Dl, Dr, d, wm);
  DBuf dL(L, sb * cL * Dl * cL), dA(A, sb * cL * d * cO), dW(wm.data(), sb * wm.size());
  DBuf dout(sb * cO * Dr * cO);
  const ll xs = std::max((ll)cL * Dl * d * cO, (ll)cL * d * Dr * cO);
  DBuf X(sb * xs), Y(sb * xs);
  env_left(dL.as<T>(), dA.as<T>(), dW.as<T>(), dout.as<T>(), X.as<T>(), Y.as<T>(), cL, cO, d, Dl,
           Dr, 0);
  DMRG2_CUDA(cudaMemcpy(out, dout.p, sb * cO * Dr * cO, cudaMemcpyDeviceToHost));
}

template <typename T>
void do_op_env_right(int cI, int cO, int d, int Dl, int Dr, const void* R, const void* B,
                     const void* W, void* out) {
  const size_t sb = sizeof(T);
  std::vector<T> wm;
  build_wmix_right((const T*)W, Dl, Dr, d, wm);
  DBuf dR(R, sb * cI * Dr * cI), dB(B, sb * cO * d * cI), dW(wm.data(), sb * wm.size());
  DBuf dout(sb * cO * Dl * cO);
  const ll xs = std::max((ll)cI * Dr * d * cO, (ll)d * cI * Dl * cO);
  DBuf X(sb * xs), Y(sb * xs);
  env_right(dR.as<T>(), dB.as<T>(), dW.as<T>(), dout.as<T>(), X.as<T>(), Y.as<T>(), cI, cO, d, Dl,
            Dr, 0);
  DMRG2_CUDA(cudaMemcpy(out, dout.p, sb * cO * Dl * cO, cudaMemcpyDeviceToHost));
}

template <typename T>
void do_op_svd_eig(int m, int n, const void* M, int max_bond, double cutoff, char dir, double* S,
                   void* left, void* right, int* k_out, double* te_out) {
  const size_t sb = sizeof(T);
  const bool R = (dir == 'R');
  const int nn = R ? m : n;
  const int kmin = std::min(m, n);
  DBuf dM(M, sb * (size_t)m * n), dl(sb * (size_t)m * kmin), dr(sb * (size_t)kmin * n);
  EigWork<T> W;
  std::vector<double> lam(nn);
  try {
    W.init(nn, nn);
    SvdOut o = eig_split<T>(W, dM.as<T>(), m, n, R ? 'R' : 'L', std::min(max_bond, kmin), cutoff,
                            false, dl.as<T>(), dr.as<T>(), 0, nn, lam.data());
    const int k = o.k;
    if (S)
      for (int r = 0; r < kmin; ++r) S[r] = std::sqrt(std::max(lam[r], 0.0));
    if (left) DMRG2_CUDA(cudaMemcpy(left, dl.p, sb * (size_t)m * k, cudaMemcpyDeviceToHost));
    if (right) DMRG2_CUDA(cudaMemcpy(right, dr.p, sb * (size_t)k * n, cudaMemcpyDeviceToHost));
    if (k_out) *k_out = k;
    if (te_out) *te_out = o.trunc_err;
  } catch (...) {
    W.release();
    throw;
  }
  W.release();
}

// warm-started split of M (m x n) at rank k from the orthonormal factor `warm`
// (dir 'R': k x n rows, dir 'L': m x k columns); false when CholeskyQR gave up
bool do_op_warm_split(int m, int n, const void* M, const void* warm, int k, char dir, void* left, void* right,
                      double* te_out) {
  const size_t sb = sizeof(double);
  const bool R = (dir == 'R');
  DBuf dM(M, sb * (size_t)m * n), dw(warm, sb * (size_t)(R ? (size_t)k * n : (size_t)m * k));
  DBuf dl(sb * (size_t)m * k), dr(sb * (size_t)k * n);
  RedScratch red;
  DBuf part(sizeof(double) * 2400), cnt(sizeof(unsigned) * 4);
  red.part = part.as<double>();
  red.counter = cnt.as<unsigned>();
  red.nblk = 1184;
  DMRG2_CUDA(cudaMemset(cnt.p, 0, sizeof(unsigned) * 4));
  WstWork W;
  bool ok = false;
  double te = 0.0;
  try {
    W.init(std::max(m, n), k);
    ok = wst_split(W, red, dM.as<double>(), m, n, dir, k, dw.as<double>(), dl.as<double>(), dr.as<double>(), te, 0);
    if (ok) {
      if (left) DMRG2_CUDA(cudaMemcpy(left, dl.p, sb * (size_t)m * k, cudaMemcpyDeviceToHost));
      if (right) DMRG2_CUDA(cudaMemcpy(right, dr.p, sb * (size_t)k * n, cudaMemcpyDeviceToHost));
      if (te_out) *te_out = te;
    }
  } catch (...) {
    W.release();
    throw;
  }
  W.release();
  return ok;
}

template <typename T>
void do_op_svd(int m, int n, const void* M, int max_bond, double cutoff, char dir, double* S,
               void* left, void* right, int* k_out, double* te_out) {
  const size_t sb = sizeof(T);
  const ll mn = (ll)m * n;
  const bool R = (dir == 'R' || dir == 'r');
  const int nvec = R ? m : n;
  const ll len = R ? n : m;
  DBuf dM(M, sb * mn), X(sb * mn), Q(sb * (size_t)nvec * nvec), sig(sizeof(double) * nvec),
      perm(sizeof(int) * nvec), out(sizeof(SvdOut)), ctl(sizeof(JacobiCtl)), fro(sizeof(double) * 2);
  RedScratch red;
  DBuf part(sizeof(double) * 1200), cnt(sizeof(unsigned) * 4);
  red.part = part.as<double>();
  red.counter = cnt.as<unsigned>();
  red.nblk = 1184;
  DMRG2_CUDA(cudaMemset(cnt.p, 0, sizeof(unsigned) * 4));
  if (R) DMRG2_CUDA(cudaMemcpy(X.p, dM.p, sb * mn, cudaMemcpyDeviceToDevice));
  else transpose(dM.as<T>(), X.as<T>(), m, n, 0);
  norm2(X.as<T>(), mn, fro.as<double>(), red, 0);
  set_identity(Q.as<T>(), nvec, 0);
  double tol = 2.2e-16 * std::max<double>(16.0, (double)len);
  svd_jacobi(X.as<T>(), Q.as<T>(), nvec, len, ctl.as<JacobiCtl>(), 40, tol, fro.as<double>(), 0);
  svd_sort_truncate(X.as<T>(), nvec, len, sig.as<double>(), perm.as<int>(), out.as<SvdOut>(),
                    max_bond, cutoff, false, ctl.as<JacobiCtl>(), 0);
  SvdOut o;
  DMRG2_CUDA(cudaMemcpy(&o, out.p, sizeof(SvdOut), cudaMemcpyDeviceToHost));
  if (o.jacobi_err) throw std::runtime_error("Jacobi SVD barrier timed out");
  const int k = o.k;
  DBuf dl(sb * (size_t)m * k), dr(sb * (size_t)k * n);
  svd_gather(X.as<T>(), Q.as<T>(), perm.as<int>(), nvec, len, k, R ? 0 : 1, dl.as<T>(),
             dr.as<T>(), 0);
  std::vector<double> hs(nvec);
  std::vector<int> hp(nvec);
  DMRG2_CUDA(cudaMemcpy(hs.data(), sig.p, sizeof(double) * nvec, cudaMemcpyDeviceToHost));
  DMRG2_CUDA(cudaMemcpy(hp.data(), perm.p, sizeof(int) * nvec, cudaMemcpyDeviceToHost));
  const int kmin = std::min(m, n);
  if (S)
    for (int r = 0; r < kmin; ++r) S[r] = hs[hp[r]];
  if (left) DMRG2_CUDA(cudaMemcpy(left, dl.p, sb * (size_t)m * k, cudaMemcpyDeviceToHost));
  if (right) DMRG2_CUDA(cudaMemcpy(right, dr.p, sb * (size_t)k * n, cudaMemcpyDeviceToHost));
  if (k_out) *k_out = k;
  if (te_out) *te_out = o.trunc_err;
}

template <typename T>
void do_op_lanczos(int cL, int cR, int d, int Dl, int Dm, int Dr, const void* L, const void* R,
                   const void* WL, const void* WR, void* theta, int kmax, double tol, int restarts,
                   double* energy, int* iters) {
  const size_t sb = sizeof(T);
  const ll dd = (ll)d * d;
  std::vector<T> wwt;
  build_wwt((const T*)WL, (const T*)WR, Dl, Dm, Dr, d, wwt);
  const ll n = (ll)cL * dd * cR;
  DBuf dL(L, sb * cL * Dl * cL), dR(R, sb * cR * Dr * cR), dW(wwt.data(), sb * wwt.size());
  DBuf dth(theta, sb * n);
  const ll xs = std::max((ll)cL * Dl * dd * cR, (ll)cL * dd * Dr * cR);
  DBuf X(sb * xs), Y(sb * xs);
  cudaStream_t s;
  DMRG2_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  LanczosWork<T> W;
  try {
    W.init(kmax, n);
    auto mv = [&](const T* in, T* out, const int* skip) {
      heff_apply(dL.as<T>(), dR.as<T>(), dW.as<T>(), in, out, X.as<T>(), Y.as<T>(), cL, cR, d, Dl,
                 Dr, skip, s);
    };
    LanczosResult r = lanczos_solve<T>(W, dth.as<T>(), n, kmax, tol, restarts, 1234u, mv, s);
    DMRG2_CUDA(cudaStreamSynchronize(s));
    DMRG2_CUDA(cudaMemcpy(theta, dth.p, sb * n, cudaMemcpyDeviceToHost));
    if (energy) *energy = r.energy;
    if (iters) *iters = r.iters;
  } catch (...) {
    W.release();
    cudaStreamDestroy(s);
    throw;
  }
  W.release();
  cudaStreamDestroy(s);
}

template <typename T>
void do_op_gemm(int ta, int tb, int M, int N, int K, const double* alpha, const void* A, ll lda,
                const void* B, ll ldb, const double* beta, void* C, ll ldc) {
  const size_t sb = sizeof(T);
  const ll arows = (ta == 1 || ta == 2) ? K : M;
  const ll brows = (tb == 1 || tb == 2) ? N : K;
  DBuf dA(A, sb * (size_t)arows * lda), dB(B, sb * (size_t)brows * ldb), dC(C, sb * (size_t)M * ldc);
  Gemm<T> g;
  g.ta = (ta == 1 || ta == 2);
  g.ca = (ta == 2 || ta == 3);
  g.tb = (tb == 1 || tb == 2);
  if (tb >= 2) throw std::invalid_argument("op_gemm: conjugated B is not supported");
  g.M = M; g.N = N; g.K = K;
  g.A = dA.as<T>(); g.lda = lda;
  g.B = dB.as<T>(); g.ldb = ldb;
  g.C = dC.as<T>(); g.ldc = ldc;
  g.alpha = ST<T>::make(alpha[0], alpha[1]);
  g.beta = ST<T>::make(beta[0], beta[1]);
  launch_gemm(g, 0);
  DMRG2_CUDA(cudaMemcpy(C, dC.p, sb * (size_t)M * ldc, cudaMemcpyDeviceToHost));
}

template <typename T>
void do_op_gemm_bf16x3(int ta, int tb, int M, int N, int K, const double* alpha, const void* A, ll lda,
                       const void* B, ll ldb, const double* beta, void* C, ll ldc) {
  const size_t sb = sizeof(T);
  const ll arows = (ta == 1 || ta == 2) ? K : M;
  const ll brows = (tb == 1 || tb == 2) ? N : K;
  DBuf dA(A, sb * (size_t)arows * lda), dB(B, sb * (size_t)brows * ldb), dC(C, sb * (size_t)M * ldc);
  SplitScratch ws;
  try {
    gemm_bf16x3<T>(ta, tb, M, N, K, ST<T>::make(alpha[0], alpha[1]), dA.as<T>(), lda, 0, dB.as<T>(), ldb, 0,
                   ST<T>::make(beta[0], beta[1]), dC.as<T>(), ldc, 0, 1, ws, 0);
    int err = 0;
    DMRG2_CUDA(cudaMemcpy(&err, ws.err, sizeof(int), cudaMemcpyDeviceToHost));
    if (err) throw std::runtime_error("op_gemm_bf16x3: tensor-core completion wait timed out");
    DMRG2_CUDA(cudaMemcpy(C, dC.p, sb * (size_t)M * ldc, cudaMemcpyDeviceToHost));
  } catch (...) {
    ws.release();
    throw;
  }
  ws.release();
}

void check_dtype(int dt) {
  if (dt != DMRG2_F64 && dt != DMRG2_C128) throw std::invalid_argument("unknown dtype");
}

// dmrg2_config -> engine configuration (fields at 0 take the reference defaults)
EngineConfig engine_config(const dmrg2_config* cfg) {
  EngineConfig c;
  c.L = cfg->L;
  c.d = cfg->d;
  c.chi_max = cfg->chi_max;
  c.complex = cfg->dtype == DMRG2_C128;
  c.tol = cfg->tol > 0 ? cfg->tol : 1e-10;
  c.krylov_max = cfg->krylov_max > 0 ? cfg->krylov_max : 100;
  c.lanczos_tol = cfg->lanczos_tol > 0 ? cfg->lanczos_tol : 1e-12;
  c.max_restarts = cfg->max_restarts > 0 ? cfg->max_restarts : 0;
  c.cutoff = cfg->cutoff > 0 ? cfg->cutoff : (cfg->cutoff < 0 ? 0.0 : 1e-14);
  c.min_sweeps = cfg->min_sweeps > 0 ? cfg->min_sweeps : 2;
  c.seed = (unsigned)(cfg->seed ^ (cfg->seed >> 32));
  if (cfg->svd_method != 0 && cfg->svd_method != 1) throw std::invalid_argument("unknown svd_method");
  c.svd_method = cfg->svd_method;
  if (cfg->precision != 0 && cfg->precision != 1) throw std::invalid_argument("unknown precision form");
  c.precision = cfg->precision;
  if (cfg->single_site != 0 && cfg->single_site != 1) throw std::invalid_argument("single_site must be 0 or 1");
  c.single_site = cfg->single_site;
  if (cfg->truncation < 0 || cfg->truncation > 2) throw std::invalid_argument("unknown truncation");
  c.truncation = cfg->truncation;
  return c;
}
void check_pos(std::initializer_list<int> v) {
  for (int x : v)
    if (x < 1) throw std::invalid_argument("dimensions must be positive");
}

}  // namespace

extern "C" {

int dmrg2_abi_version(void) { return DMRG2_ABI_VERSION; }

const char* dmrg2_last_error(const dmrg2_handle* h) { return h ? h->err.c_str() : g_err.c_str(); }

}  // extern "C"

namespace {
int create_handle(const dmrg2_config* cfg, dmrg2_handle** out, bool graphs) {
  if (!cfg || !out) { g_err = "null argument"; return DMRG2_ERR_ARG; }
  *out = nullptr;
  return guarded(nullptr, [&] {
    check_dtype(cfg->dtype);
    check_pos({cfg->L, cfg->d, cfg->chi_max});
    if (cfg->L < 2) throw std::invalid_argument("L must be >= 2");
    DMRG2_CUDA(cudaSetDevice(cfg->device));
    EngineConfig c = engine_config(cfg);
    c.graphs = graphs;
    std::unique_ptr<dmrg2_handle> h(new dmrg2_handle);
    h->cfg = c;
    h->dtype = cfg->dtype;
    h->eng = make_engine(c);
    *out = h.release();
  });
}
}  // namespace

extern "C" {

int dmrg2_create(const dmrg2_config* cfg, dmrg2_handle** out) { return create_handle(cfg, out, true); }

void dmrg2_destroy(dmrg2_handle* h) { delete h; }

int dmrg2_set_mpo(dmrg2_handle* h, const void* const* W, const int* Dl, const int* Dr, int layout) {
  if (!h || !W || !Dl) { if (h) h->err = "null argument"; return DMRG2_ERR_ARG; }
  return guarded(h, [&] {
    const int L = h->cfg.L, d = h->cfg.d;
    const size_t sb = scalar_bytes(h->dtype);
    std::vector<const void*> ptrs(L);
    std::vector<int> dl(L), dr(L);
    std::vector<std::vector<char>> conv;
    if (layout == DMRG2_LAYOUT_ROWMAJOR) {
      if (!Dr) throw std::invalid_argument("set_mpo: Dr is required for the row-major layout");
      for (int i = 0; i < L; ++i) {
        ptrs[i] = W[i];
        dl[i] = Dl[i];
        dr[i] = Dr[i];
      }
    } else if (layout == DMRG2_LAYOUT_REFERENCE) {
      const int D = Dl[0];
      if (D < 1) throw std::invalid_argument("set_mpo: D_mpo must be positive");
      conv.resize(L);
      for (int i = 0; i < L; ++i) {
        const int a = (i == 0) ? 1 : D, b = (i == L - 1) ? 1 : D;
        dl[i] = a;
        dr[i] = b;
        conv[i].resize((size_t)a * b * d * d * sb);
        const char* src = (const char*)W[i];
        for (int w = 0; w < a; ++w)
          for (int wp = 0; wp < b; ++wp)
            for (int s = 0; s < d; ++s)
              for (int sp = 0; sp < d; ++sp) {
                const int ws = (i == 0) ? 0 : w;
                const int wps = (i == L - 1) ? D - 1 : wp;
                const size_t si = (size_t)ws + (size_t)s * D + (size_t)sp * D * d + (size_t)wps * D * d * d;
                const size_t di = (((size_t)w * b + wp) * d + s) * d + sp;
                std::memcpy(conv[i].data() + di * sb, src + si * sb, sb);
              }
        ptrs[i] = conv[i].data();
      }
    } else {
      throw std::invalid_argument("set_mpo: unknown layout");
    }
    h->eng->set_mpo(ptrs, dl, dr);
  });
}

int dmrg2_set_mps(dmrg2_handle* h, const void* const* A, const int* bond_dims, int layout) {
  if (!h || !A || !bond_dims) { if (h) h->err = "null argument"; return DMRG2_ERR_ARG; }
  return guarded(h, [&] {
    const int L = h->cfg.L, d = h->cfg.d;
    const size_t sb = scalar_bytes(h->dtype);
    std::vector<int> dims(bond_dims, bond_dims + L + 1);
    std::vector<const void*> ptrs(L);
    std::vector<std::vector<char>> conv;
    if (layout == DMRG2_LAYOUT_ROWMAJOR) {
      for (int i = 0; i < L; ++i) ptrs[i] = A[i];
    } else if (layout == DMRG2_LAYOUT_REFERENCE) {
      conv.resize(L);
      for (int i = 0; i < L; ++i) {
        conv[i].resize((size_t)dims[i] * d * dims[i + 1] * sb);
        mps_ref_to_row((const char*)A[i], conv[i].data(), dims[i], d, dims[i + 1], sb);
        ptrs[i] = conv[i].data();
      }
    } else {
      throw std::invalid_argument("set_mps: unknown layout");
    }
    h->eng->set_mps(ptrs, dims);
  });
}

int dmrg2_init_mps(dmrg2_handle* h, int kind, uint64_t seed) {
  if (!h) return DMRG2_ERR_ARG;
  return guarded(h, [&] {
    const int L = h->cfg.L, d = h->cfg.d;
    const bool cplx = h->dtype == DMRG2_C128;
    std::vector<int> dims;
    if (kind == DMRG2_INIT_PRODUCT) dims.assign(L + 1, 1);
    else dims = reference_bond_dims(L, d, h->cfg.chi_max);
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<double> U(-1.0, 1.0);
    std::vector<std::vector<double>> t(L);
    std::vector<const void*> ptrs(L);
    const int per = cplx ? 2 : 1;
    for (int i = 0; i < L; ++i) {
      const int cl = dims[i], cr = dims[i + 1];
      t[i].assign((size_t)cl * d * cr * per, 0.0);
      if (kind == DMRG2_INIT_RANDOM) {
        for (auto& v : t[i]) v = 0.1 * U(rng);
      } else {
        const int s = (kind == DMRG2_INIT_NEEL) ? (i % 2) : 0;
        for (int a = 0; a < std::min(cl, cr); ++a) t[i][(((size_t)a * d + s) * cr + a) * per] = 1.0;
      }
      ptrs[i] = t[i].data();
    }
    if (kind != DMRG2_INIT_RANDOM && kind != DMRG2_INIT_PRODUCT && kind != DMRG2_INIT_NEEL)
      throw std::invalid_argument("init_mps: unknown kind");
    h->eng->set_mps(ptrs, dims);
  });
}

static void fill_reports(const std::vector<SweepStats>& st, dmrg2_sweep_report* out, int max_out,
                         int* n_out) {
  if (n_out) *n_out = (int)st.size();
  for (int s = 0; s < (int)st.size() && out && s < max_out; ++s) {
    dmrg2_sweep_report& r = out[s];
    r.sweep = st[s].sweep;
    r.chi_max = st[s].chi_max;
    r.energy = st[s].energy;
    r.trunc_err_max = st[s].trunc_err_max;
    r.trunc_err_sum = st[s].trunc_err_sum;
    r.max_bond = st[s].max_bond;
    r.wall_s = st[s].wall_s;
    r.matvecs = st[s].matvecs;
    r.heff_s = st[s].heff_s;
    r.heff_flops = st[s].heff_flops;
    r.lanczos_iters = st[s].lanczos_iters;
    r.lanczos_unconverged = st[s].lanczos_unconverged;
    r.svd_s = st[s].svd_s;
    r.jacobi_sweeps_max = st[s].jacobi_sweeps_max;
    r.device_s = st[s].device_s;
    r.lowprec_matvecs = st[s].lowprec_matvecs;
    r.warm_splits = st[s].warm_splits;
    r.warm_fallbacks = st[s].warm_fallbacks;
    r.warm_short = st[s].warm_short;
    r.rsvd_splits = st[s].rsvd_splits;
    r.rsvd_fallbacks = st[s].rsvd_fallbacks;
    r.eig_fallbacks = st[s].eig_fallbacks;
    r.phase = st[s].phase;
    r.device_loops = st[s].device_loops;
  }
}

static std::vector<int> make_schedule(const dmrg2_handle* h, const int* chi_schedule, int n) {
  if (n < 1) throw std::invalid_argument("n_sweeps must be >= 1");
  std::vector<int> sched(n, h->cfg.chi_max);
  if (chi_schedule)
    for (int s = 0; s < n; ++s) sched[s] = chi_schedule[s];
  return sched;
}

int dmrg2_run(dmrg2_handle* h, const int* chi_schedule, int n_sweeps, dmrg2_sweep_report* out,
              int max_out, int* n_out) {
  if (!h) return DMRG2_ERR_ARG;
  return guarded(h, [&] {
    fill_reports(h->eng->run(make_schedule(h, chi_schedule, n_sweeps)), out, max_out, n_out);
  });
}

int dmrg2_resume(dmrg2_handle* h, const int* chi_schedule, int n_sweeps, dmrg2_sweep_report* out,
                 int max_out, int* n_out) {
  if (!h) return DMRG2_ERR_ARG;
  return guarded(h, [&] {
    fill_reports(h->eng->resume(make_schedule(h, chi_schedule, n_sweeps)), out, max_out, n_out);
  });
}

int dmrg2_pdmrg_run(dmrg2_handle* h, const dmrg2_pdmrg_options* opt, dmrg2_sweep_report* out, int max_out,
                    int* n_out) {
  if (!h || !opt) return DMRG2_ERR_ARG;
  return guarded(h, [&] {
    PdmrgOptions o;
    o.n_segments = opt->n_segments;
    o.n_outer = opt->n_outer;
    o.n_local = opt->n_local;
    o.n_warmup = opt->n_warmup;
    o.n_polish = opt->n_polish;
    o.n_recal = opt->n_recal;
    o.chi = opt->chi;
    fill_reports(h->eng->pdmrg(o), out, max_out, n_out);
  });
}

long long dmrg2_get_launch_count(void) { return launch_counter().load(); }

int dmrg2_get_energy(const dmrg2_handle* h, double* e) {
  if (!h || !e) return DMRG2_ERR_ARG;
  *e = h->eng->energy();
  return DMRG2_OK;
}

int dmrg2_get_env_build_seconds(const dmrg2_handle* h, double* s) {
  if (!h || !s) return DMRG2_ERR_ARG;
  *s = h->eng->env_build_s();
  return DMRG2_OK;
}

int dmrg2_get_bond_dims(const dmrg2_handle* h, int* dims) {
  if (!h || !dims) return DMRG2_ERR_ARG;
  const auto& b = h->eng->bond_dims();
  std::copy(b.begin(), b.end(), dims);
  return DMRG2_OK;
}

int dmrg2_get_device_bytes(const dmrg2_handle* h, size_t* bytes) {
  if (!h || !bytes) return DMRG2_ERR_ARG;
  *bytes = h->eng->device_bytes();
  return DMRG2_OK;
}

int dmrg2_get_mps(dmrg2_handle* h, void* const* out, int layout) {
  if (!h || !out) return DMRG2_ERR_ARG;
  return guarded(h, [&] {
    const int L = h->cfg.L, d = h->cfg.d;
    const size_t sb = scalar_bytes(h->dtype);
    const auto dims = h->eng->bond_dims();
    if (layout == DMRG2_LAYOUT_ROWMAJOR) {
      std::vector<void*> p(out, out + L);
      h->eng->get_mps(p);
    } else if (layout == DMRG2_LAYOUT_REFERENCE) {
      std::vector<std::vector<char>> tmp(L);
      std::vector<void*> p(L);
      for (int i = 0; i < L; ++i) {
        tmp[i].resize((size_t)dims[i] * d * dims[i + 1] * sb);
        p[i] = tmp[i].data();
      }
      h->eng->get_mps(p);
      for (int i = 0; i < L; ++i)
        mps_row_to_ref(tmp[i].data(), (char*)out[i], dims[i], d, dims[i + 1], sb);
    } else {
      throw std::invalid_argument("get_mps: unknown layout");
    }
  });
}

int dmrg2_expect_local(dmrg2_handle* h, const void* op, double* re, double* im) {
  if (!h || !op || !re) return DMRG2_ERR_ARG;
  return guarded(h, [&] {
    std::vector<double> r, i;
    h->eng->expect_local(op, r, i);
    std::copy(r.begin(), r.end(), re);
    if (im) std::copy(i.begin(), i.end(), im);
  });
}

int dmrg2_op_heff(int dtype, int cL, int cR, int d, int Dl, int Dm, int Dr, const void* L,
                  const void* R, const void* WL, const void* WR, const void* theta, void* out) {
  return guarded(nullptr, [&] {
    check_dtype(dtype);
    check_pos({cL, cR, d, Dl, Dm, Dr});
    if (dtype == DMRG2_C128) do_op_heff<zc>(cL, cR, d, Dl, Dm, Dr, L, R, WL, WR, theta, out);
    else do_op_heff<double>(cL, cR, d, Dl, Dm, Dr, L, R, WL, WR, theta, out);
  });
}

int dmrg2_op_env_left(int dtype, int cL, int cO, int d, int Dl, int Dr, const void* L,
                      const void* A, const void* W, void* out) {
  return guarded(nullptr, [&] {
    check_dtype(dtype);
    check_pos({cL, cO, d, Dl, Dr});
    if (dtype == DMRG2_C128) do_op_env_left<zc>(cL, cO, d, Dl, Dr, L, A, W, out);
    else do_op_env_left<double>(cL, cO, d, Dl, Dr, L, A, W, out);
  });
}

int dmrg2_op_env_right(int dtype, int cI, int cO, int d, int Dl, int Dr, const void* R,
                       const void* B, const void* W, void* out) {
  return guarded(nullptr, [&] {
    check_dtype(dtype);
    check_pos({cI, cO, d, Dl, Dr});
    if (dtype == DMRG2_C128) do_op_env_right<zc>(cI, cO, d, Dl, Dr, R, B, W, out);
    else do_op_env_right<double>(cI, cO, d, Dl, Dr, R, B, W, out);
  });
}

int dmrg2_op_svd(int dtype, int m, int n, const void* M, int max_bond, double cutoff,
                 char direction, double* S, void* left, void* right, int* k, double* trunc_err) {
  return guarded(nullptr, [&] {
    check_dtype(dtype);
    check_pos({m, n, max_bond});
    if (direction != 'R' && direction != 'L' && direction != 'r' && direction != 'l')
      throw std::invalid_argument("op_svd: direction must be 'R' or 'L'");
    const bool jac = (direction == 'r' || direction == 'l');
    if (dtype == DMRG2_C128) {
      if (jac) do_op_svd<zc>(m, n, M, max_bond, cutoff, direction, S, left, right, k, trunc_err);
      else do_op_svd_eig<zc>(m, n, M, max_bond, cutoff, direction, S, left, right, k, trunc_err);
    } else {
      if (jac) do_op_svd<double>(m, n, M, max_bond, cutoff, direction, S, left, right, k, trunc_err);
      else do_op_svd_eig<double>(m, n, M, max_bond, cutoff, direction, S, left, right, k, trunc_err);
    }
  });
}

int dmrg2_op_warm_split(int dtype, int m, int n, const void* M, const void* warm, int k, char direction,
                        void* left, void* right, double* trunc_err) {
  return guarded(nullptr, [&] {
    check_dtype(dtype);
    check_pos({m, n, k});
    if (dtype != DMRG2_F64) throw std::invalid_argument("op_warm_split: real (f64) data only");
    if (direction != 'R' && direction != 'L') throw std::invalid_argument("op_warm_split: direction must be 'R' or 'L'");
    if (!M || !warm) throw std::invalid_argument("op_warm_split: null input");
    if (k > CHOL_MAX || k >= std::min(m, n)) throw std::invalid_argument("op_warm_split: need k < min(m, n) and k <= 512");
    if (!do_op_warm_split(m, n, M, warm, k, direction, left, right, trunc_err))
      throw NumericError("op_warm_split: CholeskyQR gave up (a kept singular value below ~1e-6 of the largest)");
  });
}

int dmrg2_op_lanczos(int dtype, int cL, int cR, int d, int Dl, int Dm, int Dr, const void* L,
                     const void* R, const void* WL, const void* WR, void* theta, int krylov_max,
                     double tol, int max_restarts, double* energy, int* iters) {
  return guarded(nullptr, [&] {
    check_dtype(dtype);
    check_pos({cL, cR, d, Dl, Dm, Dr, krylov_max});
    if (dtype == DMRG2_C128)
      do_op_lanczos<zc>(cL, cR, d, Dl, Dm, Dr, L, R, WL, WR, theta, krylov_max, tol, max_restarts,
                        energy, iters);
    else
      do_op_lanczos<double>(cL, cR, d, Dl, Dm, Dr, L, R, WL, WR, theta, krylov_max, tol,
                            max_restarts, energy, iters);
  });
}

int dmrg2_op_gemm(int dtype, int transA, int transB, int M, int N, int K, const double* alpha,
                  const void* A, long long lda, const void* B, long long ldb, const double* beta,
                  void* C, long long ldc) {
  return guarded(nullptr, [&] {
    check_dtype(dtype);
    check_pos({M, N, K});
    if (dtype == DMRG2_C128) do_op_gemm<zc>(transA, transB, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
    else do_op_gemm<double>(transA, transB, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
  });
}

int dmrg2_op_gemm_bf16x3(int dtype, int transA, int transB, int M, int N, int K, const double* alpha,
                         const void* A, long long lda, const void* B, long long ldb, const double* beta,
                         void* C, long long ldc) {
  return guarded(nullptr, [&] {
    check_dtype(dtype);
    check_pos({M, N, K});
    if (!alpha || !beta || !A || !B || !C) throw std::invalid_argument("op_gemm_bf16x3: null argument");
    if (transA < 0 || transA > 3 || transB < 0 || transB > 2) throw std::invalid_argument("op_gemm_bf16x3: bad trans");
    if (dtype == DMRG2_C128)
      do_op_gemm_bf16x3<zc>(transA, transB, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
    else
      do_op_gemm_bf16x3<double>(transA, transB, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
  });
}

int dmrg2_op_heff_noalloc(int dtype, int cL, int cR, int d, int Dl, int Dm, int Dr, const void* L,
                          const void* R, const void* WL, const void* WR, const void* theta, void* out,
                          void* stream) {
  return guarded(nullptr, [&] {
    check_dtype(dtype);
    check_pos({cL, cR, d, Dl, Dm, Dr});
    if (!L || !R || !WL || !WR || !theta || !out)
      throw std::invalid_argument("op_heff_noalloc: null device pointer");
    cudaStream_t s = (cudaStream_t)stream;
    if (dtype == DMRG2_C128)
      heff_noalloc<zc>(cL, cR, d, Dl, Dm, Dr, (const zc*)L, (const zc*)R, (const zc*)WL, (const zc*)WR,
                       (const zc*)theta, (zc*)out, s);
    else
      heff_noalloc<double>(cL, cR, d, Dl, Dm, Dr, (const double*)L, (const double*)R, (const double*)WL,
                           (const double*)WR, (const double*)theta, (double*)out, s);
  });
}

}  // extern "C"

// ============================================================================
// Served / batched form. Requests are copied at submit, admitted in arrival
// order while a worker slot is idle and their device footprint fits in the
// budget, and solved by the worker that admitted them, each on its own engine
// and CUDA stream, so the kernels of different solves overlap on the device.
// ============================================================================
namespace {

struct ServedRequest {
  long long id = 0;
  dmrg2_config cfg{};
  std::vector<std::vector<char>> W;
  std::vector<int> Dl, Dr;
  std::vector<std::vector<char>> A;
  std::vector<int> dims;
  int init_kind = DMRG2_INIT_RANDOM;
  std::vector<int> schedule;
  dmrg2_result res{};
};

void set_message(dmrg2_result& r, const std::string& m) {
  std::strncpy(r.message, m.c_str(), sizeof(r.message) - 1);
  r.message[sizeof(r.message) - 1] = 0;
}

}  // namespace

struct dmrg2_server {
  int device = 0;
  int max_active = 8;
  size_t budget = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<ServedRequest*> queue;
  std::map<long long, std::unique_ptr<ServedRequest>> reqs;
  size_t reserved = 0;
  int active = 0;
  bool stop = false;
  long long next_id = 1;
  std::vector<std::thread> workers;
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();

  double now() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }

  void worker() {
    (void)cudaSetDevice(device);
    for (;;) {
      ServedRequest* r = nullptr;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv_work.wait(lk, [&] {
          return stop || (!queue.empty() && reserved + queue.front()->res.footprint_bytes <= budget);
        });
        if (stop) return;
        r = queue.front();
        queue.pop_front();
        reserved += r->res.footprint_bytes;
        ++active;
        r->res.state = DMRG2_REQ_RUNNING;
        r->res.t_admit = now();
      }
      solve(r);
      {
        std::lock_guard<std::mutex> lk(mu);
        reserved -= r->res.footprint_bytes;
        --active;
        r->res.t_done = now();
        r->res.state = r->res.status == DMRG2_OK ? DMRG2_REQ_DONE : DMRG2_REQ_FAILED;
      }
      cv_done.notify_all();
      cv_work.notify_all();
    }
  }

  // one solve through the public entry points, on this worker's own handle
  static void solve(ServedRequest* r) {
    dmrg2_handle* h = nullptr;
    int rc = create_handle(&r->cfg, &h, false);
    const int L = r->cfg.L;
    if (rc == DMRG2_OK) {
      std::vector<const void*> w(L);
      for (int i = 0; i < L; ++i) w[i] = r->W[i].data();
      rc = dmrg2_set_mpo(h, w.data(), r->Dl.data(), r->Dr.data(), DMRG2_LAYOUT_ROWMAJOR);
    }
    if (rc == DMRG2_OK) {
      if (!r->A.empty()) {
        std::vector<const void*> a(L);
        for (int i = 0; i < L; ++i) a[i] = r->A[i].data();
        rc = dmrg2_set_mps(h, a.data(), r->dims.data(), DMRG2_LAYOUT_ROWMAJOR);
      } else {
        rc = dmrg2_init_mps(h, r->init_kind, r->cfg.seed);
      }
    }
    std::vector<dmrg2_sweep_report> rep(r->schedule.size());
    int n_out = 0;
    if (rc == DMRG2_OK)
      rc = dmrg2_run(h, r->schedule.data(), (int)r->schedule.size(), rep.data(), (int)rep.size(), &n_out);
    if (rc == DMRG2_OK && n_out > 0) {
      const dmrg2_sweep_report& last = rep[(size_t)std::min<int>(n_out, (int)rep.size()) - 1];
      r->res.energy = last.energy;
      r->res.sweeps = n_out;
      r->res.trunc_err_max = last.trunc_err_max;
      r->res.max_bond = last.max_bond;
      for (int i = 0; i < std::min<int>(n_out, (int)rep.size()); ++i) r->res.device_s += rep[i].device_s;
    } else if (rc != DMRG2_OK) {
      set_message(r->res, dmrg2_last_error(h));
    }
    r->res.status = rc;
    if (h) dmrg2_destroy(h);
  }
};

extern "C" {

int dmrg2_server_create(const dmrg2_server_config* cfg, dmrg2_server** out) {
  if (!cfg || !out) { g_err = "null argument"; return DMRG2_ERR_ARG; }
  *out = nullptr;
  return guarded(nullptr, [&] {
    if (cfg->max_active < 0) throw std::invalid_argument("server: max_active must be >= 0");
    DMRG2_CUDA(cudaSetDevice(cfg->device));
    std::unique_ptr<dmrg2_server> s(new dmrg2_server);
    s->device = cfg->device;
    s->max_active = cfg->max_active > 0 ? cfg->max_active : 8;
    size_t budget = cfg->hbm_budget_bytes;
    if (budget == 0) {
      size_t fr = 0, tot = 0;
      DMRG2_CUDA(cudaMemGetInfo(&fr, &tot));
      budget = fr / 10 * 9;
    }
    s->budget = budget;
    dmrg2_server* raw = s.get();
    for (int i = 0; i < s->max_active; ++i) s->workers.emplace_back([raw] { raw->worker(); });
    *out = s.release();
  });
}

int dmrg2_server_submit(dmrg2_server* s, const dmrg2_request* q, long long* id) {
  if (!s || !q || !id) { g_err = "null argument"; return DMRG2_ERR_ARG; }
  return guarded(nullptr, [&] {
    const dmrg2_config& c = q->cfg;
    check_dtype(c.dtype);
    check_pos({c.L, c.d, c.chi_max, q->n_sweeps});
    if (c.L < 2) throw std::invalid_argument("L must be >= 2");
    if (!q->W || !q->Dl || !q->Dr || !q->schedule) throw std::invalid_argument("submit: null MPO or schedule");
    std::unique_ptr<ServedRequest> r(new ServedRequest);
    r->cfg = c;
    r->cfg.device = s->device;
    const int L = c.L, d = c.d;
    const size_t sb = scalar_bytes(c.dtype);
    r->Dl.assign(q->Dl, q->Dl + L);
    r->Dr.assign(q->Dr, q->Dr + L);
    r->W.resize(L);
    for (int i = 0; i < L; ++i) {
      if (r->Dl[i] < 1 || r->Dr[i] < 1) throw std::invalid_argument("submit: MPO bonds must be positive");
      const size_t b = (size_t)r->Dl[i] * r->Dr[i] * d * d * sb;
      r->W[i].assign((const char*)q->W[i], (const char*)q->W[i] + b);
    }
    if (q->A) {
      if (!q->bond_dims) throw std::invalid_argument("submit: MPS without bond dimensions");
      r->dims.assign(q->bond_dims, q->bond_dims + L + 1);
      r->A.resize(L);
      for (int i = 0; i < L; ++i) {
        const size_t b = (size_t)r->dims[i] * d * r->dims[i + 1] * sb;
        r->A[i].assign((const char*)q->A[i], (const char*)q->A[i] + b);
      }
    }
    r->init_kind = q->init_kind;
    r->schedule.assign(q->schedule, q->schedule + q->n_sweeps);
    for (int x : r->schedule)
      if (x < 1 || x > c.chi_max) throw std::invalid_argument("submit: schedule entry outside [1, chi_max]");
    r->res.footprint_bytes = engine_footprint(engine_config(&c), r->Dl, r->Dr);
    if (r->res.footprint_bytes > s->budget)
      throw std::invalid_argument("submit: request needs " + std::to_string(r->res.footprint_bytes) +
                                  " device bytes, above the server budget of " + std::to_string(s->budget));
    {
      std::lock_guard<std::mutex> lk(s->mu);
      if (s->stop) throw std::logic_error("submit: server is shutting down");
      r->id = s->next_id++;
      r->res.state = DMRG2_REQ_QUEUED;
      r->res.t_submit = s->now();
      *id = r->id;
      s->queue.push_back(r.get());
      s->reqs[r->id] = std::move(r);
    }
    s->cv_work.notify_one();
  });
}

int dmrg2_server_poll(dmrg2_server* s, long long id, int wait_ms, dmrg2_result* out) {
  if (!s || !out) { g_err = "null argument"; return DMRG2_ERR_ARG; }
  return guarded(nullptr, [&] {
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) throw std::invalid_argument("poll: unknown request id");
    ServedRequest* r = it->second.get();
    auto finished = [&] { return r->res.state == DMRG2_REQ_DONE || r->res.state == DMRG2_REQ_FAILED; };
    if (wait_ms < 0) s->cv_done.wait(lk, finished);
    else if (wait_ms > 0) s->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), finished);
    *out = r->res;
  });
}

void dmrg2_server_destroy(dmrg2_server* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    for (ServedRequest* r : s->queue) {
      r->res.state = DMRG2_REQ_FAILED;
      r->res.status = DMRG2_ERR_STATE;
      set_message(r->res, "server destroyed before admission");
    }
    s->queue.clear();
  }
  s->cv_work.notify_all();
  for (auto& t : s->workers) t.join();  // running solves finish first
  s->cv_done.notify_all();
  delete s;
}

}  // extern "C"
