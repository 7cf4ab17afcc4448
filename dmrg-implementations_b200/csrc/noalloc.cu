// H_eff matvec on device-resident operands that allocates no device memory.
//
// Who needs this: callers that must not allocate on the device while they
// run -- a solver that drives its own Lanczos loop between kernels it has
// already enqueued on a stream, code running under a fixed memory budget, or
// a host that records a stream and may not call cudaMalloc/cudaFree in the
// middle of it. The host-buffer entry point (dmrg2_op_heff) allocates staging
// and scratch buffers on every call, so it cannot serve them.
//
// How: the two intermediates of the three-GEMM contraction (X, Y) and the
// fused two-site MPO (WWt) live in one file-scope static device array. Its
// address is taken once per device and CUDA context, with that device
// current, through cudaGetSymbolAddress; every later call in the same context
// only launches kernels. When the context changes (after cudaDeviceReset, or
// when another primary context replaced it) the module is loaded anew and the
// array may sit elsewhere, so the address is looked up again. The first call
// in a context therefore does this set-up (it allocates nothing) and should
// come before any stream capture. The array belongs to this translation
// unit's module, so it takes device memory only once this entry point is
// first used, and every GPU that loaded it keeps it until the process exits.
//
// Limits: WWt, X and Y together (each rounded up to 256 bytes) must fit in
// NOALLOC_SCRATCH_BYTES; larger problems are rejected before any device work.
// Every call on a device shares the same array: calls on one stream run one
// after the other and are safe, calls that overlap in time (other streams or
// host threads on the same device) race on it. Nothing in the array needs to
// start at zero: the WWt kernel writes every entry, and the GEMMs and the MPO
// mixing kernel write every element of X and Y (beta = 0) before reading it.
#include <cuda.h>

#include <algorithm>
#include <mutex>

#include "common.cuh"
#include "contract.cuh"
#include "noalloc.cuh"
#include "../../include/dmrg2_b200.h"

static_assert(NOALLOC_SCRATCH_BYTES == DMRG2_NOALLOC_SCRATCH_BYTES, "scratch size differs from the public header");

namespace dmrg2 {

namespace {

constexpr size_t kScratchDoubles = NOALLOC_SCRATCH_BYTES / sizeof(double);
static __device__ __align__(256) double g_heff_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
struct ScratchSlot {
  unsigned long long ctx_id = 0;  // driver's unique id of the context the address belongs to
  void* ptr = nullptr;
};
ScratchSlot g_scratch[kMaxDevices];

// Unique id of the calling thread's current context, 0 when there is none. The
// driver entry points are looked up through the runtime, so the library does not
// link the driver library (it still loads on a machine without one).
unsigned long long current_context_id() {
  using GetCurrent = CUresult (*)(CUcontext*);
  using GetId = CUresult (*)(CUcontext, unsigned long long*);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<GetCurrent>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<GetId>(f);
  });
  if (!get_current || !get_id) throw CudaError("op_heff_noalloc: driver context queries unavailable");
  CUcontext ctx = nullptr;
  if (get_current(&ctx) != CUDA_SUCCESS || !ctx) return 0;
  unsigned long long id = 0;
  if (get_id(ctx, &id) != CUDA_SUCCESS) return 0;
  return id;
}

// Address of the static scratch in the current device's current context. The first
// call in a context resolves the symbol (which loads this module there); a changed
// context id means the module may have been reloaded, so the address is resolved
// again.
void* scratch_on_current_device() {
  int dev = 0;
  DMRG2_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) throw std::invalid_argument("op_heff_noalloc: device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_setup_mu);
  ScratchSlot& slot = g_scratch[dev];
  const unsigned long long id = current_context_id();
  if (slot.ptr && id != 0 && id == slot.ctx_id) return slot.ptr;
  void* p = nullptr;
  DMRG2_CUDA(cudaGetSymbolAddress(&p, g_heff_scratch));  // makes the device's context current if needed
  if (!p) throw CudaError("op_heff_noalloc: cudaGetSymbolAddress returned a null scratch address");
  slot.ptr = p;
  slot.ctx_id = current_context_id();
  return p;
}

size_t round256(size_t b) { return (b + 255) & ~(size_t)255; }

// WWt[(p,q,n)][(w,s,r)] = sum_m WL[w][m][s][p] * WR[m][n][r][q]; one thread per entry,
// the sum over m in the same order as the host builder of the engine.
template <typename T>
__global__ void wwt_kernel(const T* __restrict__ WL, const T* __restrict__ WR, T* __restrict__ out,
                           int Dl, int Dm, int Dr, int d) {
  const ll rows = (ll)d * d * Dr, cols = (ll)Dl * d * d;
  const ll i = (ll)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows * cols) return;
  const ll row = i / cols, col = i % cols;
  const int n = (int)(row % Dr), q = (int)((row / Dr) % d), p = (int)(row / ((ll)Dr * d));
  const int r = (int)(col % d), s = (int)((col / d) % d), w = (int)(col / ((ll)d * d));
  T acc = ST<T>::zero();
  for (int m = 0; m < Dm; ++m) {
    const T a = WL[(((ll)w * Dm + m) * d + s) * d + p];
    const T b = WR[(((ll)m * Dr + n) * d + r) * d + q];
    acc = acc + ST<T>::mul(a, b);
  }
  out[i] = acc;
}

}  // namespace

size_t heff_noalloc_scratch_bytes(int cL, int cR, int d, int Dl, int Dr, size_t scalar_bytes) {
  // every product is checked: absurd shapes must not wrap to a small count
  if (cL < 1 || cR < 1 || d < 1 || Dl < 1 || Dr < 1) return SIZE_MAX;
  auto mul = [](size_t a, size_t b, bool& ovf) {
    size_t r = 0;
    if (__builtin_mul_overflow(a, b, &r)) ovf = true;
    return r;
  };
  bool ovf = false;
  const size_t dd = mul((size_t)d, (size_t)d, ovf);
  const size_t wwt = mul(mul(mul(dd, (size_t)Dr, ovf), mul((size_t)Dl, dd, ovf), ovf), scalar_bytes, ovf);
  const size_t lr = mul((size_t)cL, (size_t)cR, ovf);
  const size_t x1 = mul(mul(lr, (size_t)Dl, ovf), dd, ovf), x2 = mul(mul(lr, (size_t)Dr, ovf), dd, ovf);
  const size_t xs = mul(std::max(x1, x2), scalar_bytes, ovf);
  if (ovf || wwt > SIZE_MAX / 4 || xs > SIZE_MAX / 4) return SIZE_MAX;
  return round256(wwt) + 2 * round256(xs);
}

template <typename T>
void heff_noalloc(int cL, int cR, int d, int Dl, int Dm, int Dr, const T* L, const T* R, const T* WL,
                  const T* WR, const T* theta, T* out, cudaStream_t s) {
  const size_t need = heff_noalloc_scratch_bytes(cL, cR, d, Dl, Dr, sizeof(T));
  if (need == SIZE_MAX)
    throw std::invalid_argument("op_heff_noalloc: shape too large (its scratch size overflows), above the "
                                "static limit of " + std::to_string((size_t)NOALLOC_SCRATCH_BYTES) + " bytes");
  if (need > NOALLOC_SCRATCH_BYTES)
    throw std::invalid_argument("op_heff_noalloc: problem needs " + std::to_string(need) +
                                " bytes of scratch, above the static limit of " +
                                std::to_string((size_t)NOALLOC_SCRATCH_BYTES) + " bytes");
  char* base = (char*)scratch_on_current_device();
  const ll dd = (ll)d * d;
  const size_t wwt_b = round256((size_t)(dd * Dr) * (size_t)(Dl * dd) * sizeof(T));
  const size_t xs_b = round256((size_t)std::max((ll)cL * Dl * dd * cR, (ll)cL * dd * Dr * cR) * sizeof(T));
  T* WWt = (T*)base;
  T* X = (T*)(base + wwt_b);
  T* Y = (T*)(base + wwt_b + xs_b);
  const ll entries = dd * Dr * Dl * dd;
  wwt_kernel<T><<<(unsigned)((entries + 255) / 256), 256, 0, s>>>(WL, WR, WWt, Dl, Dm, Dr, d);
  DMRG2_CHECK_LAUNCH();
  heff_apply<T>(L, R, WWt, theta, out, X, Y, cL, cR, d, Dl, Dr, nullptr, s);
}

template void heff_noalloc<double>(int, int, int, int, int, int, const double*, const double*,
                                   const double*, const double*, const double*, double*, cudaStream_t);
template void heff_noalloc<zc>(int, int, int, int, int, int, const zc*, const zc*, const zc*, const zc*,
                               const zc*, zc*, cudaStream_t);

}  // namespace dmrg2
