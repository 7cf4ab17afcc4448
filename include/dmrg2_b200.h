/*
 * dmrg2_b200.h - C ABI of the B200-native two-site DMRG engine.
 *
 * The solver entry points replace the C++ class DMRG2GPU<Scalar> of the
 * reference driver (gpu-rocm/dmrg2-gpu/src/dmrg2_gpu.h:24-203) with plain C
 * functions: integer status codes instead of exceptions, caller-owned host
 * buffers, handle-owned device memory. The op-level entry points replace the
 * reference's numpy two-site primitives (the modules of cpu/pdmrg/pdmrg/numerics/ and
 * cpu/pdmrg/pdmrg/environments/update.py) one for one and run them on the GPU.
 *
 * Scalars: DMRG2_F64 = double, DMRG2_C128 = interleaved (re, im) doubles,
 * ABI-compatible with cuDoubleComplex / hipDoubleComplex / numpy complex128.
 *
 * Tensor layouts (DMRG2_LAYOUT_ROWMAJOR, the numpy C-order of the oracle):
 *   MPS site   A[i]  shape (chi_i, d, chi_{i+1})          index (a*d + s)*chi_{i+1} + b
 *   MPO site   W[i]  shape (Dl_i, Dr_i, d, d)              axes (mpo_l, mpo_r, s_in, s_out);
 *                    the applied operator is O[s_out][s_in] = W[..., s_in, s_out];
 *                    Dl_0 = Dr_{L-1} = 1.
 *   local op   op    d x d row-major, op[s_out*d + s_in] = <s_out|O|s_in>
 *   envs       (bra, mpo, ket)
 * DMRG2_LAYOUT_REFERENCE is the column-major layout of the reference driver:
 *   MPS  A[a + s*chi_l + b*chi_l*d]
 *   MPO  W[w + s*D + sp*D*d + wp*D*d*d] with one padded D for all sites, the left
 *        boundary picking row 0 of W[0] and the right boundary column D-1 of
 *        W[L-1] (gpu-rocm/common/challenge_mpos.h:4-7).
 *
 * Threading: one handle per host thread; calls on one handle are not
 * reentrant. All functions return DMRG2_OK (0) on success.
 */
#ifndef DMRG2_B200_H
#define DMRG2_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DMRG2_ABI_VERSION 7

enum dmrg2_status {
  DMRG2_OK = 0,
  DMRG2_ERR_ARG = 1,     /* invalid argument or shape */
  DMRG2_ERR_CUDA = 2,    /* CUDA runtime error (message in dmrg2_last_error) */
  DMRG2_ERR_STATE = 3,   /* call out of order (e.g. run before set_mpo) */
  DMRG2_ERR_NUMERIC = 4, /* solver failure (e.g. Jacobi barrier timeout) */
  DMRG2_ERR_INTERNAL = 5
};

enum dmrg2_dtype { DMRG2_F64 = 0, DMRG2_C128 = 1 };
enum dmrg2_layout { DMRG2_LAYOUT_ROWMAJOR = 0, DMRG2_LAYOUT_REFERENCE = 1 };
enum dmrg2_init_kind { DMRG2_INIT_RANDOM = 0, DMRG2_INIT_PRODUCT = 1, DMRG2_INIT_NEEL = 2 };

typedef struct dmrg2_handle dmrg2_handle;

/* Solver configuration. Fields left at 0 take the reference driver's defaults
 * (dmrg2_gpu_impl.h:138,975-976,1276; dmrg2_gpu.h:30). */
typedef struct dmrg2_config {
  int L;              /* chain length */
  int d;              /* local dimension */
  int chi_max;        /* largest bond dimension any sweep may use */
  int dtype;          /* dmrg2_dtype */
  double tol;         /* sweep stop rule |E_sweep - E_prev| < tol (0 -> 1e-10) */
  int krylov_max;     /* Lanczos vectors per pass (0 -> 100, capped at 128) */
  double lanczos_tol; /* Lanczos stop rule on successive Ritz values (0 -> 1e-12) */
  int max_restarts;   /* explicit Lanczos restarts from the Ritz vector (default 0) */
  double cutoff;      /* absolute singular-value cutoff (0 -> 1e-14; <0 -> none) */
  int min_sweeps;     /* sweeps before the stop rule applies (0 -> 2) */
  int device;         /* CUDA device ordinal */
  uint64_t seed;      /* seed for random initial states and Lanczos restarts */
  int svd_method;     /* truncation: 0 = eigen-decomposition of the reduced density matrix
                         (default), 1 = one-sided block Jacobi SVD of theta */
  int precision;      /* H_eff arithmetic: 0 = FP64 (default); 1 = precision form: Lanczos on
                         split-BF16 matvecs (tcgen05 tensor cores, FP32 accumulation), then
                         refined with FP64 matvecs from the Ritz vector; energies are FP64 */
  int single_site;    /* 0 = two-site sweeps (default); 1 = single-site sweeps, the reference's
                         dmrg-gpu driver (gpu-rocm/dmrg-gpu/src/dmrg_gpu_impl.h:1119-1450):
                         bond dimensions stay at those of the initial MPS (or shrink) */
  int truncation;     /* 0 = warm-started subspace split (default): on a sweep that repeats
                         the previous sweep's bond cap (cap <= 512 for real data, <= 256 for
                         complex data), a bond keeps its dimension, and the kept space
                         comes from three power steps on theta starting from the MPS factor
                         next to it (unit columns, orthonormalised by CholeskyQR; complex
                         blocks on their real embedding). It is exact for that space. The
                         first sweep at a cap, a bond below the cap whose discarded weight
                         exceeds the exact split's threshold, or one where CholeskyQR gives
                         up, takes the exact split of svd_method.
                         1 = the exact split on every bond
                         2 = randomised split (the reference's RSVD option, dmrg2_gpu_impl.h:
                         1178-1266): r = k + 10 random sketch columns on the side that takes
                         the isometry, shifted CholeskyQR3, the density-matrix split of the
                         r-row projection; where full_k > k + 10 and that side is longer than
                         2k (and r <= 512 real / 256 complex), the exact split elsewhere.
                         Approximate: its discarded weight is at least the exact split's */
} dmrg2_config;

/* One row per sweep (left-to-right + right-to-left half sweep). */
typedef struct dmrg2_sweep_report {
  int sweep;
  int chi_max;             /* bond dimension cap of this sweep */
  double energy;           /* eigenvalue of the last bond optimised */
  double trunc_err_max;    /* largest discarded weight of any bond */
  double trunc_err_sum;    /* summed discarded weight over the sweep */
  int max_bond;            /* largest bond dimension after the sweep */
  double wall_s;           /* host wall time of the sweep */
  long long matvecs;       /* H_eff applications */
  double heff_s;           /* device time inside the H_eff contractions */
  double heff_flops;       /* algorithmic real flops of those contractions */
  long long lanczos_iters; /* Krylov vectors built */
  int lanczos_unconverged; /* bonds whose Lanczos hit the Krylov cap */
  double svd_s;            /* device time of the SVD truncations */
  int jacobi_sweeps_max;
  double device_s;         /* device time of the whole sweep (CUDA events on the solver stream) */
  long long lowprec_matvecs; /* precision form: matvecs on the split-BF16 operator */
  int warm_splits;           /* bonds split by the warm-started subspace truncation */
  int warm_fallbacks;        /* bonds where it gave up and the exact split ran */
  int eig_fallbacks;         /* bonds whose density-matrix eigenvectors could not be made
                                orthonormal, split by the one-sided Jacobi SVD instead */
  int warm_short;            /* warm splits kept after one power half-step (of warm_splits) */
  int rsvd_splits;           /* bonds split by the randomised split (truncation 2) */
  int rsvd_fallbacks;        /* bonds where it could not orthonormalise its sketch */
  int phase;                 /* 0 = sweep (dmrg2_run / dmrg2_resume); dmrg2_pdmrg_run: 1 = warm-up
                                sweep, 2 = outer iteration, 3 = recalibration sweep, 4 = polish */
  int device_loops;          /* Lanczos solves (restarts counted) run as one cached CUDA graph
                                whose conditional loop iterates the Krylov steps on the device
                                (the rest: host-driven, e.g. the first solve of each bond shape) */
} dmrg2_sweep_report;

/* ---------------------------------------------------------------- solver */

/* DMRG2GPU<Scalar>::DMRG2GPU(L, d, chi_max, D_mpo, tol)  (dmrg2_gpu.h:30) */
int dmrg2_create(const dmrg2_config* cfg, dmrg2_handle** out);
/* DMRG2GPU<Scalar>::~DMRG2GPU()  (dmrg2_gpu_impl.h:265-343) */
void dmrg2_destroy(dmrg2_handle* h);

/* DMRG2GPU<Scalar>::set_mpo(const std::vector<Scalar*>&)  (dmrg2_gpu.h:38, impl:436-485).
 * ROWMAJOR: Dl/Dr hold the per-site MPO bonds. REFERENCE: Dl points to the single
 * padded D_mpo and Dr is ignored. Host buffers are copied; the caller keeps them. */
int dmrg2_set_mpo(dmrg2_handle* h, const void* const* W, const int* Dl, const int* Dr, int layout);

/* Load an MPS (no reference counterpart: the reference only has the initialisers
 * below). bond_dims has L+1 entries with bond_dims[0] = bond_dims[L] = 1. */
int dmrg2_set_mps(dmrg2_handle* h, const void* const* A, const int* bond_dims, int layout);

/* DMRG2GPU<Scalar>::initialize_mps_random / _product / _neel  (dmrg2_gpu.h:34-36,
 * impl:383-429). Random entries are 0.1*U[-1,1] from the seeded generator. */
int dmrg2_init_mps(dmrg2_handle* h, int kind, uint64_t seed);

/* DMRG2GPU<Scalar>::run(n_sweeps)  (dmrg2_gpu.h:32, impl:1427-1457).
 * chi_schedule[s] is the bond cap of sweep s (NULL: chi_max for every sweep).
 * Up to max_out reports are written; *n_out receives the number of sweeps run. */
int dmrg2_run(dmrg2_handle* h, const int* chi_schedule, int n_sweeps, dmrg2_sweep_report* out,
              int max_out, int* n_out);

/* Continue sweeping from the state left by the last dmrg2_run or dmrg2_resume
 * (environments are kept; no stop rule). No reference counterpart: the reference
 * run() always rebuilds environments (impl:1427-1436). */
int dmrg2_resume(dmrg2_handle* h, const int* chi_schedule, int n_sweeps, dmrg2_sweep_report* out,
                 int max_out, int* n_out);

/* Parallel (segmented) DMRG: PDMRGGPU<Scalar>(L, d, chi_max, D_mpo, n_segments, tol) and
 * PDMRGGPU::run(n_outer, n_local, n_warmup, n_polish, n_recal) (gpu-rocm/pdmrg-gpu/src/
 * pdmrg_gpu.h:24-40, pdmrg_gpu_impl.h:2585-2760). The handle's tol is the outer stop rule.
 * Warm-up, recalibration and polish sweeps are full-chain two-site sweeps at chi (the
 * reference's warm-up and polish are single-site). One report per full sweep and per
 * outer iteration (phase); the final MPS is right-canonical (dmrg2_get_mps). */
typedef struct dmrg2_pdmrg_options {
  int n_segments; /* >= 2, each segment >= 2 sites */
  int n_outer;    /* outer iterations (reference default 20) */
  int n_local;    /* local iterations per outer one (2) */
  int n_warmup;   /* full-chain sweeps first (1; at least 1: its left-to-right half builds
                     the left environments the segments start from) */
  int n_polish;   /* full-chain sweeps at the end unless the outer loop converged (0) */
  int n_recal;    /* a full-chain sweep every n_recal outer iterations (0 = never) */
  int chi;        /* bond cap, <= chi_max (0 = chi_max) */
} dmrg2_pdmrg_options;
int dmrg2_pdmrg_run(dmrg2_handle* h, const dmrg2_pdmrg_options* opt, dmrg2_sweep_report* out, int max_out,
                    int* n_out);

/* get_energy() (dmrg2_gpu.h:40) */
int dmrg2_get_energy(const dmrg2_handle* h, double* energy);
/* seconds spent right-canonicalising and building environments in the last run
 * (the reference's env_build_sec, impl:1428-1436) */
int dmrg2_get_env_build_seconds(const dmrg2_handle* h, double* seconds);
/* chi_L / chi_R (dmrg2_gpu.h:42-43): all L+1 bond dimensions */
int dmrg2_get_bond_dims(const dmrg2_handle* h, int* bond_dims);
/* get_mps (dmrg2_gpu.h:41, impl:1464-1472): out[i] must hold
 * bond_dims[i]*d*bond_dims[i+1] scalars. */
int dmrg2_get_mps(dmrg2_handle* h, void* const* out, int layout);
/* <psi|O_i|psi>/<psi|psi> for every site (no reference counterpart on the GPU
 * path; the oracle computes it from the final MPS). re/im hold L doubles. */
int dmrg2_expect_local(dmrg2_handle* h, const void* op, double* re, double* im);
/* device memory held by the handle */
int dmrg2_get_device_bytes(const dmrg2_handle* h, size_t* bytes);

/* Message of the last failed call on h (h may be NULL for create and op calls). */
const char* dmrg2_last_error(const dmrg2_handle* h);
int dmrg2_abi_version(void);
/* number of CUDA kernels this library has launched in this process */
long long dmrg2_get_launch_count(void);

/* ---------------------------------------------------------------- ops
 * One GPU launch sequence per call on host buffers (copied in and out), for
 * parity tests and for callers that drive their own sweep. Shapes and
 * conventions follow the numpy primitives they replace. */

/* apply_heff(L, R, W_left, W_right, theta)  (cpu/pdmrg/pdmrg/numerics/effective_ham.py:21-81;
 * GPU: apply_heff_two_site, dmrg2_gpu_impl.h:607-780)
 *   L (cL, Dl, cL), R (cR, Dr, cR), WL (Dl, Dm, d, d), WR (Dm, Dr, d, d),
 *   theta/out (cL, d, d, cR). */
int dmrg2_op_heff(int dtype, int cL, int cR, int d, int Dl, int Dm, int Dr, const void* L,
                  const void* R, const void* WL, const void* WR, const void* theta, void* out);

/* update_left_env(L, A, W)  (cpu/pdmrg/pdmrg/environments/update.py:16-80; GPU: impl:787-860)
 *   L (cL, Dl, cL), A (cL, d, cO), W (Dl, Dr, d, d) -> out (cO, Dr, cO) */
int dmrg2_op_env_left(int dtype, int cL, int cO, int d, int Dl, int Dr, const void* L,
                      const void* A, const void* W, void* out);

/* update_right_env(R, B, W)  (update.py:83-127; GPU: impl:867-934)
 *   R (cI, Dr, cI), B (cO, d, cI), W (Dl, Dr, d, d) -> out (cO, Dl, cO) */
int dmrg2_op_env_right(int dtype, int cI, int cO, int d, int Dl, int Dr, const void* R,
                       const void* B, const void* W, void* out);

/* truncated_svd(M, max_bond, cutoff)  (cpu/pdmrg/pdmrg/numerics/accurate_svd.py:82-110;
 * GPU: svd_split, impl:1167-1343). M is m x n row-major. direction 'R' returns
 * left = U (m x k, isometric) and right = S*Vh (k x n); 'L' returns left = U*S
 * and right = Vh (isometric rows). S receives the min(m,n) singular values in
 * descending order. left/right must hold m*min(m,n) and min(m,n)*n scalars.
 * 'R'/'L' use the density-matrix eigensolver (singular values below ~1e-7 of
 * the largest are resolved only as zero); 'r'/'l' use the one-sided block
 * Jacobi SVD (full relative accuracy). */
int dmrg2_op_svd(int dtype, int m, int n, const void* M, int max_bond, double cutoff,
                 char direction, double* S, void* left, void* right, int* k,
                 double* trunc_err);

/* optimize_two_site(L, R, W_left, W_right, theta0)  (cpu/pdmrg/pdmrg/numerics/eigensolver.py:13-63;
 * GPU: lanczos_eigensolver, impl:971-1160). theta is the start vector on entry
 * and the normalised ground state on exit. */
/* The warm-started subspace split of the engine (dmrg2_config.truncation = 0) on one
 * matrix, real data: M (m x n, row-major) split at rank k (k < min(m, n), k <= 512)
 * from an orthonormal factor `warm` of a previous split, k x n rows (dir 'R') or m x k
 * columns (dir 'L'). Three CholeskyQR-orthonormalised power steps; 'R': left (m x k)
 * isometric columns, right = left^T M; 'L': right (k x n) isometric rows, left =
 * M right^T; trunc_err = |M|^2 - |kept factor|^2. DMRG2_ERR_NUMERIC when CholeskyQR
 * gives up (then the engine takes the exact split). Replaces, with svd_split's
 * truncation, the reference's gesvd step (gpu-rocm/dmrg2-gpu/src/dmrg2_gpu_impl.h:1167-1343)
 * on sweeps that repeat the bond cap. */
int dmrg2_op_warm_split(int dtype, int m, int n, const void* M, const void* warm, int k, char direction,
                        void* left, void* right, double* trunc_err);

int dmrg2_op_lanczos(int dtype, int cL, int cR, int d, int Dl, int Dm, int Dr, const void* L,
                     const void* R, const void* WL, const void* WR, void* theta, int krylov_max,
                     double tol, int max_restarts, double* energy, int* iters);

/* C = alpha*op(A)*op(B) + beta*C on the FP64 tensor cores (row-major; test hook
 * for the contraction kernel). trans: 0 = N, 1 = T, 2 = C (conjugate transpose),
 * 3 = R (conjugate, no transpose; A only). alpha/beta are (re, im) pairs. */
int dmrg2_op_gemm(int dtype, int transA, int transB, int M, int N, int K, const double* alpha,
                  const void* A, long long lda, const void* B, long long ldb, const double* beta,
                  void* C, long long ldc);

/* The same product computed by the precision form: each operand split into three
 * BF16 pieces (x = x1 + x2 + x3), the six leading piece products accumulated in FP32
 * on the tcgen05 tensor cores, the result written in FP64 (complex via the real
 * embedding [[Ar, -Ai], [Ai, Ar]]). Relative error ~1e-7 of sum |a_ik b_kj|. No
 * counterpart in the reference (its GEMMs are FP64 only). transB 2 = conjugate
 * transpose; alpha and beta must be real. */
int dmrg2_op_gemm_bf16x3(int dtype, int transA, int transB, int M, int N, int K, const double* alpha,
                         const void* A, long long lda, const void* B, long long ldb, const double* beta,
                         void* C, long long ldc);

/* apply_heff on DEVICE pointers, allocating no device memory. No counterpart in
 * the reference: its GPU path only applies H_eff inside its own Lanczos loop on
 * buffers it allocated up front. For callers that must not allocate while they
 * run (a solver enqueuing its own loop on a stream, a fixed memory budget): the
 * scratch (fused two-site MPO plus the two contraction intermediates) lives in a
 * static device array of DMRG2_NOALLOC_SCRATCH_BYTES, and shapes that need more
 * are rejected with DMRG2_ERR_ARG before any device work. Shapes and layouts as
 * dmrg2_op_heff; all six arrays are on the current device. Work is enqueued on
 * `stream` (a cudaStream_t; NULL = legacy default stream) and the call returns
 * without synchronising. The first call on each device resolves the scratch
 * address and loads its module; make it before any stream capture. All calls
 * on a device share the one scratch array: calls on the same stream are safe,
 * calls that overlap in time on other streams or threads race. */
#define DMRG2_NOALLOC_SCRATCH_BYTES (64ull << 20)
int dmrg2_op_heff_noalloc(int dtype, int cL, int cR, int d, int Dl, int Dm, int Dr, const void* L,
                          const void* R, const void* WL, const void* WR, const void* theta, void* out,
                          void* stream);

/* ---------------------------------------------------------------- served / batched form
 * A server owns one device and runs many independent ground-state solves at once.
 * No counterpart in the reference, where one DMRG2GPU object runs one solve at a time.
 *
 * Requests are copied at submit. They are admitted in arrival order while one of
 * max_active worker slots is idle and their device footprint fits the budget. The
 * footprint covers the MPS, environments, Krylov space, eigen workspace and
 * contraction scratch, and equals dmrg2_get_device_bytes of the same solve after
 * set_mpo. Each admitted request is solved on its own engine and CUDA stream, so
 * solves that arrive while others run overlap with them on the device (continuous
 * admission; no batch boundary). A request that fits no budget is rejected at
 * submit. */
typedef struct dmrg2_server dmrg2_server;

typedef struct dmrg2_server_config {
  int device;               /* CUDA device ordinal */
  int max_active;           /* solves running at once (0 -> 8) */
  size_t hbm_budget_bytes;  /* admission budget (0 -> 90% of the free device memory at create) */
} dmrg2_server_config;

typedef struct dmrg2_request {
  dmrg2_config cfg;         /* as for dmrg2_create (device is the server's) */
  const void* const* W;     /* L row-major MPO tensors (Dl, Dr, d, d) */
  const int* Dl;            /* L left MPO bonds */
  const int* Dr;            /* L right MPO bonds */
  const void* const* A;     /* initial MPS (L row-major tensors), or NULL */
  const int* bond_dims;     /* L+1 bond dimensions of A */
  int init_kind;            /* dmrg2_init_kind when A is NULL (seeded by cfg.seed) */
  const int* schedule;      /* bond cap per sweep, each in [1, cfg.chi_max] */
  int n_sweeps;             /* length of schedule; the cfg.tol stop rule applies */
} dmrg2_request;

enum dmrg2_request_state {
  DMRG2_REQ_QUEUED = 0,
  DMRG2_REQ_RUNNING = 1,
  DMRG2_REQ_DONE = 2,
  DMRG2_REQ_FAILED = 3
};

typedef struct dmrg2_result {
  int state;                /* dmrg2_request_state */
  int status;               /* dmrg2_status of the solve (set when it finished) */
  double energy;            /* energy of the last sweep */
  int sweeps;               /* sweeps run */
  double trunc_err_max;     /* largest discarded weight of the last sweep */
  int max_bond;
  double device_s;          /* device time of the sweeps (CUDA events on the solve's stream) */
  double t_submit, t_admit, t_done;  /* seconds since dmrg2_server_create */
  size_t footprint_bytes;   /* device bytes reserved at admission */
  char message[256];        /* error message of a failed solve */
} dmrg2_result;

int dmrg2_server_create(const dmrg2_server_config* cfg, dmrg2_server** out);
/* Copies the request and queues it; *id identifies it for dmrg2_server_poll. */
int dmrg2_server_submit(dmrg2_server* s, const dmrg2_request* req, long long* id);
/* State and result of request id. Waits up to wait_ms for it to finish
 * (0: no wait, < 0: until it finishes). */
int dmrg2_server_poll(dmrg2_server* s, long long id, int wait_ms, dmrg2_result* out);
/* Fails queued requests, waits for running solves, frees the server. */
void dmrg2_server_destroy(dmrg2_server* s);

#ifdef __cplusplus
}
#endif

#endif /* DMRG2_B200_H */
