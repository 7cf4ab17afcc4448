// Two-site DMRG engine (host orchestration of the device kernels).
//
// B200-native counterpart of the reference's DMRG2GPU<Scalar> class
// (gpu-rocm/dmrg2-gpu/src/dmrg2_gpu.h:24-203, dmrg2_gpu_impl.h).
#pragma once

#include <memory>
#include <string>
#include <vector>

#include "common.cuh"
#include "kernels.cuh"

namespace dmrg2 {

struct EngineConfig {
  int L = 0;
  int d = 2;
  int chi_max = 32;
  bool complex = false;
  double tol = 1e-10;          // sweep stop rule |dE| < tol (dmrg2_gpu.h:30)
  int krylov_max = 100;        // Lanczos vectors per pass (dmrg2_gpu_impl.h:138: min(100, n))
  double lanczos_tol = 1e-12;  // |dE| between Lanczos steps (dmrg2_gpu_impl.h:976)
  int max_restarts = 0;        // explicit restarts from the Ritz vector
  double cutoff = 1e-14;       // absolute singular-value cutoff (dmrg2_gpu_impl.h:1276)
  int min_sweeps = 2;          // the stop rule applies from the second sweep on
  int jacobi_max_sweeps = 40;
  int svd_method = 0;          // 0: reduced density matrix eigensolver, 1: one-sided block Jacobi
  int precision = 0;           // 0: FP64 matvecs; 1: split-BF16 matvecs on tcgen05, then FP64 refinement
  int single_site = 0;         // 1: single-site sweeps (the reference's dmrg-gpu driver)
  int truncation = 0;          // 0: warm-started subspace split on sweeps that repeat the previous
                               //    sweep's bond cap (real data), exact otherwise; 1: exact always;
                               //    2: randomised split where it applies (full_k > k + 10 and the
                               //    sketched side longer than 2k), exact otherwise
  unsigned seed = 42;
  // cached CUDA graphs for the Lanczos solves and warm splits (also subject to DMRG2_GRAPHS);
  // the server turns them off: with a dozen engines capturing concurrently a capture costs
  // several times its single-engine time and short solves replay too few times to repay it
  bool graphs = true;
};

// Parallel (segmented) sweep, the reference's PDMRGGPU::run(n_outer, n_local, n_warmup,
// n_polish, n_recal) with n_segments from its constructor (gpu-rocm/pdmrg-gpu/src/
// pdmrg_gpu.h:24-40)
struct PdmrgOptions {
  int n_segments = 2;  // P segments, each >= 2 sites
  int n_outer = 20;    // outer iterations (stop when |dE| < tol after one)
  int n_local = 2;     // local iterations per outer one: two staggered half-sweeps and merges each
  int n_warmup = 1;    // full-chain sweeps before the segments start
  int n_polish = 0;    // full-chain sweeps after the outer loop (unless it converged)
  int n_recal = 0;     // a full-chain sweep every n_recal outer iterations (0: none)
  int chi = 0;         // bond cap (0: chi_max)
};

struct SweepStats {
  int sweep = 0;
  int phase = 0;             // 0 sweep; parallel sweep: 1 warm-up, 2 outer iteration, 3 recalibration, 4 polish
  int chi_max = 0;
  double energy = 0.0;
  double trunc_err_max = 0.0;
  double trunc_err_sum = 0.0;
  int max_bond = 0;
  double wall_s = 0.0;
  long long matvecs = 0;
  double heff_s = 0.0;       // device time inside the H_eff contractions
  double heff_flops = 0.0;   // algorithmic flops of those contractions
  long long lanczos_iters = 0;
  int lanczos_unconverged = 0;
  double svd_s = 0.0;
  int jacobi_sweeps_max = 0;
  double device_s = 0.0;     // device time of the whole sweep (CUDA events on the engine stream)
  long long lowprec_matvecs = 0;  // precision form: matvecs on the split-BF16 operator
  int warm_splits = 0;       // bonds split by the warm-started subspace truncation
  int warm_fallbacks = 0;    // bonds where it gave up and the exact split ran
  int warm_short = 0;        // warm splits kept after one power half-step
  int rsvd_splits = 0;       // bonds split by the randomised split
  int rsvd_fallbacks = 0;    // bonds where it gave up and the exact split ran
  int eig_fallbacks = 0;     // bonds where the density-matrix eigenvectors could not be made
                             // orthonormal and the Jacobi SVD split the bond
  int device_loops = 0;      // Lanczos solves run as a device-looped graph (restarts counted)
};

class EngineBase {
 public:
  virtual ~EngineBase() = default;
  virtual void set_mpo(const std::vector<const void*>& W, const std::vector<int>& Dl,
                       const std::vector<int>& Dr) = 0;
  virtual void set_mps(const std::vector<const void*>& A, const std::vector<int>& dims) = 0;
  virtual std::vector<SweepStats> run(const std::vector<int>& schedule) = 0;
  // continue sweeping from the current state (environments kept from the last run)
  virtual std::vector<SweepStats> resume(const std::vector<int>& schedule) = 0;
  // segmented parallel sweeps with boundary merges (see PdmrgOptions)
  virtual std::vector<SweepStats> pdmrg(const PdmrgOptions& opt) = 0;
  virtual void get_mps(std::vector<void*>& out) = 0;
  virtual void expect_local(const void* op, std::vector<double>& re, std::vector<double>& im) = 0;
  virtual double energy() const = 0;
  virtual double env_build_s() const = 0;
  virtual const std::vector<int>& bond_dims() const = 0;
  virtual EngineConfig& config() = 0;
  virtual size_t device_bytes() const = 0;
};

std::unique_ptr<EngineBase> make_engine(const EngineConfig& cfg);

// device bytes an engine with this configuration holds once its MPO is set
// (equals device_bytes() after set_mpo; used for admission by the server)
size_t engine_footprint(const EngineConfig& cfg, const std::vector<int>& Dl, const std::vector<int>& Dr);

}  // namespace dmrg2
