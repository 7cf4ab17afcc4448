"""Oracle fixtures for the full-size configurations (test infrastructure only).

The CPU oracle (``oracle/dmrg2_oracle.py``, the reference's numpy two-site
DMRG restated and pinned by ``make_golden.py``) is run once on each full-size
configuration below, and its per-sweep energies, truncation errors, bond
dimensions and final local observables are written to ``large_<case>.json``.
The GPU tests (``tests/test_gpu_large.py``) rebuild the same MPO and the same
seeded initial MPS and compare against these numbers, so the slow oracle runs
(tens of minutes each on a few host cores) happen here and not in the tests.

Cases (all from seeded synthetic inputs):

* ``xxz48`` / ``xxz100``: Heisenberg XXZ chain, open BC, J=1, Delta=1 (MPO D=5,
  d=2, float64), initial MPS i.i.d. N(0,1) with chi=16 (numpy
  ``default_rng(0)``), chi_max ramped 32 -> 64 -> 128 -> 256 over 12 sweeps
  (3 each), singular-value cutoff 1e-12, every sweep run (no early stop).
  Observable: <S^z_i>.
* ``jos24``: Josephson-junction array in the charge basis, complex128, L=24,
  d=5 (n in -2..2), H = E_C sum (n_i - n_g)^2 - (E_J/2) sum (e^{iA} a_i^+ a_{i+1}
  + h.c.), E_C=1, E_J=2, n_g=0.25, A = 2 pi 0.1 / L (MPO D=4); initial MPS with
  complex Gaussian entries (re, im ~ N(0,1), seed 0) and chi=16; chi_max=128,
  10 sweeps, cutoff 1e-14. Observable: <n_i>.

Usage: ``python tests/golden/make_large_fixtures.py xxz48 [xxz100 jos24]``.
"""

from __future__ import annotations

import json
import os
import platform
import sys
import time
from pathlib import Path

import numpy as np
import scipy

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

from oracle import dmrg2_oracle as O  # noqa: E402
from oracle import models as M  # noqa: E402


def case_inputs(case):
    """(mpo, mps, schedule, cutoff, observable) of a full-size configuration."""
    if case in ("xxz48", "xxz100"):
        L = 48 if case == "xxz48" else 100
        return (M.heisenberg_mpo(L, 1.0, 1.0), O.random_mps(L, 2, 16, seed=0),
                O.ramp_schedule([32, 64, 128, 256], 12), 1e-12, M.SZ)
    if case == "jos24":
        L = 24
        mpo = M.josephson_mpo(L, 2, 2.0, 1.0, 0.25, 2 * np.pi * 0.1 / L, "shifted")
        _, n, _, _ = M.josephson_ops(2)
        return mpo, O.random_mps(L, 5, 16, seed=0, dtype=np.complex128), [128] * 10, 1e-14, n
    raise KeyError(case)


def main(cases):
    for case in cases:
        mpo, mps, sched, cutoff, op = case_inputs(case)
        t0 = time.perf_counter()
        out = O.dmrg2(mpo, mps, sched, cutoff=cutoff, tol=0.0, verbose=True)
        wall = time.perf_counter() - t0
        obs = O.expect_local(out["mps"], op)
        rec = {
            "case": case,
            "L": len(mpo),
            "schedule": sched,
            "cutoff": cutoff,
            "energies": [float(e) for e in out["energies"]],
            "trunc_err_max": [float(t) for t in out["trunc_err_max"]],
            "trunc_err_sum": [float(t) for t in out["trunc_err_sum"]],
            "max_bond": [int(b) for b in out["max_bond"]],
            "bond_dims": [1] + [int(a.shape[2]) for a in out["mps"]],
            "observable": [float(x) for x in np.real(obs)],
            "wall_s": wall,
            "sweep_wall_s": [float(w) for w in out["wall"]],
            "host": {"cpus": os.cpu_count(), "blas_threads": os.environ.get("OPENBLAS_NUM_THREADS"),
                     "numpy": np.__version__, "scipy": scipy.__version__,
                     "python": platform.python_version()},
        }
        (HERE / f"large_{case}.json").write_text(json.dumps(rec, indent=1) + "\n")
        print(f"{case}: E={rec['energies'][-1]:.14f} in {wall:.0f} s", flush=True)


if __name__ == "__main__":
    main(sys.argv[1:] or ["xxz48", "xxz100", "jos24"])
