"""Batched configuration: 64 XXZ chains solved together, each against its own plain run.

The chains are the batched workload of bench.py: L drawn from {24, 32, 48, 64},
Delta ~ U[0.5, 1.5], J = 1, chi_max from {64, 128}, seeded N(0,1) chi=16 starts, all
from numpy default_rng(7); each solve ramps chi 16, 32, ... to its chi_max and then
continues at chi_max until |dE| < 1e-10 (at most 8 more sweeps). All 64 run at once
through the server (dmrg2_server_*) in the precision form (split-BF16 tcgen05
matvecs, FP64 refinement), and all 64 again in the plain FP64 form; every chain's
precision-form energy must match its own plain-form energy to 1e-10 relative.
"""
import sys
from pathlib import Path

import numpy as np
import pytest

import dmrg2

REPO = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(REPO))
import bench  # noqa: E402

pytestmark = pytest.mark.gpu


def solve_all(reqs, precision):
    with dmrg2.Server(max_active=12) as srv:
        ids = [srv.submit(r["mpo"], r["schedule"], mps=r["mps"], tol=1e-10, min_sweeps=r["min_sweeps"],
                          krylov_max=bench.KRYLOV, max_restarts=bench.RESTARTS, cutoff=1e-12, precision=precision)
               for r in reqs]
        return [srv.result(i) for i in ids]


def test_batched_chains_precision_form_matches_own_plain_run():
    reqs = bench.batched_requests(64, seed=7)
    split = solve_all(reqs, 1)
    plain = solve_all(reqs, 0)
    rel = []
    for r, a, b in zip(reqs, split, plain):
        assert a["state"] == dmrg2.REQ_DONE, a["message"]
        assert b["state"] == dmrg2.REQ_DONE, b["message"]
        rel.append(abs(a["energy"] - b["energy"]) / abs(b["energy"]))
    rel = np.array(rel)
    print("64 chains: max rel dE (precision vs plain) %.2e, median %.2e" % (rel.max(), np.median(rel)))
    assert rel.max() <= 1e-10
