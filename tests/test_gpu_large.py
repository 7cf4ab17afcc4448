"""Full-size configurations on the GPU against committed oracle fixtures.

The CPU oracle (the reference's numpy two-site DMRG restated, pinned to the
reference by tests/golden/make_golden.py) was run once on each configuration by
tests/golden/make_large_fixtures.py; its per-sweep energies, truncation errors
and final local observables are in tests/golden/large_<case>.json. Here the GPU
engine runs the same MPO, the same seeded initial MPS and the same schedule
through the C ABI, every sweep run (no early stop), and is compared with them:

* xxz48 / xxz100: Heisenberg XXZ L=48 and L=100, Delta=1, chi 32 -> 64 -> 128 ->
  256 over 12 sweeps, cutoff 1e-12; final energy to 1e-10 relative, truncation
  error to 1e-8, <S^z_i> to 1e-8 (plain FP64 form);
* jos24: Josephson array L=24, d=5, complex128, chi=128, 10 sweeps; final energy
  to 1e-10 relative, truncation error and <n_i> to 1e-8; the precision form on the
  same inputs to 1e-10 relative in energy, its <n_i> error against the fixture
  stated (1e-6: an energy-converged Lanczos certifies the vector only to about
  sqrt(1e-12); measured 2.9e-7 to 7.2e-7 depending on the FP64 GEMM configurations).
"""
import json
import sys
from pathlib import Path

import numpy as np
import pytest

import dmrg2

REPO = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(REPO / "tests" / "golden"))
from make_large_fixtures import case_inputs  # noqa: E402

pytestmark = pytest.mark.gpu
GOLDEN = REPO / "tests" / "golden"


def fixture(case):
    p = GOLDEN / f"large_{case}.json"
    if not p.exists():
        pytest.fail(f"missing oracle fixture {p.name}: run tests/golden/make_large_fixtures.py {case}")
    return json.loads(p.read_text())


def run_case(case, **kw):
    mpo, mps, sched, cutoff, op = case_inputs(case)
    L, d = len(mpo), mpo[0].shape[2]
    cplx = np.iscomplexobj(mpo[0]) or np.iscomplexobj(mps[0])
    eng = dmrg2.DMRG2GPU(L, d, max(sched), dtype=np.complex128 if cplx else np.float64, krylov_max=30,
                         max_restarts=2, cutoff=cutoff, tol=1e-300, min_sweeps=len(sched) + 1, **kw)
    eng.set_mpo(mpo)
    eng.set_mps(mps)
    rep = eng.run(schedule=sched)
    return eng, rep, op


@pytest.mark.parametrize("case", ["xxz48", "xxz100", "jos24"])
def test_full_size_vs_oracle(case):
    fx = fixture(case)
    eng, rep, op = run_case(case)
    assert len(rep) == len(fx["energies"])
    E, Er = rep[-1]["energy"], fx["energies"][-1]
    print(case, "E_gpu", E, "E_oracle", Er, "rel", abs(E - Er) / abs(Er),
          "trunc", rep[-1]["trunc_err_max"], fx["trunc_err_max"][-1],
          "warm splits", [r["warm_splits"] for r in rep])
    assert abs(E - Er) <= 1e-10 * abs(Er)
    assert abs(rep[-1]["trunc_err_max"] - fx["trunc_err_max"][-1]) <= 1e-8
    obs = np.asarray(eng.expect_local(op)).real
    err = np.abs(obs - np.asarray(fx["observable"])).max()
    print(case, "max |d obs|", err)
    assert err <= 1e-8
    eng.close()


def test_full_size_josephson_precision_form_vs_oracle():
    fx = fixture("jos24")
    eng, rep, op = run_case("jos24", precision=1)
    assert sum(r["lowprec_matvecs"] for r in rep) > 0
    E, Er = rep[-1]["energy"], fx["energies"][-1]
    err = np.abs(np.asarray(eng.expect_local(op)).real - np.asarray(fx["observable"])).max()
    print("jos24 precision form: rel dE", abs(E - Er) / abs(Er), "max |d n|", err)
    assert abs(E - Er) <= 1e-10 * abs(Er)
    assert err <= 1e-6
    eng.close()
