"""Parallel (segmented) DMRG, the reference's pdmrg-gpu driver (gpu-rocm/pdmrg-gpu/src/
pdmrg_gpu_impl.h:2320-2760), against exact diagonalisation.

The reference's own tests (test_pdmrg_gpu.cpp:196-245) run Heisenberg L=8 chi=32 with two
segments, 20 outer and 2 local iterations and one warm-up sweep, and require the energy to
1e-10 of the exact value (-3.374932598688 at L=8, -6.911737145575 at L=16). The same
settings run here through dmrg2_pdmrg_run, plus three and four segments (odd boundaries),
a complex Josephson chain, and the final MPS: right-canonical, with <H> equal to the
reported energy.
"""
import numpy as np
import pytest

import dmrg2
from oracle import dmrg2_oracle as O, models as M

pytestmark = pytest.mark.gpu


def pdmrg_run(mpo, mps, chi, n_segments, **kw):
    L, d = len(mpo), mpo[0].shape[2]
    cplx = np.iscomplexobj(mpo[0]) or np.iscomplexobj(mps[0])
    eng = dmrg2.PDMRGGPU(L, d, chi, n_segments=n_segments, tol=1e-10,
                         dtype=np.complex128 if cplx else np.float64, krylov_max=30, max_restarts=2,
                         cutoff=1e-14)
    eng.set_mpo(mpo)
    eng.set_mps(mps)
    e = eng.run(**kw)
    return eng, e


def check_state(eng, mpo, e):
    A = eng.get_mps()
    for k in range(1, len(A)):
        a = A[k].reshape(A[k].shape[0], -1)
        np.testing.assert_allclose(a @ a.conj().T, np.eye(a.shape[0]), atol=1e-12)
    assert abs(O.mpo_expectation(A, mpo).real - e) < 1e-8


@pytest.mark.parametrize("L,chi,P,exact", [(8, 32, 2, -3.374932598688), (16, 128, 2, -6.911737145575),
                                           (16, 128, 4, -6.911737145575)])
def test_pdmrg_heisenberg_matches_exact(L, chi, P, exact):
    mpo = M.heisenberg_mpo(L)
    eng, e = pdmrg_run(mpo, O.random_mps(L, 2, 8, seed=0), chi, P, n_outer_sweeps=20, n_local_sweeps=2,
                       n_warmup=1)
    rep = eng.reports
    outer = [r for r in rep if r["phase"] == 2]
    print(L, P, "E", e, "outer iterations", len(outer), "matvecs", sum(r["matvecs"] for r in rep))
    assert [r["phase"] for r in rep][:1] == [1] and len(outer) >= 1
    assert abs(e - exact) < 1e-10
    check_state(eng, mpo, e)


def test_pdmrg_three_segments_odd_boundaries_matches_ed():
    """L=12 in three segments: boundaries 0 (even) and 1 (odd) both merge."""
    L = 12
    mpo = M.heisenberg_mpo(L, delta=0.7)
    ed = M.ground_energy(M.ham_heisenberg(L, delta=0.7))
    eng, e = pdmrg_run(mpo, O.random_mps(L, 2, 8, seed=4), 64, 3, n_outer_sweeps=30, n_local_sweeps=2,
                       n_warmup=1)
    print("L=12 P=3 E", e, "ED", ed)
    assert abs(e - ed) < 1e-10
    check_state(eng, mpo, e)


def test_pdmrg_josephson_complex_matches_ed():
    L = 8
    mpo = M.josephson_mpo(L, n_max=1, E_J=2.0, E_C=1.0, n_g=0.25, phi=0.3, onsite="shifted")
    ed = M.ground_energy(M.ham_josephson(L, n_max=1, E_J=2.0, E_C=1.0, n_g=0.25, phi=0.3, onsite="shifted"))
    eng, e = pdmrg_run(mpo, O.random_mps(L, 3, 8, 1, np.complex128), 81, 2, n_outer_sweeps=30,
                       n_local_sweeps=2, n_warmup=1)
    print("Josephson L=8 P=2 E", e, "ED", ed)
    assert abs(e - ed) < 1e-10
    check_state(eng, mpo, e)


def test_pdmrg_polish_and_recalibration_run():
    """n_recal and n_polish insert full-chain sweeps (phases 3 and 4) and keep the energy."""
    L = 16
    mpo = M.heisenberg_mpo(L)
    eng, e = pdmrg_run(mpo, O.random_mps(L, 2, 8, seed=2), 128, 4, n_outer_sweeps=4, n_local_sweeps=1,
                       n_warmup=1, n_polish=2, n_recal=2)
    phases = [r["phase"] for r in eng.reports]
    print("phases", phases, "E", e)
    assert 3 in phases and phases[-1] in (2, 4)
    assert abs(e - (-6.911737145575)) < 1e-8
    check_state(eng, mpo, e)


def test_pdmrg_needs_a_warmup_sweep():
    L = 8
    eng = dmrg2.PDMRGGPU(L, 2, 16, n_segments=2)
    eng.set_mpo(M.heisenberg_mpo(L))
    eng.set_mps(O.random_mps(L, 2, 4, seed=0))
    with pytest.raises(dmrg2.Dmrg2Error):
        eng.run(n_outer_sweeps=2, n_warmup=0)
