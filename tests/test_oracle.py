"""The CPU oracle against the reference's golden vectors and known answers.

* primitives vs outputs of the reference's own numpy modules
  (tests/golden/ref_primitives.npz, made by tests/golden/make_golden.py);
* the oracle sweep vs the reference sweep loop (tests/golden/ref_dmrg.json);
* MPO builders vs exact diagonalisation of the same Hamiltonian;
* the known-answer energies of gpu-rocm/dmrg2-gpu/src/test_dmrg2_gpu.cpp.
"""
import json

import numpy as np
import pytest

from oracle import models as M
from oracle import dmrg2_oracle as O

TAGS = ["r0", "r1", "r2", "c0", "c1"]


@pytest.fixture(scope="module")
def prim(golden_dir):
    return np.load(golden_dir / "ref_primitives.npz")


@pytest.mark.parametrize("tag", TAGS)
def test_apply_heff_matches_reference(prim, tag):
    g = lambda k: prim[f"{tag}_{k}"]
    out = O.apply_heff(g("L"), g("R"), g("WL"), g("WR"), g("theta"))
    np.testing.assert_allclose(out, g("heff"), rtol=0, atol=1e-12 * np.abs(g("heff")).max())


@pytest.mark.parametrize("tag", TAGS)
def test_env_updates_match_reference(prim, tag):
    g = lambda k: prim[f"{tag}_{k}"]
    le = O.update_left_env(g("L"), g("A"), g("WL"))
    re = O.update_right_env(g("R"), g("B"), g("WR"))
    np.testing.assert_allclose(le, g("lenv"), atol=1e-12 * np.abs(g("lenv")).max())
    np.testing.assert_allclose(re, g("renv"), atol=1e-12 * np.abs(g("renv")).max())


@pytest.mark.parametrize("tag", TAGS)
def test_truncated_svd_matches_reference(prim, tag):
    M_ = prim[f"{tag}_M"]
    U, S, Vh, te = O.truncated_svd(M_, max(1, min(M_.shape) - 2))
    np.testing.assert_allclose(S, prim[f"{tag}_svd_S"], rtol=1e-12)
    assert abs(te - float(prim[f"{tag}_svd_te"])) <= 1e-12 * max(1.0, te)
    np.testing.assert_allclose(U.conj().T @ U, np.eye(len(S)), atol=1e-12)


def test_sweep_matches_reference_fixture(golden_dir):
    ref = json.loads((golden_dir / "ref_dmrg.json").read_text())["heis_L12_fixture"]
    mpo = O.load_npz_mpo(golden_dir / "heis_L12_mpo.npz")
    mps = O.load_npz_mps(golden_dir / "heis_L12_mps.npz")
    r = O.dmrg2(mpo, mps, [20] * 4, min_sweeps=4, tol=0)
    for e, er in zip(r["energies"], ref["ref_sweep_chi20"]):
        assert abs(e - er) <= 1e-10 * abs(er)
    # quimb DMRG2 golden energy of the same fixture (benchmark_data golden_results.json)
    assert abs(r["energy"] - ref["quimb_dmrg2_energy"]) <= 1e-10 * abs(ref["quimb_dmrg2_energy"])


@pytest.mark.parametrize("key,build", [
    ("heis_L12_seed0_chi32", lambda: (M.heisenberg_mpo(12), O.random_mps(12, 2, 8, 0))),
    ("xxz_L10_d07_seed1_chi16", lambda: (M.heisenberg_mpo(10, 1.0, 0.7), O.random_mps(10, 2, 4, 1))),
    ("jos_L6_nmax1_seed2_chi16", lambda: (M.josephson_mpo(6), O.random_mps(6, 3, 4, 2, np.complex128))),
    ("j1j2_L10_seed3_chi24", lambda: (M.j1j2_mpo(10, 1.0, 0.3), O.random_mps(10, 2, 4, 3))),
])
def test_sweeps_match_reference_loop(golden_dir, key, build):
    ref = json.loads((golden_dir / "ref_dmrg.json").read_text())[key]
    mpo, mps = build()
    r = O.dmrg2(mpo, mps, [ref["chi"]] * ref["sweeps"], min_sweeps=ref["sweeps"], tol=0)
    # converged sweeps agree to the eigensolver tolerance
    e_ref = ref["ref_sweep"][-1]
    assert abs(r["energies"][-1] - e_ref) <= 1e-9 * abs(e_ref)


MODELS = [
    ("heis", lambda L: M.heisenberg_mpo(L, 1.0, 0.7), lambda L: M.ham_heisenberg(L, 1.0, 0.7), 6),
    ("tfim", lambda L: M.tfim_mpo(L, 1.0, 0.8), lambda L: M.ham_tfim(L, 1.0, 0.8), 6),
    ("jos_ref", lambda L: M.josephson_mpo(L), lambda L: M.ham_josephson(L), 4),
    ("jos_shift", lambda L: M.josephson_mpo(L, 2, 2.0, 1.0, 0.25, 0.26, "shifted"),
     lambda L: M.ham_josephson(L, 2, 2.0, 1.0, 0.25, 0.26, "shifted"), 4),
    ("j1j2", lambda L: M.j1j2_mpo(L, 1.0, 0.35), lambda L: M.ham_longrange(L, [1.0, 0.35]), 6),
    ("j1j2j3", lambda L: M.j1j2j3_mpo(L), lambda L: M.ham_longrange(L, [1.0, 0.4, 0.2]), 6),
    ("ladder", lambda L: M.ladder_mpo(L), lambda L: M.ham_ladder(L), 3),
]


@pytest.mark.parametrize("name,mpo,ham,L", MODELS)
def test_mpo_equals_hamiltonian(name, mpo, ham, L):
    np.testing.assert_allclose(M.mpo_to_dense(mpo(L)), ham(L).toarray(), atol=1e-13)


# gpu-rocm/dmrg2-gpu/src/test_dmrg2_gpu.cpp:208-211,294-297,344,388-392,440-444
KATS = [
    (lambda: M.ham_heisenberg(4), -1.616025403784, 1e-10),
    (lambda: M.ham_heisenberg(8), -3.374932598688, 1e-10),
    (lambda: M.ham_josephson(4), -1.053346829927396, 1e-10),
    (lambda: M.ham_josephson(6), -1.748843818181493, 1e-10),
    (lambda: M.ham_longrange(4, [1.0, 0.5]), -1.5, 1e-10),
    (lambda: M.ham_longrange(6, [1.0, 0.5]), -2.25, 1e-10),
    (lambda: M.ham_longrange(8, [1.0, 0.5]), -3.0, 1e-10),
    (lambda: M.ham_longrange(6, [1.0, 0.4, 0.2]), -2.3229239173, 1e-8),
    (lambda: M.ham_longrange(8, [1.0, 0.4, 0.2]), -3.1205086380, 1e-8),
    (lambda: M.ham_longrange(8, [1.0, 0.5, 0.25]), -3.0690408638, 1e-8),
    (lambda: M.ham_ladder(2), -2.0, 1e-10),
    (lambda: M.ham_ladder(3), -3.1293852415718166, 1e-8),
    (lambda: M.ham_ladder(4), -4.2930664566945656, 1e-8),
]


@pytest.mark.parametrize("i", range(len(KATS)))
def test_known_answer_energies(i):
    ham, E, tol = KATS[i]
    assert abs(M.ground_energy(ham()) - E) < tol


def test_oracle_dmrg_reaches_ed():
    """Exact MPS (chi=64 at L=12) reproduces ED to 1e-12."""
    L = 12
    r = O.dmrg2(M.heisenberg_mpo(L), O.random_mps(L, 2, 8, 0), [64] * 6)
    e_ed = M.ground_energy(M.ham_heisenberg(L))
    assert abs(r["energy"] - e_ed) <= 1e-12 * abs(e_ed)


def test_oracle_observables_match_ed():
    L = 8
    H = M.ham_josephson(L, 1, 1.0, 0.5, 0.1, 0.3)
    e, v = M.ground_state(H)
    r = O.dmrg2(M.josephson_mpo(L, 1, 1.0, 0.5, 0.1, 0.3), O.random_mps(L, 3, 4, 5, np.complex128), [81] * 6)
    assert abs(r["energy"] - e) < 1e-10
    _, n, _, _ = M.josephson_ops(1)
    nd = O.expect_local(r["mps"], n)
    ned = [np.vdot(v, M._site_op(n, i, L, 3) @ v).real for i in range(L)]
    np.testing.assert_allclose(nd.real, ned, atol=1e-8)


def test_single_site_oracle_reaches_ed_at_exact_bond_dimension():
    """Single-site sweeps (the reference's dmrg-gpu algorithm) from a full-rank
    random MPS: at an exact bond dimension the energy is the ED ground energy."""
    L = 8
    mpo = M.heisenberg_mpo(L)
    res = O.dmrg1(mpo, O.random_mps(L, 2, 16, seed=3), [16] * 8, cutoff=0.0)
    e_ed = M.ground_energy(M.ham_heisenberg(L))
    assert abs(res["energy"] - e_ed) < 1e-10 * abs(e_ed)
    # the MPS it returns has that energy
    assert abs(O.mpo_expectation(res["mps"], mpo).real / O.mps_norm2(res["mps"]).real - e_ed) < 1e-9


def test_single_site_heff_matches_dense():
    rng = np.random.default_rng(4)
    cL, d, cR, D = 3, 2, 4, 5
    Lenv, Renv = rng.standard_normal((cL, D, cL)), rng.standard_normal((cR, D, cR))
    W, A = rng.standard_normal((D, D, d, d)), rng.standard_normal((cL, d, cR))
    ref = np.einsum("awc,cse,wvst,fve->atf", Lenv, A, W, Renv)
    np.testing.assert_allclose(O.apply_heff1(Lenv, Renv, W, A), ref, atol=1e-12)
