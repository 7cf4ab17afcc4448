"""Served / batched form (dmrg2_server_*) on the GPU.

The bar: every request gives the same result when it runs alone and when it
runs in a mix with others (energy to 1e-12 relative: each solve is
deterministic and has its own engine, stream and buffers); requests that
arrive while others run are admitted and overlap with them; admission respects
the device-memory budget; a failing request does not disturb the others.
"""
import time

import numpy as np
import pytest

import dmrg2
from oracle import dmrg2_oracle as O
from oracle import models as M

pytestmark = pytest.mark.gpu


def requests():
    """A mixed stream: XXZ chains of several L and Delta, J1-J2 (D=8), complex Josephson."""
    rng = np.random.default_rng(11)
    out = []
    for L, delta in [(12, 0.7), (16, 1.0), (20, 1.3), (24, 0.9)]:
        out.append(dict(mpo=M.heisenberg_mpo(L, delta=delta), schedule=[16, 32, 32, 32],
                        mps=O.random_mps(L, 2, 8, seed=int(rng.integers(1 << 30)))))
    out.append(dict(mpo=M.j1j2_mpo(16, 1.0, float(rng.uniform(0, 0.5))), schedule=[16, 32, 32, 32],
                    mps=O.random_mps(16, 2, 8, seed=3)))
    out.append(dict(mpo=M.josephson_mpo(8, n_max=1, E_J=2.0, E_C=1.0, n_g=0.25, phi=0.3, onsite="shifted"),
                    schedule=[16, 24, 24], mps=O.random_mps(8, 3, 6, seed=5, dtype=np.complex128)))
    return out


def submit_all(srv, reqs):
    return [srv.submit(r["mpo"], r["schedule"], mps=r["mps"], tol=1e-300, min_sweeps=100) for r in reqs]


@pytest.fixture(scope="module")
def alone():
    reqs = requests()
    res = []
    with dmrg2.Server(max_active=1) as srv:
        for r in reqs:
            rid = srv.submit(r["mpo"], r["schedule"], mps=r["mps"], tol=1e-300, min_sweeps=100)
            res.append(srv.result(rid))
    return reqs, res


def test_served_results_equal_alone_and_in_the_mix(alone):
    reqs, ref = alone
    for r in ref:
        assert r["state"] == dmrg2.REQ_DONE, r["message"]
    with dmrg2.Server(max_active=4) as srv:
        ids = submit_all(srv, reqs)
        mix = [srv.result(i) for i in ids]
    for a, b in zip(ref, mix):
        assert b["state"] == dmrg2.REQ_DONE, b["message"]
        assert abs(a["energy"] - b["energy"]) <= 1e-12 * abs(a["energy"])
        assert a["sweeps"] == b["sweeps"] and a["max_bond"] == b["max_bond"]
    # the solves overlapped on the device
    iv = sorted((m["t_admit"], m["t_done"]) for m in mix)
    assert any(iv[k + 1][0] < iv[k][1] for k in range(len(iv) - 1))
    for m in mix:
        assert m["t_submit"] <= m["t_admit"] <= m["t_done"]


def test_served_matches_the_plain_solver(alone):
    reqs, ref = alone
    r = reqs[1]
    eng = dmrg2.DMRG2GPU(len(r["mpo"]), 2, 32, krylov_max=30, max_restarts=2, cutoff=1e-14, tol=1e-300,
                         min_sweeps=100, seed=0)
    eng.set_mpo(r["mpo"])
    eng.set_mps(r["mps"])
    rep = eng.run(schedule=r["schedule"])
    assert abs(rep[-1]["energy"] - ref[1]["energy"]) <= 1e-12 * abs(ref[1]["energy"])
    assert ref[1]["footprint_bytes"] == eng.device_bytes()
    e_ed = M.ground_energy(M.ham_heisenberg(16))
    assert abs(ref[1]["energy"] - e_ed) < 1e-8


def test_admission_respects_the_budget(alone):
    reqs, ref = alone
    budget = int(1.2 * max(r["footprint_bytes"] for r in ref))
    with dmrg2.Server(max_active=4, hbm_budget_bytes=budget) as srv:
        ids = submit_all(srv, reqs[:4])
        res = [srv.result(i) for i in ids]
    running = sorted((r["t_admit"], r["t_done"], r["footprint_bytes"]) for r in res)
    # at every admission the reserved bytes of the overlapping solves fit the budget
    for a, _, fp in running:
        live = sum(f for s, e, f in running if s <= a < e)
        assert live <= budget
    for a, b in zip(ref[:4], res):
        assert abs(a["energy"] - b["energy"]) <= 1e-12 * abs(a["energy"])


def test_failed_request_leaves_the_others_intact(alone):
    reqs, ref = alone
    bad = dict(reqs[0])
    # middle bonds of 50 exceed chi_max = 32 (and cannot be reduced exactly): set_mps fails on the worker
    mps = O.random_mps(len(bad["mpo"]), 2, 50, seed=9)
    with dmrg2.Server(max_active=2) as srv:
        i_bad = srv.submit(bad["mpo"], bad["schedule"], mps=mps, tol=1e-300, min_sweeps=100)
        i_ok = srv.submit(reqs[1]["mpo"], reqs[1]["schedule"], mps=reqs[1]["mps"], tol=1e-300, min_sweeps=100)
        rb, ro = srv.result(i_bad), srv.result(i_ok)
    assert rb["state"] == dmrg2.REQ_FAILED and rb["status"] != 0 and "bond" in rb["message"]
    assert ro["state"] == dmrg2.REQ_DONE
    assert abs(ro["energy"] - ref[1]["energy"]) <= 1e-12 * abs(ref[1]["energy"])
    with dmrg2.Server(max_active=1) as srv:
        with pytest.raises(dmrg2.Dmrg2Error):
            srv.submit(reqs[0]["mpo"], [64], mps=reqs[0]["mps"], chi_max=32)  # schedule above chi_max


def test_destroy_with_queued_requests_returns():
    reqs = requests()[:3]
    srv = dmrg2.Server(max_active=1)
    ids = submit_all(srv, reqs)
    first = srv.poll(ids[0], wait=0.0)
    assert first["state"] in (dmrg2.REQ_QUEUED, dmrg2.REQ_RUNNING, dmrg2.REQ_DONE)
    t = time.perf_counter()
    srv.close()  # running solve finishes, queued ones are dropped
    assert time.perf_counter() - t < 120


def test_complex_request_footprint_matches_the_engine(alone):
    """The admission footprint of the complex Josephson request (its engine holds the
    complex warm-split workspace) equals what an engine of the same configuration
    allocates."""
    reqs, ref = alone
    r = reqs[5]
    eng = dmrg2.DMRG2GPU(len(r["mpo"]), 3, 24, dtype=np.complex128, krylov_max=30, max_restarts=2, cutoff=1e-14,
                         tol=1e-300, min_sweeps=100, seed=0)
    eng.set_mpo(r["mpo"])
    eng.set_mps(r["mps"])
    assert ref[5]["footprint_bytes"] == eng.device_bytes()
