"""Generate the golden fixtures that pin the oracle to the reference.

Run this where the reference checkout is available (it is NOT needed at test
time):

    python tests/golden/make_golden.py /path/to/dmrg-implementations

It imports the reference's own numpy two-site primitives by file path (the
package ``__init__`` pulls in quimb, which is not needed for these modules):

* cpu/pdmrg/pdmrg/numerics/effective_ham.py   (apply_heff)
* cpu/pdmrg/pdmrg/numerics/eigensolver.py     (optimize_two_site)
* cpu/pdmrg/pdmrg/numerics/accurate_svd.py    (truncated_svd)
* cpu/pdmrg/pdmrg/environments/update.py      (update_left_env / update_right_env)

and writes:

* ``ref_primitives.npz``  seeded inputs and the reference outputs of every primitive,
                           real and complex, several shapes;
* ``ref_dmrg.json``        energies of the reference sweep loop
                           (test_numerics.py:230-287 structure) on the L=12
                           Heisenberg fixture and on seeded synthetic chains;
* ``heis_L12_mpo.npz`` / ``heis_L12_mps.npz``  copies of the reference's
                           ``benchmark_data/regular/heisenberg/L12_D20`` fixture,
                           with its quimb golden energies in ``ref_dmrg.json``.
"""

from __future__ import annotations

import importlib.util
import json
import shutil
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
sys.path.insert(0, str(REPO))

from oracle import models  # noqa: E402
from oracle.dmrg2_oracle import random_mps, right_canonicalize  # noqa: E402


def load_reference(ref_root: Path):
    pkg_root = ref_root / "cpu" / "pdmrg" / "pdmrg"
    for name in ("pdmrg", "pdmrg.numerics", "pdmrg.environments"):
        mod = types.ModuleType(name)
        mod.__path__ = []
        sys.modules[name] = mod

    def load(modname, rel):
        spec = importlib.util.spec_from_file_location(modname, pkg_root / rel)
        mod = importlib.util.module_from_spec(spec)
        sys.modules[modname] = mod
        spec.loader.exec_module(mod)
        return mod

    eh = load("pdmrg.numerics.effective_ham", "numerics/effective_ham.py")
    es = load("pdmrg.numerics.eigensolver", "numerics/eigensolver.py")
    sv = load("pdmrg.numerics.accurate_svd", "numerics/accurate_svd.py")
    up = load("pdmrg.environments.update", "environments/update.py")
    return eh, es, sv, up


def ref_sweep(eh, es, sv, up, mpo, mps, chi, n_sweeps, maxiter=50, tol=1e-12):
    """The reference's serial sweep (test_numerics.py:230-287) on given inputs."""
    L = len(mpo)
    A = right_canonicalize(mps)
    dtype = np.result_type(A[0].dtype, mpo[0].dtype)
    A = [a.astype(dtype) for a in A]
    R = {L - 1: up.init_right_env(A[-1].shape[2], mpo[-1].shape[1], dtype)}
    for i in range(L - 2, 0, -1):
        R[i] = up.update_right_env(R[i + 1], A[i + 1], mpo[i + 1])
    Lenv = {0: up.init_left_env(A[0].shape[0], mpo[0].shape[0], dtype)}
    energies = []
    for _ in range(n_sweeps):
        for i in range(L - 1):
            theta = np.einsum("ijk,klm->ijlm", A[i], A[i + 1])
            E, th = es.optimize_two_site(Lenv[i], R[i + 1], mpo[i], mpo[i + 1], theta,
                                         max_iter=maxiter, tol=tol)
            cl, d1, d2, cr = th.shape
            U, S, Vh, _ = sv.truncated_svd(th.reshape(cl * d1, d2 * cr), chi)
            A[i] = U.reshape(cl, d1, -1)
            A[i + 1] = (np.diag(S) @ Vh).reshape(-1, d2, cr)
            Lenv[i + 1] = up.update_left_env(Lenv[i], A[i], mpo[i])
        R[L - 1] = up.init_right_env(A[-1].shape[2], mpo[-1].shape[1], dtype)
        for i in range(L - 2, -1, -1):
            theta = np.einsum("ijk,klm->ijlm", A[i], A[i + 1])
            E, th = es.optimize_two_site(Lenv[i], R[i + 1], mpo[i], mpo[i + 1], theta,
                                         max_iter=maxiter, tol=tol)
            cl, d1, d2, cr = th.shape
            U, S, Vh, _ = sv.truncated_svd(th.reshape(cl * d1, d2 * cr), chi)
            A[i + 1] = Vh.reshape(-1, d2, cr)
            A[i] = (U @ np.diag(S)).reshape(cl, d1, -1)
            R[i] = up.update_right_env(R[i + 1], A[i + 1], mpo[i + 1])
        energies.append(float(E))
    return energies


def main(ref_root: Path):
    eh, es, sv, up = load_reference(ref_root)
    rng = np.random.default_rng(20260101)
    fx = {}
    cases = [("r0", 3, 4, 2, 5, np.float64), ("r1", 7, 5, 2, 5, np.float64),
             ("r2", 6, 6, 3, 4, np.float64), ("c0", 4, 3, 2, 5, np.complex128),
             ("c1", 5, 7, 5, 4, np.complex128)]
    for tag, cl, cr, d, D, dt in cases:
        def rnd(*s):
            x = rng.standard_normal(s)
            if np.dtype(dt).kind == "c":
                x = x + 1j * rng.standard_normal(s)
            return x.astype(dt)
        Lenv, Renv = rnd(cl, D, cl), rnd(cr, D, cr)
        WL, WR = rnd(D, D, d, d), rnd(D, D, d, d)
        th = rnd(cl, d, d, cr)
        A = rnd(cl, d, cr)
        B = rnd(cl, d, cr)
        M = rnd(cl * d, d * cr)
        fx.update({f"{tag}_L": Lenv, f"{tag}_R": Renv, f"{tag}_WL": WL, f"{tag}_WR": WR,
                   f"{tag}_theta": th, f"{tag}_A": A, f"{tag}_B": B, f"{tag}_M": M})
        fx[f"{tag}_heff"] = eh.apply_heff(Lenv, Renv, WL, WR, th)
        fx[f"{tag}_lenv"] = up.update_left_env(Lenv, A, WL)
        fx[f"{tag}_renv"] = up.update_right_env(Renv, B, WR)
        U, S, Vh, te = sv.truncated_svd(M, max(1, min(M.shape) - 2))
        fx[f"{tag}_svd_S"] = S
        fx[f"{tag}_svd_te"] = np.array(te)
    np.savez_compressed(HERE / "ref_primitives.npz", **fx)

    # fixture copy
    src = ref_root / "benchmark_data" / "regular" / "heisenberg" / "L12_D20"
    shutil.copyfile(src / "mpo.npz", HERE / "heis_L12_mpo.npz")
    shutil.copyfile(src / "initial_mps.npz", HERE / "heis_L12_mps.npz")
    golden = json.loads((src / "golden_results.json").read_text())

    from oracle.dmrg2_oracle import load_npz_mpo, load_npz_mps
    mpo = load_npz_mpo(HERE / "heis_L12_mpo.npz")
    mps = load_npz_mps(HERE / "heis_L12_mps.npz")
    out = {"heis_L12_fixture": {
        "quimb_dmrg2_energy": golden["quimb_dmrg2"]["energy"],
        "quimb_dmrg1_energy": golden["quimb_dmrg1"]["energy"],
        "ref_sweep_chi20": ref_sweep(eh, es, sv, up, mpo, mps, 20, 4),
    }}
    runs = {
        "heis_L12_seed0_chi32": (models.heisenberg_mpo(12), random_mps(12, 2, 8, 0), 32, 4),
        "xxz_L10_d07_seed1_chi16": (models.heisenberg_mpo(10, 1.0, 0.7), random_mps(10, 2, 4, 1), 16, 4),
        "jos_L6_nmax1_seed2_chi16": (models.josephson_mpo(6), random_mps(6, 3, 4, 2, np.complex128), 16, 4),
        "j1j2_L10_seed3_chi24": (models.j1j2_mpo(10, 1.0, 0.3), random_mps(10, 2, 4, 3), 24, 4),
    }
    for k, (mpo, mps, chi, ns) in runs.items():
        out[k] = {"chi": chi, "sweeps": ns,
                  "ref_sweep": ref_sweep(eh, es, sv, up, mpo, mps, chi, ns)}
    (HERE / "ref_dmrg.json").write_text(json.dumps(out, indent=1))
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path of the reference checkout>")
    main(Path(sys.argv[1]))
