"""CPU oracle for the two-site DMRG hot path (test infrastructure only).

This module is the correctness oracle. Only ``tests/``, ``__graft_entry__.smoke``
and the CPU-baseline leg of ``bench.py`` import it. The GPU engine never calls
it, and nothing in the product path falls back to it.

It restates, in numpy/scipy, the reference's CPU two-site DMRG primitives and
its serial sweep loop:

* ``apply_heff``       <- ``cpu/pdmrg/pdmrg/numerics/effective_ham.py:21-81``
* ``optimize_two_site``<- ``cpu/pdmrg/pdmrg/numerics/eigensolver.py:13-63``
  (ARPACK ``eigsh(which='SA')`` on a matrix-free operator)
* ``truncated_svd``    <- ``cpu/pdmrg/pdmrg/numerics/accurate_svd.py:82-110``,
  extended with the absolute singular-value cutoff of the reference GPU driver
  (``gpu-rocm/common/scalar_traits.h:497-505``)
* ``update_left_env`` / ``update_right_env``
                       <- ``cpu/pdmrg/pdmrg/environments/update.py:16-127``
* ``dmrg2``            <- the serial sweep of
  ``cpu/pdmrg/pdmrg/tests/test_numerics.py:230-287``, extended with a bond
  dimension schedule, cutoff, per-sweep energy, truncation error and the
  ``|dE| < tol`` stop rule of ``gpu-rocm/dmrg2-gpu/src/dmrg2_gpu_impl.h:1440-1447``.

Parity of these restatements is pinned against the reference modules
themselves (``tests/golden/make_golden.py`` imports them in a container that
has the reference checked out and commits the outputs as fixtures) and against
the reference's known-answer energies.

Tensor conventions:
  MPS  A[i]: (chi_left, d, chi_right)
  MPO  W[i]: (D_left, D_right, s_in, s_out)          (see oracle/models.py)
  Env  L/R : (bra, mpo, ket)
"""

from __future__ import annotations

import time

import numpy as np
from scipy.sparse.linalg import LinearOperator, eigsh


# ----------------------------------------------------------------------------
# primitives
# ----------------------------------------------------------------------------

def apply_heff(Lenv, Renv, WL, WR, theta):
    """theta'[a,p,q,f] = L[a,w,c] theta[c,s,r,e] WL[w,m,s,p] WR[m,n,r,q] R[f,n,e].

    Same contraction order as effective_ham.py:60-79 (four tensordots).
    """
    X = np.tensordot(Lenv, theta, axes=(2, 0))            # a w s r e
    Y = np.tensordot(X, WL, axes=([1, 2], [0, 2]))         # a r e m p
    Z = np.tensordot(Y, WR, axes=([1, 3], [2, 0]))         # a e p n q
    return np.tensordot(Z, Renv, axes=([1, 3], [2, 1]))    # a p q f


def update_left_env(Lenv, A, W):
    """L'[a',w',c'] = L[a,w,c] conj(A)[a,t,a'] W[w,w',s,t] A[c,s,c'] (update.py:16-80)."""
    X = np.tensordot(Lenv, A, axes=(2, 0))                 # a w s c'
    Y = np.tensordot(X, W, axes=([1, 2], [0, 2]))          # a c' w' t
    Z = np.tensordot(Y, A.conj(), axes=([0, 3], [0, 1]))   # c' w' a'
    return np.transpose(Z, (2, 1, 0))


def update_right_env(Renv, B, W):
    """R'[a',w',c'] = R[a,w,c] conj(B)[a',t,a] W[w',w,s,t] B[c',s,c] (update.py:83-127)."""
    X = np.tensordot(Renv, B, axes=(2, 2))                 # a w c' s
    Y = np.tensordot(X, W, axes=([1, 3], [1, 2]))          # a c' w' t
    Z = np.tensordot(Y, B.conj(), axes=([0, 3], [2, 1]))   # c' w' a'
    return np.transpose(Z, (2, 1, 0))


def optimize_two_site(Lenv, Renv, WL, WR, theta0, maxiter=50, tol=1e-12,
                      dense_below=32):
    """Lowest eigenpair of H_eff by ARPACK Lanczos (eigensolver.py:13-63).

    For operator dimensions below ``dense_below`` (where ARPACK cannot run with
    k=1) the operator is formed densely and diagonalised exactly.
    """
    shape = theta0.shape
    n = int(np.prod(shape))
    dtype = np.result_type(theta0.dtype, Lenv.dtype, Renv.dtype, WL.dtype, WR.dtype)

    def mv(v):
        return apply_heff(Lenv, Renv, WL, WR, v.reshape(shape)).ravel()

    if n < dense_below:
        H = np.empty((n, n), dtype)
        e = np.zeros(n, dtype)
        for j in range(n):
            e[:] = 0
            e[j] = 1
            H[:, j] = mv(e)
        H = 0.5 * (H + H.conj().T)
        w, V = np.linalg.eigh(H)
        return float(w[0]), V[:, 0].reshape(shape)
    op = LinearOperator((n, n), matvec=mv, dtype=dtype)
    v0 = theta0.ravel().astype(dtype)
    try:
        w, V = eigsh(op, k=1, v0=v0, which="SA", maxiter=maxiter, tol=tol)
    except Exception:
        w, V = eigsh(op, k=1, v0=v0, which="SA", maxiter=maxiter * 10, tol=tol * 10)
    return float(w[0].real), V[:, 0].reshape(shape)


def truncated_svd(M, max_bond, cutoff=0.0):
    """SVD truncated to ``max_bond`` and to singular values >= ``cutoff``.

    accurate_svd.py:82-110 keeps min(len(S), max_bond) (>= 1) and reports
    trunc_err = sum of discarded S^2. The reference GPU driver additionally
    stops at the first S[i] < cutoff (scalar_traits.h:497-505); cutoff=0 gives
    the numpy reference exactly.
    """
    U, S, Vh = np.linalg.svd(M, full_matrices=False)
    k = min(len(S), max_bond)
    if cutoff > 0.0:
        below = np.nonzero(S[:k] < cutoff)[0]
        if below.size:
            k = int(below[0])
    k = max(k, 1)
    trunc_err = float(np.sum(S[k:] ** 2))
    return U[:, :k], S[:k], Vh[:k, :], trunc_err


# ----------------------------------------------------------------------------
# MPS helpers
# ----------------------------------------------------------------------------

def random_mps(L, d, chi, seed=0, dtype=np.float64):
    """Seeded i.i.d. N(0,1) MPS with bond dims min(d^min(i,L-i), chi).

    For complex dtypes real and imaginary parts are independent N(0,1).
    """
    rng = np.random.default_rng(seed)
    dims = [1] + [min(d ** min(i, L - i), chi) for i in range(1, L)] + [1]
    mps = []
    for i in range(L):
        shape = (dims[i], d, dims[i + 1])
        if np.dtype(dtype).kind == "c":
            A = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
        else:
            A = rng.standard_normal(shape)
        mps.append(A.astype(dtype))
    return mps


def right_canonicalize(mps):
    """Bring sites 1..L-1 into right-canonical form; normalise the state.

    Equivalent to quimb's ``mps.canonize(0)`` used at test_numerics.py:241-242.
    """
    mps = [A.copy() for A in mps]
    for i in range(len(mps) - 1, 0, -1):
        cl, d, cr = mps[i].shape
        M = mps[i].reshape(cl, d * cr)
        U, S, Vh = np.linalg.svd(M, full_matrices=False)
        k = len(S)
        mps[i] = Vh.reshape(k, d, cr)
        mps[i - 1] = np.tensordot(mps[i - 1], U * S, axes=(2, 0))
    mps[0] = mps[0] / np.linalg.norm(mps[0])
    return mps


def mps_norm2(mps):
    E = np.ones((1, 1), dtype=mps[0].dtype)
    for A in mps:
        E = np.einsum("ab,asc,bsd->cd", E, A.conj(), A, optimize=True)
    return float(E[0, 0].real)


def expect_local(mps, op):
    """<psi| O_i |psi> / <psi|psi> for every site, op[s_out, s_in]."""
    L = len(mps)
    out = np.zeros(L, dtype=np.result_type(mps[0].dtype, np.asarray(op).dtype))
    left = [np.ones((1, 1), dtype=mps[0].dtype)]
    for A in mps:
        left.append(np.einsum("ab,asc,bsd->cd", left[-1], A.conj(), A, optimize=True))
    right = [None] * (L + 1)
    right[L] = np.ones((1, 1), dtype=mps[0].dtype)
    for i in range(L - 1, -1, -1):
        A = mps[i]
        right[i] = np.einsum("cd,asc,bsd->ab", right[i + 1], A.conj(), A, optimize=True)
    nrm = left[L][0, 0]
    for i, A in enumerate(mps):
        out[i] = np.einsum("ab,atc,ts,bsd,cd->", left[i], A.conj(), op, A, right[i + 1], optimize=True) / nrm
    return out


def mpo_expectation(mps, mpo):
    E = np.ones((1, 1, 1), dtype=np.result_type(mps[0].dtype, mpo[0].dtype))
    for A, W in zip(mps, mpo):
        E = update_left_env(E, A, W)
    return E[0, 0, 0] / mps_norm2(mps)


# ----------------------------------------------------------------------------
# the sweep
# ----------------------------------------------------------------------------

def dmrg2(mpo, mps, schedule, cutoff=0.0, tol=1e-10, lanczos_tol=1e-12,
          lanczos_maxiter=50, min_sweeps=2, verbose=False):
    """Serial two-site DMRG (test_numerics.py:230-287 extended).

    ``schedule`` is a list of chi_max per sweep (its length is the sweep budget).
    A sweep is a left-to-right half sweep followed by a right-to-left half
    sweep; the sweep energy is the eigenvalue of the last bond optimised
    (bond (0,1) of the right-to-left half), as in dmrg2_gpu_impl.h:1396-1413.
    The run stops once |E_sweep - E_prev| < tol after at least ``min_sweeps``.

    Returns a dict with per-sweep energies, truncation errors (max and sum of
    discarded weight over the sweep), max bond dims, wall times, the final MPS
    and the number of sweeps run.
    """
    L = len(mpo)
    A = right_canonicalize(mps)
    dtype = np.result_type(A[0].dtype, mpo[0].dtype)
    A = [a.astype(dtype) for a in A]
    # Renv[i] = contraction of sites i..L-1 ; Lenv[i] = contraction of sites 0..i-1
    Renv = [None] * (L + 1)
    Lenv = [None] * (L + 1)
    Renv[L] = np.ones((1, 1, 1), dtype)
    Lenv[0] = np.ones((1, 1, 1), dtype)
    for i in range(L - 1, 1, -1):
        Renv[i] = update_right_env(Renv[i + 1], A[i], mpo[i])

    out = dict(energies=[], trunc_err_max=[], trunc_err_sum=[], max_bond=[],
               wall=[], sweeps=0)
    E_prev = None
    E = 0.0
    for sweep, chi in enumerate(schedule):
        t0 = time.perf_counter()
        tmax, tsum = 0.0, 0.0
        for i in range(L - 1):
            theta = np.tensordot(A[i], A[i + 1], axes=(2, 0))
            E, th = optimize_two_site(Lenv[i], Renv[i + 2], mpo[i], mpo[i + 1], theta,
                                      maxiter=lanczos_maxiter, tol=lanczos_tol)
            cl, d1, d2, cr = th.shape
            U, S, Vh, te = truncated_svd(th.reshape(cl * d1, d2 * cr), chi, cutoff)
            tmax, tsum = max(tmax, te), tsum + te
            k = len(S)
            A[i] = U.reshape(cl, d1, k)
            A[i + 1] = (S[:, None] * Vh).reshape(k, d2, cr)
            Lenv[i + 1] = update_left_env(Lenv[i], A[i], mpo[i])
        for i in range(L - 2, -1, -1):
            theta = np.tensordot(A[i], A[i + 1], axes=(2, 0))
            E, th = optimize_two_site(Lenv[i], Renv[i + 2], mpo[i], mpo[i + 1], theta,
                                      maxiter=lanczos_maxiter, tol=lanczos_tol)
            cl, d1, d2, cr = th.shape
            U, S, Vh, te = truncated_svd(th.reshape(cl * d1, d2 * cr), chi, cutoff)
            tmax, tsum = max(tmax, te), tsum + te
            k = len(S)
            A[i + 1] = Vh.reshape(k, d2, cr)
            A[i] = (U * S).reshape(cl, d1, k)
            Renv[i + 1] = update_right_env(Renv[i + 2], A[i + 1], mpo[i + 1])
        out["energies"].append(E)
        out["trunc_err_max"].append(tmax)
        out["trunc_err_sum"].append(tsum)
        out["max_bond"].append(max(a.shape[2] for a in A))
        out["wall"].append(time.perf_counter() - t0)
        out["sweeps"] = sweep + 1
        if verbose:
            print(f"sweep {sweep}: E={E:.14f} chi={chi} trunc={tmax:.3e}")
        if E_prev is not None and sweep + 1 >= min_sweeps and abs(E - E_prev) < tol:
            break
        E_prev = E
    out["energy"] = E
    out["mps"] = A
    return out


# ----------------------------------------------------------------------------
# single-site sweep (the reference's dmrg-gpu driver)
# ----------------------------------------------------------------------------

def apply_heff1(Lenv, Renv, W, A):
    """A'[a,t,f] = L[a,w,c] A[c,s,e] W[w,v,s,t] R[f,v,e]: the one-site H_eff of
    gpu-rocm/dmrg-gpu/src/dmrg_gpu_impl.h (apply_heff), restated with tensordots."""
    X = np.tensordot(Lenv, A, axes=(2, 0))                 # a w s e
    Y = np.tensordot(X, W, axes=([1, 2], [0, 2]))          # a e v t
    return np.tensordot(Y, Renv, axes=([1, 2], [2, 1]))    # a t f


def optimize_one_site(Lenv, Renv, W, A0, maxiter=50, tol=1e-12, dense_below=32):
    """Lowest eigenpair of the one-site H_eff (ARPACK, or dense below ``dense_below``)."""
    shape = A0.shape
    n = int(np.prod(shape))
    dtype = np.result_type(A0.dtype, Lenv.dtype, Renv.dtype, W.dtype)

    def mv(v):
        return apply_heff1(Lenv, Renv, W, v.reshape(shape)).ravel()

    if n < dense_below:
        H = np.empty((n, n), dtype)
        e = np.zeros(n, dtype)
        for j in range(n):
            e[:] = 0
            e[j] = 1
            H[:, j] = mv(e)
        H = 0.5 * (H + H.conj().T)
        w, V = np.linalg.eigh(H)
        return float(w[0]), V[:, 0].reshape(shape)
    op = LinearOperator((n, n), matvec=mv, dtype=dtype)
    w, V = eigsh(op, k=1, v0=A0.ravel().astype(dtype), which="SA", maxiter=maxiter * 10, tol=tol)
    return float(w[0].real), V[:, 0].reshape(shape)


def dmrg1(mpo, mps, schedule, cutoff=0.0, tol=1e-10, lanczos_tol=1e-12, lanczos_maxiter=50,
          min_sweeps=2):
    """Serial single-site DMRG, restating DMRGGPU::run / sweep_left_to_right /
    sweep_right_to_left / optimize_site / svd_and_update_mps
    (gpu-rocm/dmrg-gpu/src/dmrg_gpu_impl.h:1119-1470).

    Left to right, sites 0..L-2 are optimised and split (A[i] = U, S Vh absorbed
    into A[i+1]); site L-1 is optimised without a split. Right to left, sites
    L-1..1 are optimised and split (A[i] = Vh, U S absorbed into A[i-1]); site 0
    is optimised without a split and its eigenvalue is the sweep energy. The
    truncation is the oracle's truncated_svd (max bond, absolute cutoff), so
    bond dimensions never grow past those of the initial MPS.
    """
    L = len(mpo)
    A = right_canonicalize(mps)
    dtype = np.result_type(A[0].dtype, mpo[0].dtype)
    A = [a.astype(dtype) for a in A]
    Renv = [None] * (L + 1)
    Lenv = [None] * (L + 1)
    Renv[L] = np.ones((1, 1, 1), dtype)
    Lenv[0] = np.ones((1, 1, 1), dtype)
    for i in range(L - 1, 0, -1):
        Renv[i] = update_right_env(Renv[i + 1], A[i], mpo[i])
    out = dict(energies=[], trunc_err_max=[], max_bond=[], sweeps=0)
    E_prev, E = None, 0.0
    for sweep, chi in enumerate(schedule):
        tmax = 0.0
        for i in range(L - 1):
            E, th = optimize_one_site(Lenv[i], Renv[i + 1], mpo[i], A[i], lanczos_maxiter, lanczos_tol)
            cl, d, cr = th.shape
            U, S, Vh, te = truncated_svd(th.reshape(cl * d, cr), chi, cutoff)
            tmax = max(tmax, te)
            A[i] = U.reshape(cl, d, len(S))
            A[i + 1] = np.tensordot(S[:, None] * Vh, A[i + 1], axes=(1, 0))
            Lenv[i + 1] = update_left_env(Lenv[i], A[i], mpo[i])
        E, A[L - 1] = optimize_one_site(Lenv[L - 1], Renv[L], mpo[L - 1], A[L - 1], lanczos_maxiter, lanczos_tol)
        for i in range(L - 1, 0, -1):
            E, th = optimize_one_site(Lenv[i], Renv[i + 1], mpo[i], A[i], lanczos_maxiter, lanczos_tol)
            cl, d, cr = th.shape
            U, S, Vh, te = truncated_svd(th.reshape(cl, d * cr), chi, cutoff)
            tmax = max(tmax, te)
            A[i] = Vh.reshape(len(S), d, cr)
            A[i - 1] = np.tensordot(A[i - 1], U * S, axes=(2, 0))
            Renv[i] = update_right_env(Renv[i + 1], A[i], mpo[i])
        E, A[0] = optimize_one_site(Lenv[0], Renv[1], mpo[0], A[0], lanczos_maxiter, lanczos_tol)
        out["energies"].append(E)
        out["trunc_err_max"].append(tmax)
        out["max_bond"].append(max(a.shape[2] for a in A))
        out["sweeps"] = sweep + 1
        if E_prev is not None and sweep + 1 >= min_sweeps and abs(E - E_prev) < tol:
            break
        E_prev = E
    out["energy"] = E
    out["mps"] = A
    return out


def ramp_schedule(chis, n_sweeps):
    """Spread the chi values of ``chis`` evenly over ``n_sweeps`` sweeps."""
    per = max(1, n_sweeps // len(chis))
    sched = []
    for c in chis:
        sched += [c] * per
    while len(sched) < n_sweeps:
        sched.append(chis[-1])
    return sched[:n_sweeps]


# ----------------------------------------------------------------------------
# fixture I/O (benchmark_data npz format, benchmarks/lib/data_loader.py:114-152)
# ----------------------------------------------------------------------------

def load_npz_mpo(path):
    z = np.load(path, allow_pickle=False)
    keys = sorted((k for k in z.files if k.startswith("tensor_")),
                  key=lambda k: int(k.split("_")[1]))
    Ws = [np.asarray(z[k]) for k in keys]
    L = len(Ws)
    out = []
    for i, W in enumerate(Ws):
        if W.ndim == 3 and i == 0:
            W = W[None]                 # (1, Dr, d, d)
        elif W.ndim == 3 and i == L - 1:
            W = W[:, None]              # (Dl, 1, d, d)
        out.append(np.ascontiguousarray(W))
    return out


def load_npz_mps(path):
    z = np.load(path, allow_pickle=False)
    keys = sorted((k for k in z.files if k.startswith("tensor_")),
                  key=lambda k: int(k.split("_")[1]))
    As = [np.asarray(z[k]) for k in keys]
    L = len(As)
    out = []
    for i, A in enumerate(As):
        # regular-tier layout: (d, chi) on the left end, (chi, d) on the right
        if A.ndim == 2 and i == 0:
            A = A[None]
        elif A.ndim == 2 and i == L - 1:
            A = A[:, :, None]
        out.append(np.ascontiguousarray(A))
    return out
