"""Oracle MPO builders and exact diagonalisation (test infrastructure only).

This module is part of the CPU oracle. Only the test-suite, the smoke check
and the CPU-baseline leg of bench.py import it; the GPU engine never does.

Conventions (shared by the whole oracle and by the GPU engine):

* MPO site tensor ``W[i]`` has shape ``(Dl, Dr, d, d)`` with axes
  ``(mpo_left, mpo_right, s_in, s_out)``. The physical operator that the site
  applies is ``O[s_out, s_in] = W[..., s_in, s_out]``. This is the convention of
  the reference's numpy primitives (``cpu/pdmrg/pdmrg/numerics/effective_ham.py:53-59``:
  the ket index of theta is contracted with MPO axis 2).
* Boundary sites carry explicit unit MPO bonds: ``Dl = 1`` on site 0 and
  ``Dr = 1`` on site ``L-1``.

Models restated from the reference's MPO builders:

* Heisenberg XXZ, D=5 automaton (``gpu-rocm/dmrg2-gpu/src/test_dmrg2_gpu.cpp:20-63``),
  here with a free anisotropy ``delta``.
* Transverse-field Ising, D=3 (``test_dmrg2_gpu.cpp:65-113``).
* Josephson-junction array in the charge basis, D=4
  (``test_dmrg2_gpu.cpp:115-191``), with either the reference's on-site form
  ``E_C n^2 - n_g n`` or the shifted form ``E_C (n - n_g)^2``.
* J1-J2 and J1-J2-J3 chains (``gpu-rocm/common/challenge_mpos.h:50-200``) built
  here with a compact delay-line automaton (D = 2 + 3*range).
* Two-leg Heisenberg ladder with d=4 rung supersites
  (``gpu-rocm/common/challenge_mpos.h:200-360``), D = 8.

Exact diagonalisation builds the Hamiltonian from its local terms with sparse
Kronecker products, independently of the MPO, as the reference's
``gpu-rocm/common/verify_challenge_mpos.py:108-180`` does.
"""

from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

# ----------------------------------------------------------------------------
# local operators (basis index 0 = spin up / lowest charge)
# ----------------------------------------------------------------------------
SZ = np.array([[0.5, 0.0], [0.0, -0.5]])
SP = np.array([[0.0, 1.0], [0.0, 0.0]])  # |up><down|
SM = SP.T.copy()
SX = np.array([[0.0, 1.0], [1.0, 0.0]])  # Pauli matrices for TFIM
PZ = np.array([[1.0, 0.0], [0.0, -1.0]])
I2 = np.eye(2)


def _put(W, wl, wr, op):
    """Place operator ``op`` (rows = s_out, cols = s_in) on MPO entry (wl, wr)."""
    W[wl, wr, :, :] = np.asarray(op).T


def _finish(bulk, L, left_row, right_col):
    """Turn a bulk tensor template into L site tensors with unit boundaries."""
    Ws = []
    for i in range(L):
        W = bulk(i)
        if i == 0:
            W = W[left_row:left_row + 1]
        if i == L - 1:
            W = W[:, right_col:right_col + 1]
        Ws.append(np.ascontiguousarray(W))
    return Ws


def heisenberg_mpo(L, J=1.0, delta=1.0, hz=0.0):
    """XXZ chain H = J sum (Sx Sx + Sy Sy + delta Sz Sz) - hz sum Sz, D = 5."""
    D, d = 5, 2
    dt = np.float64

    def bulk(i):
        W = np.zeros((D, D, d, d), dt)
        _put(W, 0, 0, I2)
        _put(W, 0, 1, SP)
        _put(W, 0, 2, SM)
        _put(W, 0, 3, SZ)
        _put(W, 0, 4, -hz * SZ)
        _put(W, 1, 4, 0.5 * J * SM)
        _put(W, 2, 4, 0.5 * J * SP)
        _put(W, 3, 4, J * delta * SZ)
        _put(W, 4, 4, I2)
        return W

    return _finish(bulk, L, 0, D - 1)


def tfim_mpo(L, J=1.0, h=1.0):
    """Transverse-field Ising H = -J sum Z Z - h sum X (Pauli matrices), D = 3."""
    D, d = 3, 2

    def bulk(i):
        W = np.zeros((D, D, d, d))
        _put(W, 0, 0, I2)
        _put(W, 0, 1, -J * PZ)
        _put(W, 0, 2, -h * SX)
        _put(W, 1, 2, PZ)
        _put(W, 2, 2, I2)
        return W

    return _finish(bulk, L, 0, D - 1)


def josephson_ops(n_max):
    d = 2 * n_max + 1
    n = np.diag(np.arange(d, dtype=np.float64) - n_max)
    raise_op = np.zeros((d, d), np.complex128)
    for k in range(d - 1):
        raise_op[k + 1, k] = 1.0
    lower_op = raise_op.conj().T.copy()
    return d, n, raise_op, lower_op


def josephson_mpo(L, n_max=1, E_J=1.0, E_C=0.5, n_g=0.0, phi=np.pi / 4,
                  onsite="reference"):
    """Josephson-junction array in the charge basis, complex128, D = 4.

    H = sum_i U(n_i) + sum_i [alpha R_i L_{i+1} + conj(alpha) L_i R_{i+1}],
    alpha = -(E_J/2) e^{i phi}, R/L = charge raising/lowering.
    ``onsite='reference'``: U(n) = E_C n^2 - n_g n (test_dmrg2_gpu.cpp:135).
    ``onsite='shifted'``:   U(n) = E_C (n - n_g)^2.
    """
    d, n, R, Lo = josephson_ops(n_max)
    if onsite == "reference":
        U = E_C * n @ n - n_g * n
    elif onsite == "shifted":
        m = n - n_g * np.eye(d)
        U = E_C * m @ m
    else:
        raise ValueError(onsite)
    alpha = -0.5 * E_J * np.exp(1j * phi)
    D = 4
    Id = np.eye(d)

    def bulk(i):
        W = np.zeros((D, D, d, d), np.complex128)
        _put(W, 0, 0, Id)
        _put(W, 0, 1, alpha * R)
        _put(W, 0, 2, np.conj(alpha) * Lo)
        _put(W, 0, 3, U)
        _put(W, 1, 3, Lo)
        _put(W, 2, 3, R)
        _put(W, 3, 3, Id)
        return W

    return _finish(bulk, L, 0, D - 1)


def longrange_heisenberg_mpo(L, Js):
    """H = sum_r Js[r-1] sum_i S_i . S_{i+r}, delay-line automaton.

    States: 0 = start, (t, k) = operator t in {S+, S-, Sz} placed k sites ago
    (k = 1..R), last = done. D = 2 + 3 R with R = len(Js).
    """
    R = len(Js)
    D, d = 2 + 3 * R, 2
    done = D - 1
    ops = [SP, SM, SZ]
    close = [SM, SP, SZ]
    wt = [0.5, 0.5, 1.0]

    def st(t, k):
        return 1 + t * R + (k - 1)

    def bulk(i):
        W = np.zeros((D, D, d, d))
        _put(W, 0, 0, I2)
        _put(W, done, done, I2)
        for t in range(3):
            _put(W, 0, st(t, 1), ops[t])
            for k in range(1, R + 1):
                if Js[k - 1] != 0.0:
                    _put(W, st(t, k), done, wt[t] * Js[k - 1] * close[t])
                if k < R:
                    _put(W, st(t, k), st(t, k + 1), I2)
        return W

    return _finish(bulk, L, 0, D - 1)


def j1j2_mpo(L, J1=1.0, J2=0.5):
    """J1-J2 chain, D = 8."""
    return longrange_heisenberg_mpo(L, [J1, J2])


def j1j2j3_mpo(L, J1=1.0, J2=0.4, J3=0.2):
    """J1-J2-J3 chain, D = 11."""
    return longrange_heisenberg_mpo(L, [J1, J2, J3])


def ladder_ops():
    """Spin operators of the two legs on a d=4 rung (index = 2*s_leg1 + s_leg2)."""
    leg1 = [np.kron(o, I2) for o in (SP, SM, SZ)]
    leg2 = [np.kron(I2, o) for o in (SP, SM, SZ)]
    return leg1, leg2


def ladder_mpo(L_rungs, J_leg=1.0, J_rung=1.0):
    """Two-leg Heisenberg ladder on d=4 rung supersites, D = 8."""
    D, d = 8, 4
    leg1, leg2 = ladder_ops()
    I4 = np.eye(4)
    rung = J_rung * (0.5 * (leg1[0] @ leg2[1] + leg1[1] @ leg2[0]) + leg1[2] @ leg2[2])
    close = [1, 0, 2]
    wt = [0.5, 0.5, 1.0]

    def bulk(i):
        W = np.zeros((D, D, d, d))
        _put(W, 0, 0, I4)
        _put(W, 0, 7, rung)
        _put(W, 7, 7, I4)
        for t in range(3):
            _put(W, 0, 1 + t, leg1[t])
            _put(W, 0, 4 + t, leg2[t])
            _put(W, 1 + t, 7, wt[t] * J_leg * leg1[close[t]])
            _put(W, 4 + t, 7, wt[t] * J_leg * leg2[close[t]])
        return W

    return _finish(bulk, L_rungs, 0, D - 1)


# ----------------------------------------------------------------------------
# exact diagonalisation from local terms
# ----------------------------------------------------------------------------

def _site_op(op, i, L, d):
    mats = [sp.identity(d, format="csr", dtype=np.complex128)] * L
    mats = list(mats)
    mats[i] = sp.csr_matrix(np.asarray(op, dtype=np.complex128))
    out = mats[0]
    for m in mats[1:]:
        out = sp.kron(out, m, format="csr")
    return out


def _bond(opa, i, opb, j, L, d):
    return _site_op(opa, i, L, d) @ _site_op(opb, j, L, d)


def ham_heisenberg(L, J=1.0, delta=1.0, hz=0.0):
    H = 0
    for i in range(L - 1):
        H = H + J * (0.5 * (_bond(SP, i, SM, i + 1, L, 2) + _bond(SM, i, SP, i + 1, L, 2))
                     + delta * _bond(SZ, i, SZ, i + 1, L, 2))
    for i in range(L):
        if hz:
            H = H - hz * _site_op(SZ, i, L, 2)
    return H


def ham_tfim(L, J=1.0, h=1.0):
    H = 0
    for i in range(L - 1):
        H = H - J * _bond(PZ, i, PZ, i + 1, L, 2)
    for i in range(L):
        H = H - h * _site_op(SX, i, L, 2)
    return H


def ham_josephson(L, n_max=1, E_J=1.0, E_C=0.5, n_g=0.0, phi=np.pi / 4,
                  onsite="reference"):
    d, n, R, Lo = josephson_ops(n_max)
    if onsite == "reference":
        U = E_C * n @ n - n_g * n
    else:
        m = n - n_g * np.eye(d)
        U = E_C * m @ m
    alpha = -0.5 * E_J * np.exp(1j * phi)
    H = 0
    for i in range(L):
        H = H + _site_op(U, i, L, d)
    for i in range(L - 1):
        H = H + alpha * _bond(R, i, Lo, i + 1, L, d) + np.conj(alpha) * _bond(Lo, i, R, i + 1, L, d)
    return H


def ham_longrange(L, Js):
    H = 0
    for r, J in enumerate(Js, start=1):
        for i in range(L - r):
            H = H + J * (0.5 * (_bond(SP, i, SM, i + r, L, 2) + _bond(SM, i, SP, i + r, L, 2))
                         + _bond(SZ, i, SZ, i + r, L, 2))
    return H


def ham_ladder(L_rungs, J_leg=1.0, J_rung=1.0):
    leg1, leg2 = ladder_ops()
    d = 4
    H = 0
    rung = J_rung * (0.5 * (leg1[0] @ leg2[1] + leg1[1] @ leg2[0]) + leg1[2] @ leg2[2])
    for i in range(L_rungs):
        H = H + _site_op(rung, i, L_rungs, d)
    for i in range(L_rungs - 1):
        for leg in (leg1, leg2):
            H = H + J_leg * (0.5 * (_bond(leg[0], i, leg[1], i + 1, L_rungs, d)
                                    + _bond(leg[1], i, leg[0], i + 1, L_rungs, d))
                             + _bond(leg[2], i, leg[2], i + 1, L_rungs, d))
    return H


def ground_energy(H, dense_below=600):
    """Lowest eigenvalue of a sparse Hermitian matrix (FP64)."""
    n = H.shape[0]
    if n <= dense_below:
        return float(np.linalg.eigvalsh(H.toarray())[0])
    w = spla.eigsh(H, k=1, which="SA", tol=1e-14, maxiter=100000,
                   return_eigenvectors=False)
    return float(w[0])


def ground_state(H, dense_below=600):
    n = H.shape[0]
    if n <= dense_below:
        w, v = np.linalg.eigh(H.toarray())
        return float(w[0]), v[:, 0]
    w, v = spla.eigsh(H, k=1, which="SA", tol=1e-14, maxiter=100000)
    return float(w[0]), v[:, 0]


def mpo_to_dense(Ws):
    """Contract an MPO to a dense matrix H[out, in] (small L only)."""
    T = Ws[0][0]  # (Dr, d_in, d_out)
    T = np.transpose(T, (0, 2, 1))  # (Dr, out, in)
    T = T[:, :, :]  # (D, O, I)
    for W in Ws[1:]:
        Wt = np.transpose(W, (0, 1, 3, 2))  # (Dl, Dr, out, in)
        T = np.einsum("aOI,abot->bOoIt", T, Wt)
        D = T.shape[0]
        o = T.shape[1] * T.shape[2]
        T = T.reshape(D, o, o)
    return T[0]
