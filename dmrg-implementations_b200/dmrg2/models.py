"""MPO builders and seeded initial states for the engine's own workloads.

MPO tensors follow the engine's row-major convention (Dl, Dr, s_in, s_out):
site i applies O[s_out, s_in] = W[a, b, s_in, s_out] on the automaton
transition a -> b, with a unit left bond on site 0 and a unit right bond on
site L-1. Each model is written as a finite-state automaton: state 0 has placed
nothing yet, the last state has completed every term, and the transitions are
listed as (from, to, operator).

Models (the reference's builders: gpu-rocm/dmrg2-gpu/src/test_dmrg2_gpu.cpp:20-191,
gpu-rocm/common/challenge_mpos.h:50-200):
  xxz        J sum (Sx Sx + Sy Sy + delta Sz Sz) - hz sum Sz,        D = 5
  heisenberg_range   sum_r J_r sum_i S_i . S_{i+r} (J1-J2: D = 8),   D = 2 + 3 R
  josephson  charge-basis junction array, complex,                    D = 4
"""
from __future__ import annotations

import numpy as np

_SZ = np.diag([0.5, -0.5])
_SP = np.array([[0.0, 1.0], [0.0, 0.0]])  # raises spin down -> up (index 1 -> 0)
_SM = _SP.T


def _automaton_mpo(L, D, d, transitions, dtype=np.float64):
    """Site tensors from (from, to, op[s_out, s_in]) transitions of a D-state automaton."""
    bulk = np.zeros((D, D, d, d), dtype)
    for a, b, op in transitions:
        bulk[a, b] += np.asarray(op, dtype).T  # (s_in, s_out) = op^T
    sites = []
    for i in range(L):
        W = bulk
        if i == 0:
            W = W[:1]
        if i == L - 1:
            W = W[:, D - 1:]
        sites.append(np.ascontiguousarray(W))
    return sites


def xxz(L, J=1.0, delta=1.0, hz=0.0):
    """S=1/2 XXZ chain with open ends, D = 5."""
    one = np.eye(2)
    t = [(0, 0, one), (4, 4, one),
         (0, 1, _SP), (1, 4, 0.5 * J * _SM),
         (0, 2, _SM), (2, 4, 0.5 * J * _SP),
         (0, 3, _SZ), (3, 4, J * delta * _SZ),
         (0, 4, -hz * _SZ)]
    return _automaton_mpo(L, 5, 2, t)


def heisenberg_range(L, couplings):
    """Heisenberg couplings at distances 1..R (J1-J2 for two couplings), D = 2 + 3R.

    State (t, k), k = 1..R, carries operator t in (S+, S-, Sz) placed k sites back.
    """
    R = len(couplings)
    D = 2 + 3 * R
    last = D - 1
    one = np.eye(2)
    first = (_SP, _SM, _SZ)
    second = (0.5 * _SM, 0.5 * _SP, _SZ)  # S.S = (S+S- + S-S+)/2 + SzSz
    state = lambda t, k: 1 + 3 * (k - 1) + t
    tr = [(0, 0, one), (last, last, one)]
    for t in range(3):
        tr.append((0, state(t, 1), first[t]))
        for k in range(1, R + 1):
            tr.append((state(t, k), last, couplings[k - 1] * second[t]))
            if k < R:
                tr.append((state(t, k), state(t, k + 1), one))
    return _automaton_mpo(L, D, 2, tr)


def j1j2(L, J1=1.0, J2=0.5):
    return heisenberg_range(L, [J1, J2])


def josephson(L, n_max=1, E_J=1.0, E_C=0.5, n_g=0.0, phi=np.pi / 4, onsite="reference"):
    """Junction array in the charge basis n = -n_max..n_max, complex, D = 4.

    onsite 'reference': E_C n^2 - n_g n; 'shifted': E_C (n - n_g)^2. Hopping
    alpha R_i L_{i+1} + conj(alpha) L_i R_{i+1}, alpha = -(E_J/2) e^{i phi}.
    """
    d = 2 * n_max + 1
    charges = np.arange(d) - n_max
    if onsite == "reference":
        U = np.diag(E_C * charges ** 2 - n_g * charges).astype(np.complex128)
    elif onsite == "shifted":
        U = np.diag(E_C * (charges - n_g) ** 2).astype(np.complex128)
    else:
        raise ValueError(f"unknown onsite form {onsite!r}")
    raise_ = np.eye(d, k=-1).astype(np.complex128)  # |n+1><n| (index k -> k+1)
    lower = raise_.T.copy()
    alpha = -0.5 * E_J * np.exp(1j * phi)
    one = np.eye(d)
    t = [(0, 0, one), (3, 3, one), (0, 3, U),
         (0, 1, alpha * raise_), (1, 3, lower),
         (0, 2, np.conj(alpha) * lower), (2, 3, raise_)]
    return _automaton_mpo(L, 4, d, t, np.complex128)


def random_mps(L, d, chi, seed=0, dtype=np.float64):
    """Seeded i.i.d. N(0,1) MPS with bond dimensions min(d^min(i, L-i), chi).

    Sites are drawn left to right from numpy's default_rng(seed); complex sites
    draw the real part, then the imaginary part.
    """
    rng = np.random.default_rng(seed)
    bonds = [min(d ** min(i, L - i), chi) for i in range(L + 1)]
    cplx = np.dtype(dtype).kind == "c"
    out = []
    for i in range(L):
        shape = (bonds[i], d, bonds[i + 1])
        x = rng.standard_normal(shape)
        if cplx:
            x = x + 1j * rng.standard_normal(shape)
        out.append(x.astype(dtype))
    return out
