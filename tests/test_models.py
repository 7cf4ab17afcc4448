"""The package's MPO builders and seeded states (used by bench.py's GPU legs)
agree with the oracle's: the same tensors for XXZ and the Josephson array, the
same Hamiltonian for the long-range chains, the same seeded MPS."""
import numpy as np
import pytest

from dmrg2 import models as P
from oracle import dmrg2_oracle as O
from oracle import models as M


@pytest.mark.parametrize("L,J,delta,hz", [(2, 1.0, 1.0, 0.0), (7, 0.8, 0.6, 0.3), (12, 1.0, 1.0, 0.0)])
def test_xxz_equals_oracle(L, J, delta, hz):
    for a, b in zip(P.xxz(L, J, delta, hz), M.heisenberg_mpo(L, J, delta, hz)):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("onsite", ["reference", "shifted"])
def test_josephson_equals_oracle(onsite):
    kw = dict(n_max=2, E_J=2.0, E_C=1.0, n_g=0.25, phi=0.26, onsite=onsite)
    for a, b in zip(P.josephson(6, **kw), M.josephson_mpo(6, **kw)):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("Js", [[1.0, 0.35], [1.0, 0.4, 0.2]])
def test_longrange_hamiltonian_equals_oracle(Js):
    L = 7
    Hp = M.mpo_to_dense(P.heisenberg_range(L, Js))
    Ho = M.mpo_to_dense(M.longrange_heisenberg_mpo(L, Js))
    np.testing.assert_allclose(Hp, Ho, atol=1e-14)
    assert P.j1j2(L, *Js[:2])[3].shape[0] == 8


@pytest.mark.parametrize("dtype", [np.float64, np.complex128])
def test_random_mps_equals_oracle(dtype):
    for a, b in zip(P.random_mps(20, 2, 16, seed=3, dtype=dtype), O.random_mps(20, 2, 16, seed=3, dtype=dtype)):
        np.testing.assert_array_equal(a, b)
