"""MPS/MPO file formats (dmrg2.io) against the reference's own data files.

tests/golden/*.bin are copies of the reference's benchmarks/data files (written
by its benchmarks/data/generate.py from quimb objects); heis_L12_*.npz come from
its benchmark_data/regular tier. The .bin MPO orientation is pinned by the
complex Josephson file: <psi|H|psi> of the file's own random state with the
loaded MPO equals the same expectation with the engine's Josephson builder at
the file's parameters (E_J=1, E_C=0.5, phi=pi/4, n_max=2), while the
transposed reading does not."""
import numpy as np
import pytest

from dmrg2 import io, models as P
from oracle import dmrg2_oracle as O


def test_bin_mpo_orientation_pinned_by_complex_josephson(golden_dir):
    W = io.load_mpo_bin(golden_dir / "josephson_L12_n2_mpo.bin")
    A = io.load_mps_bin(golden_dir / "josephson_L12_n2_chi10_mps.bin")
    assert [w.shape for w in W[:2]] == [(1, 4, 5, 5), (4, 4, 5, 5)] and A[1].shape == (10, 5, 10)
    ref = P.josephson(12, n_max=2, E_J=1.0, E_C=0.5, n_g=0.0, phi=np.pi / 4, onsite="reference")
    e_file, e_ref = O.mpo_expectation(A, W), O.mpo_expectation(A, ref)
    assert abs(e_file - e_ref) <= 1e-12 * abs(e_ref)
    e_t = O.mpo_expectation(A, [w.transpose(0, 1, 3, 2) for w in W])
    assert abs(e_t - e_ref) > 1e-3


def test_bin_heisenberg_matches_builder(golden_dir):
    W = io.load_mpo_bin(golden_dir / "heisenberg_L12_mpo.bin")
    A = io.load_mps_bin(golden_dir / "heisenberg_L12_chi10_mps.bin")
    e1, e2 = O.mpo_expectation(A, W), O.mpo_expectation(A, P.xxz(12))
    assert abs(e1 - e2) <= 1e-12


def test_bin_round_trips(tmp_path):
    rng = np.random.default_rng(0)
    mps = P.random_mps(9, 3, 7, seed=1, dtype=np.complex128)
    io.save_mps_bin(tmp_path / "a.bin", mps)
    for a, b in zip(mps, io.load_mps_bin(tmp_path / "a.bin")):
        np.testing.assert_array_equal(a, b)
    mpo = P.josephson(5, n_max=1, E_J=1.3, E_C=0.7, phi=0.4)
    mpo[2] = mpo[2] + 1e-3 * rng.standard_normal(mpo[2].shape)
    io.save_mpo_bin(tmp_path / "w.bin", mpo)
    for a, b in zip(mpo, io.load_mpo_bin(tmp_path / "w.bin")):
        np.testing.assert_array_equal(a, b)


def test_bin_truncated_file_is_rejected(tmp_path, golden_dir):
    raw = (golden_dir / "heisenberg_L12_chi10_mps.bin").read_bytes()
    (tmp_path / "t.bin").write_bytes(raw[: len(raw) - 100])
    with pytest.raises(ValueError):
        io.load_mps_bin(tmp_path / "t.bin")


def test_npz_fixtures_and_orders(tmp_path, golden_dir):
    W = io.load_mpo_npz(golden_dir / "heis_L12_mpo.npz")
    A = io.load_mps_npz(golden_dir / "heis_L12_mps.npz")
    for a, b in zip(W, O.load_npz_mpo(golden_dir / "heis_L12_mpo.npz")):
        np.testing.assert_array_equal(a, b)
    for a, b in zip(A, O.load_npz_mps(golden_dir / "heis_L12_mps.npz")):
        np.testing.assert_array_equal(a, b)
    # quimb-ordered (chi_l, chi_r, d) bulk with (chi, d) ends reads back to the same state
    q = {f"tensor_{i}": (a[0].T if i == 0 else a[:, :, 0] if i == len(A) - 1 else a.transpose(0, 2, 1))
         for i, a in enumerate(A)}
    np.savez(tmp_path / "q.npz", **q)
    for a, b in zip(A, io.load_mps_npz(tmp_path / "q.npz")):
        np.testing.assert_array_equal(a, b)
    # checkpoint round trip
    io.save_mps_npz(tmp_path / "c.npz", A, energy=-5.14)
    for a, b in zip(A, io.load_mps_npz(tmp_path / "c.npz")):
        np.testing.assert_array_equal(a, b)


def test_minimal_bonds_keeps_the_state(golden_dir):
    """quimb-style MPS with one bond dimension everywhere (the reference's .bin state:
    bond 1 of 10 at d=5) reduces exactly to the minimal bonds the engine allocates."""
    import dmrg2
    A = io.load_mps_bin(golden_dir / "josephson_L12_n2_chi10_mps.bin")
    assert A[0].shape[2] == 10 and A[0].shape[1] == 5
    B = dmrg2.minimal_bonds(A)
    assert B[0].shape[2] == 5 and B[-1].shape[0] == 5
    W = io.load_mpo_bin(golden_dir / "josephson_L12_n2_mpo.bin")
    e1 = O.mpo_expectation(A, W) / O.mps_norm2(A)
    e2 = O.mpo_expectation(B, W) / O.mps_norm2(B)
    assert abs(e1 - e2) <= 1e-12 * abs(e1)
