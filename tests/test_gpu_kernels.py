"""Kernel-level parity on the GPU through the C ABI, against the oracle.

Each GPU primitive is compared with the oracle's restatement of the
reference's numpy primitive (apply_heff, update_left_env, update_right_env,
truncated_svd, optimize_two_site) on the same seeded inputs, and with the
golden outputs of the reference modules (tests/golden/ref_primitives.npz).
Tolerance: 1e-12 relative to the largest output magnitude (FP64 with a
different summation order).
"""
import zlib

import numpy as np
import pytest

import dmrg2
from oracle import dmrg2_oracle as O

pytestmark = pytest.mark.gpu
RTOL = 1e-12


def rnd(rng, shape, cplx):
    x = rng.standard_normal(shape)
    if cplx:
        x = x + 1j * rng.standard_normal(shape)
    return x


def close(a, b, rtol=RTOL):
    scale = max(np.abs(b).max(), 1e-300)
    err = np.abs(a - b).max() / scale
    assert err <= rtol, f"relative error {err:.3e} > {rtol:.1e}"


GEMM_SHAPES = [(1, 1, 1), (3, 5, 7), (64, 64, 16), (65, 33, 17), (130, 70, 129), (200, 257, 64)]


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("shape", GEMM_SHAPES)
@pytest.mark.parametrize("ta,tb", [("N", "N"), ("N", "T"), ("T", "N"), ("T", "T"), ("C", "N"), ("R", "N"), ("C", "T")])
def test_gemm_dmma(cplx, shape, ta, tb):
    if not cplx and ta in ("C", "R"):
        pytest.skip("conjugation is the identity for real data")
    rng = np.random.default_rng(zlib.crc32(repr((cplx, shape, ta, tb)).encode()))
    M, N, K = shape
    A = rnd(rng, (K, M) if ta in ("T", "C") else (M, K), cplx)
    B = rnd(rng, (N, K) if tb == "T" else (K, N), cplx)
    C0 = rnd(rng, (M, N), cplx)
    opA = {"N": A, "T": A.T, "C": A.conj().T, "R": A.conj()}[ta]
    opB = B.T if tb == "T" else B
    alpha, beta = (0.75 - 0.5j, 0.25 + 1j) if cplx else (0.75, -0.5)
    ref = alpha * opA @ opB + beta * C0
    out = dmrg2.gemm(A, B, ta, tb, alpha=alpha, beta=beta, C=C0)
    close(out, ref)


SPLIT_SHAPES = [(1, 1, 1), (37, 45, 29), (128, 128, 64), (200, 130, 300), (256, 1024, 256), (96, 40, 1280)]


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("shape", SPLIT_SHAPES)
@pytest.mark.parametrize("ta,tb", [("N", "N"), ("N", "T"), ("T", "N"), ("C", "T")])
def test_gemm_bf16x3_tcgen05(cplx, shape, ta, tb):
    """Precision-form GEMM (three-term BF16 split, FP32 accumulation in tensor memory):
    error below (4e-7 + 2.5e-7 sqrt(K)) of sum_k |a_ik| |b_kj| per entry against the
    FP64 product (split truncation up to ~3 x 2^-24 per product, FP32 accumulation
    growing as sqrt(K))."""
    if not cplx and ta == "C":
        pytest.skip("conjugation is the identity for real data")
    rng = np.random.default_rng(zlib.crc32(repr((cplx, shape, ta, tb, 7)).encode()))
    M, N, K = shape
    A = rnd(rng, (K, M) if ta in ("T", "C") else (M, K), cplx)
    B = rnd(rng, (N, K) if tb == "T" else (K, N), cplx)
    C0 = rnd(rng, (M, N), cplx)
    opA = {"N": A, "T": A.T, "C": A.conj().T}[ta]
    opB = B.T if tb == "T" else B
    alpha, beta = 0.75, -0.5
    ref = alpha * opA @ opB + beta * C0
    out = dmrg2.gemm_bf16x3(A, B, ta, tb, alpha=alpha, beta=beta, C=C0)
    bound = (4e-7 + 2.5e-7 * np.sqrt(K)) * abs(alpha) * (np.abs(opA) @ np.abs(opB)) + 1e-15
    assert np.all(np.abs(out - ref) <= bound), float(np.max(np.abs(out - ref) / bound))
    # and it is not the FP64 product: the split really ran at reduced precision
    if K >= 64:
        assert np.max(np.abs(out - ref)) > 0


@pytest.fixture(scope="module")
def prim(golden_dir):
    return np.load(golden_dir / "ref_primitives.npz")


@pytest.mark.parametrize("tag", ["r0", "r1", "r2", "c0", "c1"])
def test_primitives_vs_reference_golden(prim, tag):
    g = lambda k: prim[f"{tag}_{k}"]
    close(dmrg2.apply_heff(g("L"), g("R"), g("WL"), g("WR"), g("theta")), g("heff"))
    close(dmrg2.update_left_env(g("L"), g("A"), g("WL")), g("lenv"))
    close(dmrg2.update_right_env(g("R"), g("B"), g("WR")), g("renv"))


HEFF_CASES = [
    # cL, cR, d, Dl, Dm, Dr, complex
    (1, 2, 2, 1, 5, 5, False),
    (8, 16, 2, 5, 5, 5, False),
    (31, 33, 2, 5, 5, 5, False),
    (64, 64, 2, 5, 5, 5, False),
    (17, 9, 3, 4, 4, 4, True),
    (25, 25, 5, 4, 4, 4, True),
    (40, 37, 2, 8, 8, 8, False),
    (50, 50, 4, 8, 8, 8, False),
]


@pytest.mark.parametrize("case", HEFF_CASES)
def test_heff_vs_oracle(case):
    cL, cR, d, Dl, Dm, Dr, cplx = case
    rng = np.random.default_rng(cL * 1000 + cR)
    L = rnd(rng, (cL, Dl, cL), cplx)
    R = rnd(rng, (cR, Dr, cR), cplx)
    WL = rnd(rng, (Dl, Dm, d, d), cplx)
    WR = rnd(rng, (Dm, Dr, d, d), cplx)
    th = rnd(rng, (cL, d, d, cR), cplx)
    close(dmrg2.apply_heff(L, R, WL, WR, th), O.apply_heff(L, R, WL, WR, th))


ENV_CASES = [(1, 2, 2, 1, 5, False), (16, 32, 2, 5, 5, False), (33, 31, 2, 5, 5, False),
             (20, 40, 5, 4, 4, True), (64, 64, 2, 8, 8, False), (7, 13, 3, 4, 1, True)]


@pytest.mark.parametrize("case", ENV_CASES)
def test_env_updates_vs_oracle(case):
    c1, c2, d, Dl, Dr, cplx = case
    rng = np.random.default_rng(c1 * 77 + c2)
    Lenv = rnd(rng, (c1, Dl, c1), cplx)
    A = rnd(rng, (c1, d, c2), cplx)
    W = rnd(rng, (Dl, Dr, d, d), cplx)
    close(dmrg2.update_left_env(Lenv, A, W), O.update_left_env(Lenv, A, W))
    Renv = rnd(rng, (c2, Dr, c2), cplx)
    close(dmrg2.update_right_env(Renv, A, W), O.update_right_env(Renv, A, W))


SVD_CASES = [(4, 4, False), (8, 32, False), (32, 8, False), (64, 64, False), (100, 37, False),
             (128, 128, False), (512, 512, False), (40, 40, True), (25, 60, True), (75, 75, True),
             (160, 160, True)]


def graded(rng, m, n, cplx, rate=0.3):
    M = rnd(rng, (m, n), cplx)
    U, s, Vh = np.linalg.svd(M, full_matrices=False)
    s = np.exp(-rate * np.arange(len(s)))
    return (U * s) @ Vh


@pytest.mark.parametrize("m,n,cplx", SVD_CASES)
@pytest.mark.parametrize("direction", ["R", "L"])
def test_density_matrix_split_vs_oracle(m, n, cplx, direction):
    """Default truncation: eigen-decomposition of the reduced density matrix.

    Squared singular values agree to 1e-14 of the largest; the kept factors
    reproduce the oracle's best rank-k approximation; the isometric side is
    orthonormal to 1e-12. Singular values below ~1e-7 of the largest sit in
    the density matrix's rounding floor and are dropped (never kept as noise).
    """
    rng = np.random.default_rng(m * 131 + n)
    rate = 0.3 if min(m, n) < 200 else 0.05
    M = graded(rng, m, n, cplx, rate)
    chi = max(1, min(m, n) - 3)
    left, S, right, te = dmrg2.truncated_svd(M, chi, 0.0, direction)
    s_np = np.linalg.svd(M, compute_uv=False)
    np.testing.assert_allclose(S ** 2, s_np ** 2, rtol=0, atol=1e-14 * s_np[0] ** 2)
    k = left.shape[1]
    assert right.shape == (k, n) and left.shape == (m, k)
    assert k <= chi and k >= min(chi, int(np.sum(s_np > 1e-6 * s_np[0])))
    Uo, So, Vho, teo = O.truncated_svd(M, k)
    assert abs(te - teo) <= 1e-13
    # kept directions with sigma ~1e-6 carry the density matrix's eps/sigma^2 rounding
    close(left @ right, (Uo * So) @ Vho, 1e-8)
    if direction == "R":
        np.testing.assert_allclose(left.conj().T @ left, np.eye(k), atol=1e-12)
    else:
        np.testing.assert_allclose(right @ right.conj().T, np.eye(k), atol=1e-12)


@pytest.mark.parametrize("m,n,cplx", [(4, 4, False), (32, 8, False), (64, 64, False), (100, 37, False),
                                      (40, 40, True), (25, 60, True)])
@pytest.mark.parametrize("direction", ["R", "L"])
def test_jacobi_split_vs_oracle(m, n, cplx, direction):
    """Optional truncation method: one-sided block Jacobi SVD (full relative accuracy)."""
    rng = np.random.default_rng(m * 7 + n)
    M = graded(rng, m, n, cplx)
    chi = max(1, min(m, n) - 3)
    left, S, right, te = dmrg2.truncated_svd(M, chi, 0.0, direction, method="jacobi")
    Uo, So, Vho, teo = O.truncated_svd(M, chi)
    np.testing.assert_allclose(S, np.linalg.svd(M, compute_uv=False), rtol=0, atol=1e-13)
    assert left.shape == (m, chi) and right.shape == (chi, n)
    assert abs(te - teo) <= 1e-13
    close(left @ right, (Uo * So) @ Vho, 1e-12)


@pytest.mark.parametrize("method", ["eig", "jacobi"])
def test_svd_rank_deficient_and_cutoff(method):
    rng = np.random.default_rng(5)
    A = rng.standard_normal((48, 5)) @ rng.standard_normal((5, 40))
    A /= np.linalg.norm(A)
    left, S, right, te = dmrg2.truncated_svd(A, 30, 1e-12, "R", method=method)
    assert left.shape[1] == 5  # cutoff stops at the numerical rank
    assert te < 1e-14  # trace minus kept weight: rounding of the density matrix
    close(left @ right, A, 1e-12)
    np.testing.assert_allclose(left.T @ left, np.eye(5), atol=1e-12)


@pytest.mark.parametrize("method", ["eig", "jacobi"])
def test_svd_degenerate_spectrum(method):
    # exactly degenerate singular values (SU(2) multiplets in Heisenberg chains)
    rng = np.random.default_rng(9)
    Q1, _ = np.linalg.qr(rng.standard_normal((64, 64)))
    Q2, _ = np.linalg.qr(rng.standard_normal((64, 64)))
    s = np.repeat([0.8, 0.4, 0.2, 0.1, 0.05, 0.01, 1e-3, 1e-4], 8)
    M = (Q1 * s) @ Q2.T
    for direction in ("R", "L"):
        left, S, right, te = dmrg2.truncated_svd(M, 24, 0.0, direction, method=method)
        np.testing.assert_allclose(S ** 2, s ** 2, atol=1e-15)
        close(left @ right, (Q1[:, :24] * s[:24]) @ Q2[:, :24].T, 1e-12)
        iso = left.T @ left if direction == "R" else right @ right.T
        np.testing.assert_allclose(iso, np.eye(24), atol=1e-12)


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("cluster", [40, 64])
def test_svd_large_degenerate_cluster(cplx, cluster):
    # one group of `cluster` equal singular values at order 512: 40 members are
    # orthogonalised in shared memory, 64 members (64 x 512 doubles) in global memory.
    # The members share one inverse-iteration shift outside the cluster, so their vectors
    # span the cluster instead of collapsing onto one block of the split tridiagonal:
    # the kept factors reproduce the truncation to 1e-12 (1e-9 with per-member shifts).
    rng = np.random.default_rng(21 + cluster + cplx)
    n = 512
    Q1, _ = np.linalg.qr(rnd(rng, (n, n), cplx))
    Q2, _ = np.linalg.qr(rnd(rng, (n, n), cplx))
    s = np.concatenate([[1.0, 0.7, 0.5, 0.3], np.full(cluster, 0.05),
                        np.geomspace(1e-2, 1e-6, n - 4 - cluster)])
    M = (Q1 * s) @ Q2.conj().T
    keep = cluster + 36
    for direction in ("R", "L"):
        left, S, right, te = dmrg2.truncated_svd(M, keep, 0.0, direction)
        np.testing.assert_allclose(S[:keep] ** 2, s[:keep] ** 2, atol=1e-14)
        close(left @ right, (Q1[:, :keep] * s[:keep]) @ Q2[:, :keep].conj().T, 1e-12)
        iso = left.conj().T @ left if direction == "R" else right @ right.conj().T
        np.testing.assert_allclose(iso, np.eye(keep), atol=1e-12)


@pytest.mark.parametrize("cplx", [False, True])
def test_svd_chained_tail_group(cplx):
    # the tail of a DMRG spectrum: 70 squared singular values 4e-15 apart (below the group
    # tolerance 1e-14 of the largest), so they chain into one group of 70 whose windows hold
    # two earlier members each; below them a gap to values under the noise floor. Kept
    # vectors of values near the floor are accurate to eps / gap ~ 1e-2, hence 5e-8 on the
    # reconstruction (tail singular values ~5e-7).
    rng = np.random.default_rng(77 + cplx)
    n = 512
    Q1, _ = np.linalg.qr(rnd(rng, (n, n), cplx))
    Q2, _ = np.linalg.qr(rnd(rng, (n, n), cplx))
    lam_tail = 3e-13 - 0.4e-14 * np.arange(70)
    s = np.concatenate([[1.0, 0.7, 0.5, 0.3], np.geomspace(0.1, 1e-5, 100), np.sqrt(lam_tail),
                        np.geomspace(1e-8, 1e-9, n - 174)])
    M = (Q1 * s) @ Q2.conj().T
    keep = 174
    for direction in ("R", "L"):
        left, S, right, te = dmrg2.truncated_svd(M, keep + 20, 1e-300, direction)
        assert left.shape[1] == keep  # the values below 16 eps of the largest are dropped
        np.testing.assert_allclose(S[:keep] ** 2, s[:keep] ** 2, atol=1e-14)
        close(left @ right, (Q1[:, :keep] * s[:keep]) @ Q2[:, :keep].conj().T, 5e-8)
        iso = left.conj().T @ left if direction == "R" else right @ right.conj().T
        np.testing.assert_allclose(iso, np.eye(keep), atol=1e-12)


@pytest.mark.parametrize("cplx", [False, True])
def test_lanczos_vs_dense(cplx):
    rng = np.random.default_rng(3 + cplx)
    cL, cR, d, D = 6, 7, 2, 3
    if cplx:
        d = 3
    L = rnd(rng, (cL, D, cL), cplx)
    R = rnd(rng, (cR, D, cR), cplx)
    WL = rnd(rng, (D, D, d, d), cplx)
    WR = rnd(rng, (D, D, d, d), cplx)
    # hermitise the environments and MPO so H_eff is Hermitian
    L = L + np.transpose(L, (2, 1, 0)).conj()
    R = R + np.transpose(R, (2, 1, 0)).conj()
    WL = WL + np.transpose(WL, (0, 1, 3, 2)).conj()
    WR = WR + np.transpose(WR, (0, 1, 3, 2)).conj()
    n = cL * d * d * cR
    H = np.zeros((n, n), complex)
    for j in range(n):
        e = np.zeros(n)
        e[j] = 1
        H[:, j] = O.apply_heff(L, R, WL, WR, e.reshape(cL, d, d, cR)).ravel()
    assert np.abs(H - H.conj().T).max() < 1e-10 * np.abs(H).max()
    w, V = np.linalg.eigh(H)
    th0 = rnd(rng, (cL, d, d, cR), cplx)
    e, th = dmrg2.optimize_two_site(L, R, WL, WR, th0, max_iter=100, tol=1e-13, max_restarts=8)
    assert abs(e - w[0]) <= 1e-10 * abs(w).max()
    ov = abs(np.vdot(V[:, 0], th.ravel()))
    assert abs(ov - 1.0) < 1e-8
    assert abs(np.linalg.norm(th) - 1.0) < 1e-12


def _orth_rows(X):
    q, _ = np.linalg.qr(X.T)
    return q.T


@pytest.mark.parametrize("m,n,k,direction", [(64, 64, 20, "R"), (96, 64, 32, "L"), (128, 160, 48, "R"),
                                             (256, 200, 100, "L"), (512, 512, 256, "R"), (512, 512, 256, "L"),
                                             (40, 64, 8, "R"), (100, 90, 37, "R"), (700, 640, 300, "R"),
                                             (640, 700, 480, "L")])
def test_warm_split_vs_numpy(m, n, k, direction):
    """The warm-started subspace split (three CholeskyQR power steps) against numpy's SVD:
    M has singular values 1 .. 1e-2 on the kept k and a gap of 100 below them; the warm
    factor is last split's subspace perturbed by 1e-3. The kept factor is orthonormal to
    1e-13, its projector equals the top-k singular projector to 1e-9, the other factor is
    its projection of M, and the discarded weight matches to 1e-12 relative to |M|^2."""
    rng = np.random.default_rng(m * 7 + n + k)
    r = min(m, n)
    U, _ = np.linalg.qr(rng.standard_normal((m, r)))
    V, _ = np.linalg.qr(rng.standard_normal((n, r)))
    s = np.concatenate([np.logspace(0, -2, k), 1e-4 * np.logspace(0, -3, r - k)])
    M = (U * s) @ V.T
    if direction == "R":
        warm = _orth_rows(V[:, :k].T + 1e-3 * rng.standard_normal((k, n)))
    else:
        warm = _orth_rows(U[:, :k].T + 1e-3 * rng.standard_normal((k, m))).T
    left, right, te = dmrg2.warm_split(M, warm, k, direction)
    Pk = U[:, :k] @ U[:, :k].T
    Qk = V[:, :k] @ V[:, :k].T
    if direction == "R":
        np.testing.assert_allclose(left.T @ left, np.eye(k), atol=1e-13)
        assert np.abs(left @ left.T - Pk).max() < 1e-9
        np.testing.assert_allclose(right, left.T @ M, atol=1e-13)
    else:
        np.testing.assert_allclose(right @ right.T, np.eye(k), atol=1e-13)
        assert np.abs(right.T @ right - Qk).max() < 1e-9
        np.testing.assert_allclose(left, M @ right.T, atol=1e-13)
    assert abs(te - np.sum(s[k:] ** 2)) <= 1e-12 * np.sum(s ** 2)


@pytest.mark.parametrize("direction", ["R", "L"])
def test_warm_split_wide_kept_spectrum(direction):
    """Kept singular values spanning 1 .. 1e-9 (a DMRG bond at a large bond cap keeps
    Schmidt values far below 1e-6 of the largest): the shifted CholeskyQR pass keeps the
    split on the warm path (no fallback), the kept factor is orthonormal to 1e-13 and
    spans the top-k singular space to 1e-6 (rounding fixes the directions of singular
    values near 1e-9 only to ~u/1e-9 ~ 1e-7, for an exact SVD as well), and the
    discarded weight matches to 1e-12 of |M|^2."""
    rng = np.random.default_rng(11)
    m = n = 512
    k = 256
    U, _ = np.linalg.qr(rng.standard_normal((m, m)))
    V, _ = np.linalg.qr(rng.standard_normal((n, n)))
    s = np.concatenate([np.logspace(0, -9, k), 1e-11 * np.logspace(0, -3, m - k)])
    M = (U * s) @ V.T
    if direction == "R":
        warm = _orth_rows(V[:, :k].T + 1e-6 * rng.standard_normal((k, n)))
    else:
        warm = _orth_rows(U[:, :k].T + 1e-6 * rng.standard_normal((k, m))).T
    left, right, te = dmrg2.warm_split(M, warm, k, direction)
    if direction == "R":
        np.testing.assert_allclose(left.T @ left, np.eye(k), atol=1e-13)
        assert np.abs(left @ left.T - U[:, :k] @ U[:, :k].T).max() < 1e-6
    else:
        np.testing.assert_allclose(right @ right.T, np.eye(k), atol=1e-13)
        assert np.abs(right.T @ right - V[:, :k] @ V[:, :k].T).max() < 1e-6
    assert abs(te - np.sum(s[k:] ** 2)) <= 1e-12 * np.sum(s ** 2)


def test_warm_split_gives_up_on_a_rank_deficient_factor():
    """A warm factor with directions outside the range of M makes CholeskyQR's Gram
    matrix singular: the split reports DMRG2_ERR_NUMERIC (the engine then runs the exact
    split) instead of returning a non-orthonormal factor."""
    rng = np.random.default_rng(3)
    m, n, k = 64, 64, 16
    M = rng.standard_normal((m, 8)) @ rng.standard_normal((8, n))  # rank 8 < k
    warm = _orth_rows(rng.standard_normal((k, n)))
    with pytest.raises(dmrg2.Dmrg2Error, match=f"status {dmrg2.ERR_NUMERIC}"):
        dmrg2.warm_split(M, warm, k, "R")


TUNE_CHILD = r"""
import numpy as np, dmrg2
rng = np.random.default_rng(5)
worst = 0.0
for (m, n, k, ta, tb) in [(512, 256, 512, "N", "N"), (256, 256, 1024, "T", "N"), (1024, 256, 1280, "N", "T"),
                          (300, 200, 700, "N", "N")]:
    A = rng.standard_normal((k, m) if ta == "T" else (m, k))
    B = rng.standard_normal((n, k) if tb == "T" else (k, n))
    C0 = rng.standard_normal((m, n))
    ref = 0.5 * ((A.T if ta == "T" else A) @ (B.T if tb == "T" else B)) - 2.0 * C0
    for rep in range(2):  # the first call of a shape tunes it, the second uses the choice
        out = dmrg2.gemm(A, B, ta, tb, alpha=0.5, beta=-2.0, C=C0.copy())
        worst = max(worst, float(np.abs(out - ref).max() / np.abs(ref).max()))
print("worst", worst)
"""


def test_gemm_autotuner_choices_match_numpy():
    """DMRG2_GEMM_TUNE=1: GEMMs of at least 1e8 flop are timed in every configuration
    (64x64 tiles with 1-8 K slices summed in a cluster, 32x32 tiles with 1-4) on their
    first call and run with the fastest afterwards; whichever is chosen, the result
    matches numpy to FP64 rounding (beta != 0 included: the timing writes a scratch
    output, not the caller's C)."""
    import os
    import subprocess
    import sys
    from pathlib import Path
    repo = Path(__file__).resolve().parent.parent
    env = dict(os.environ, DMRG2_GEMM_TUNE="1",
               PYTHONPATH=os.pathsep.join([str(repo / "dmrg-implementations_b200"), str(repo)]))
    r = subprocess.run([sys.executable, "-c", TUNE_CHILD], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    worst = float(r.stdout.split("worst")[1])
    print("autotuned GEMMs: worst relative error", worst)
    assert worst < 1e-13
