"""The real embedding that the complex CholeskyQR passes run on (the randomised split and the
complex warm-started split): a complex column block Y (len x r) becomes the real
2 len x 2 r matrix whose column pair (2j, 2j+1) is the real image of (y_j, i y_j), with row
2i holding real parts and row 2i+1 imaginary parts (the layout of embed_pairs_kernel).

Checked in numpy, without a GPU: real CholeskyQR on that embedding (Gram matrix, Cholesky
factor, triangular solve) yields, in its even columns, the complex Gram-Schmidt basis of
Y. That is the complex QR factor up to unit phases: orthonormal, triangular in the columns,
and the same column spans in order. A Newton-Schulz step on the embedding equals the
embedding of the complex step."""
import numpy as np


def embed_pairs(Y):
    n, r = Y.shape
    E = np.zeros((2 * n, 2 * r))
    E[0::2, 0::2] = Y.real
    E[0::2, 1::2] = -Y.imag
    E[1::2, 0::2] = Y.imag
    E[1::2, 1::2] = Y.real
    return E


def extract_pairs(Q):
    return Q[0::2, 0::2] + 1j * Q[1::2, 0::2]


def cholqr(E):
    G = E.T @ E
    Lc = np.linalg.cholesky(G)
    return np.linalg.solve(Lc, E.T).T  # E L^{-T}


def test_embedding_represents_complex_products():
    rng = np.random.default_rng(0)
    A = rng.standard_normal((7, 5)) + 1j * rng.standard_normal((7, 5))
    B = rng.standard_normal((5, 3)) + 1j * rng.standard_normal((5, 3))
    np.testing.assert_allclose(embed_pairs(A) @ embed_pairs(B), embed_pairs(A @ B), atol=1e-12)
    np.testing.assert_allclose(embed_pairs(A).T, embed_pairs(A.conj().T), atol=0)


def test_cholqr_on_the_embedding_is_complex_gram_schmidt():
    rng = np.random.default_rng(1)
    n, r = 40, 9
    # a block with spread singular values, as a warm start's theta B^H has
    U, _ = np.linalg.qr(rng.standard_normal((n, r)) + 1j * rng.standard_normal((n, r)))
    V, _ = np.linalg.qr(rng.standard_normal((r, r)) + 1j * rng.standard_normal((r, r)))
    Y = U @ np.diag(np.logspace(0, -3, r)) @ V
    Q = extract_pairs(cholqr(embed_pairs(Y)))
    np.testing.assert_allclose(Q.conj().T @ Q, np.eye(r), atol=1e-9)
    Qr, Rr = np.linalg.qr(Y)
    # the same basis as complex QR up to a unit phase per column (triangular in the columns)
    ph = np.diag(Qr.conj().T @ Q)
    np.testing.assert_allclose(np.abs(ph), 1.0, atol=1e-8)
    np.testing.assert_allclose(Q, Qr * ph, atol=1e-8)
    # and the odd columns are i times the even ones
    Qe = cholqr(embed_pairs(Y))
    np.testing.assert_allclose(Qe[:, 1::2], np.vstack([-Qe[1::2, 0::2], Qe[0::2, 0::2]])[
        np.argsort(np.r_[np.arange(0, 2 * n, 2), np.arange(1, 2 * n, 2)])], atol=1e-8)


def test_newton_schulz_step_commutes_with_the_embedding():
    rng = np.random.default_rng(2)
    Z, _ = np.linalg.qr(rng.standard_normal((30, 6)) + 1j * rng.standard_normal((30, 6)))
    Z = Z + 1e-4 * (rng.standard_normal(Z.shape) + 1j * rng.standard_normal(Z.shape))
    step = lambda X, H: 1.5 * X - 0.5 * X @ (H(X) @ X)
    Zc = step(Z, lambda X: X.conj().T)
    Ze = step(embed_pairs(Z), lambda X: X.T)
    np.testing.assert_allclose(Ze, embed_pairs(Zc), atol=1e-12)
    np.testing.assert_allclose(extract_pairs(Ze), Zc, atol=1e-12)
