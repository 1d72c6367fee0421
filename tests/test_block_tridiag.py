"""Host logic of the block Lanczos eigenvalue step (no GPU): lowest distinct
eigenvalues of Hermitian block-tridiagonal matrices, including the removal
of the copies a block Lanczos run without full re-orthogonalisation makes."""
import ctypes as C

import numpy as np

import __graft_entry__ as ge

ek = ge.load_package()
from edkit_b200 import _lib as E  # noqa: E402


def lowest(A, B, nev):
    m, p = len(A), A[0].shape[0]
    a = np.ascontiguousarray(np.stack([x.T for x in A]).astype(np.complex128)).view(np.float64)
    b = np.ascontiguousarray(np.stack([x.T for x in B]).astype(np.complex128)).view(np.float64) \
        if B else np.zeros(2)
    out = np.zeros(nev)
    E.check(E.load().edk_block_tridiag_lowest(p, m, E.ptr(a), E.ptr(b), nev, E.ptr(out)))
    return out


def assemble(A, B):
    m, p = len(A), A[0].shape[0]
    T = np.zeros((m * p, m * p), np.complex128)
    for j in range(m):
        T[j * p:(j + 1) * p, j * p:(j + 1) * p] = A[j]
        if j >= 1:
            T[j * p:(j + 1) * p, (j - 1) * p:j * p] = B[j - 1]
            T[(j - 1) * p:j * p, j * p:(j + 1) * p] = B[j - 1].conj().T
    return T


def herm(rng, p):
    X = rng.standard_normal((p, p)) + 1j * rng.standard_normal((p, p))
    return (X + X.conj().T) / 2


def block_lanczos_T(H, p, m, rng, full_reorth):
    """Block tridiagonal T of a block Lanczos run on the dense Hermitian H."""
    n = H.shape[0]
    V, _ = np.linalg.qr(rng.standard_normal((n, p)) + 1j * rng.standard_normal((n, p)))
    Vs = [V]
    A, B = [], []
    Vp, Bprev = np.zeros((n, p)), np.zeros((p, p))
    for j in range(m):
        W = H @ V - Vp @ Bprev.conj().T
        Aj = V.conj().T @ W
        W = W - V @ Aj
        if full_reorth:
            for _ in range(2):
                for U in Vs:
                    W = W - U @ (U.conj().T @ W)
        A.append((Aj + Aj.conj().T) / 2)
        Qn, R = np.linalg.qr(W)
        if j < m - 1:
            B.append(R)
        Vp, V, Bprev = V, Qn, R
        Vs.append(V)
    return A, B


def test_ritz_values_of_block_lanczos_T():
    """T from block Lanczos runs with full re-orthogonalisation: the lowest
    distinct eigenvalues of T itself (no copies to remove)."""
    rng = np.random.default_rng(0)
    for p, m, n in ((1, 30, 80), (3, 10, 90), (8, 6, 100)):
        X = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
        H = (X + X.conj().T) / 2
        A, B = block_lanczos_T(H, p, m, rng, True)
        w = np.linalg.eigvalsh(assemble(A, B))
        got = lowest(A, B, 4)
        assert np.allclose(got, w[:4], rtol=0, atol=1e-10 * max(1, abs(w[0]))), (p, m)


def test_single_block():
    rng = np.random.default_rng(1)
    A = [herm(rng, 5)]
    assert np.allclose(lowest(A, [], 3), np.linalg.eigvalsh(A[0])[:3], atol=1e-12)


def test_block_lanczos_on_dense_matrix_without_reorthogonalisation():
    """Run the block recurrence (local orthogonalisation only) on a dense
    Hermitian matrix long enough for converged eigenvalues to repeat in T;
    the filtered lowest values are the matrix's lowest distinct ones."""
    rng = np.random.default_rng(2)
    n, p, m = 60, 2, 40  # p * m > n: the recurrence keeps going past convergence
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    lam = np.sort(np.concatenate([[-3.0, -2.5, -2.2], rng.uniform(-2, 2, n - 3)]))
    H = (Q * lam) @ Q.T
    A, B = block_lanczos_T(H, p, m, rng, False)
    T = assemble(A, B)
    wT = np.linalg.eigvalsh(T)
    assert np.sum(np.abs(wT - lam[0]) < 1e-8) >= 2  # the lowest level repeats in T
    got = lowest(A, B, 3)
    assert np.allclose(got, lam[:3], rtol=0, atol=1e-8), got
