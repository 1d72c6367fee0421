"""Batched Lanczos: many operators advance in lockstep, one launch per kernel
per step.  Every result is checked against the oracle's dense spectrum of the
same sector / instance (E0 <= 1e-10 relative for FP64, <= 1e-9 mixed)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def xxz(S, delta):
    return S((1.0, "xx"), (1.0, "yy"), (delta, "zz"))


def test_all_momentum_sectors_in_one_batch(ek, O):
    """L=12, N=6, k=0..11 (k=0 and k=6 real, the others complex) batched."""
    L = 12
    ops, refs = [], []
    for k in range(L):
        b = ek.TranslationalBasis(L=L, N=6, k=k)
        ops.append(ek.trans_inv_operator(xxz(ek.spin, 1.5), 2, b))
        Ho = O.trans_inv_operator(xxz(O.spin, 1.5), 2, O.translational(L, k=k, N=6))
        refs.append(np.linalg.eigvalsh(Ho.dense())[:2])
    ev, info = ek.batch_lanczos_e0(ops, m=80, nev=2, tol=1e-13, check_every=5)
    for k in range(L):
        assert np.allclose(ev[k], refs[k], rtol=0, atol=1e-10 * abs(refs[k][0])), k


def random_field_instance(ek, O, L, rng):
    h = rng.uniform(-3, 3, L)
    mats = [xxz(ek.spin, 1.0)] * (L - 1) + [hi * ek.spin("z") for hi in h]
    omats = [xxz(O.spin, 1.0)] * (L - 1) + [hi * O.spin("z") for hi in h]
    inds = [[i, i + 1] for i in range(1, L)] + [[i] for i in range(1, L + 1)]
    b = ek.ProjectedBasis(L=L, N=L // 2)
    H = ek.operator(mats, inds, b)
    Ho = O.operator(omats, inds, O.projected(L, N=L // 2))
    return H, Ho


def test_random_field_ensemble_ragged(ek, O):
    """Disorder instances of uneven dimension (L in {8, 10, 12}) in one batch:
    E0 and the gap ratio of the converged low-lying Ritz values."""
    rng = np.random.default_rng(42)
    Ls = [8, 10, 12, 10, 8, 12, 12, 8]
    ops, dense = [], []
    for L in Ls:
        H, Ho = random_field_instance(ek, O, L, rng)
        ops.append(H)
        dense.append(np.linalg.eigvalsh(Ho.dense()))
    assert all(op.n_families == 1 for op in ops)
    ev, info = ek.batch_lanczos_e0(ops, m=200, nev=4, tol=1e-13, check_every=5)
    for q in range(len(Ls)):
        assert np.allclose(ev[q], dense[q][:4], rtol=0, atol=1e-9 * abs(dense[q][0])), q
        r = ek.gapratio(ev[q])
        assert np.allclose(r, O.gapratio(dense[q][:4]), atol=1e-6)


def test_mixed_precision_batch(ek):
    rng = np.random.default_rng(5)
    ops = []
    for L in (14, 16, 14, 16):
        h = rng.uniform(-3, 3, L)
        mats = [xxz(ek.spin, 1.0)] * (L - 1) + [hi * ek.spin("z") for hi in h]
        inds = [[i, i + 1] for i in range(1, L)] + [[i] for i in range(1, L + 1)]
        ops.append(ek.operator(mats, inds, ek.ProjectedBasis(L=L, N=L // 2)))
    e64, _ = ek.batch_lanczos_e0(ops, m=200, tol=1e-13, check_every=5)
    emx, info = ek.batch_lanczos_e0(ops, m=200, tol=1e-13, check_every=5, precision="mixed")
    assert np.all(np.abs(emx[:, 0] - e64[:, 0]) <= 1e-9 * np.abs(e64[:, 0]))
    assert info["steps_low"] > 0


def test_single_operator_matches_batch(ek):
    b = ek.TranslationalBasis(L=16, N=8, k=0)
    H = ek.trans_inv_operator(xxz(ek.spin, 1.0), 2, b)
    v0 = np.random.default_rng(1).standard_normal(b.size(1))
    e1, _ = ek.lanczos_e0(H, v0, m=60)
    e2, _ = ek.batch_lanczos_e0([H], [v0], m=60)
    assert abs(e1[0] - e2[0, 0]) < 1e-13 * abs(e1[0])


def test_mixed_precision_nev4_matches_fp64(ek, O):
    """The four lowest eigenvalues of each sector agree between the mixed
    (FP32 Krylov vectors + FP64 refinement) and the FP64 batched paths and the
    dense spectrum."""
    L = 14
    ops, dense = [], []
    for k in (0, 1, 7):
        b = ek.TranslationalBasis(L=L, N=7, k=k)
        ops.append(ek.trans_inv_operator(xxz(ek.spin, 1.5), 2, b))
        Ho = O.trans_inv_operator(xxz(O.spin, 1.5), 2, O.translational(L, k=k, N=7))
        dense.append(np.linalg.eigvalsh(Ho.dense())[:4])
    emx, _ = ek.batch_lanczos_e0(ops, m=150, nev=4, tol=1e-12, check_every=5, precision="mixed")
    e64, _ = ek.batch_lanczos_e0(ops, m=150, nev=4, tol=1e-12, check_every=5)
    for q in range(3):
        assert np.allclose(e64[q], dense[q], rtol=0, atol=1e-9 * abs(dense[q][0])), q
        assert np.allclose(emx[q], dense[q], rtol=0, atol=1e-9 * abs(dense[q][0])), q


def test_materialized_batch_and_krylov(ek, O):
    """Lanczos batches and Krylov evolution on materialised operators give the
    matrix-free results."""
    L = 12
    ops, refs = [], []
    for k in range(L):
        b = ek.TranslationalBasis(L=L, N=6, k=k)
        H = ek.trans_inv_operator(xxz(ek.spin, 1.5), 2, b)
        H.sparse_()
        ops.append(H)
        Ho = O.trans_inv_operator(xxz(O.spin, 1.5), 2, O.translational(L, k=k, N=6))
        refs.append(np.linalg.eigvalsh(Ho.dense())[:2])
    ev, _ = ek.batch_lanczos_e0(ops, m=80, nev=2, tol=1e-13, check_every=5)
    for k in range(L):
        assert np.allclose(ev[k], refs[k], rtol=0, atol=1e-10 * abs(refs[k][0])), k
    H = ops[3]
    rng = np.random.default_rng(3)
    psi0 = rng.standard_normal(H.size(1)) + 1j * rng.standard_normal(H.size(1))
    psi0 /= np.linalg.norm(psi0)
    a = ek.timeevolve(H, psi0, [0.5, 2.0], tol=1e-11)
    H.clear_sparse_cache_()
    b_ = ek.timeevolve(H, psi0, [0.5, 2.0], tol=1e-11)
    assert np.linalg.norm(a - b_) < 1e-9


def test_mixed_ensemble_all_four_levels(ek, O):
    """Every one of the four lowest levels of a disorder ensemble (some with
    close levels) from the mixed path matches the FP64 batched path and, for
    the small chains, the dense spectrum."""
    rng = np.random.default_rng(2024)
    ops, dense = [], []
    for q in range(24):
        L = (10, 12, 14)[q % 3]
        H, Ho = random_field_instance(ek, O, L, rng)
        ops.append(H)
        dense.append(np.linalg.eigvalsh(Ho.dense())[:4] if L <= 12 else None)
    e64, _ = ek.batch_lanczos_e0(ops, m=200, nev=4, tol=1e-12, check_every=10)
    emx, info = ek.batch_lanczos_e0(ops, m=200, nev=4, tol=1e-12, check_every=10,
                                    precision="mixed")
    for q in range(len(ops)):
        assert np.allclose(emx[q], e64[q], rtol=0, atol=1e-9 * abs(e64[q][0])), q
        if dense[q] is not None:
            assert np.allclose(e64[q], dense[q], rtol=0, atol=1e-9 * abs(dense[q][0])), q


def test_large_krylov_capacity_takes_the_two_pass_sweep(ek, O):
    """With room for 7,000 Krylov vectors the fused update + dot-product pass
    no longer fits its shared memory, and the second sweep runs as separate
    dot-product and update passes: same eigenvalues as the fused path and the
    dense spectrum."""
    ops, dense = [], []
    for L, k in ((14, 0), (16, 3), (14, 5)):
        b = ek.TranslationalBasis(L=L, N=L // 2, k=k)
        ops.append(ek.trans_inv_operator(xxz(ek.spin, 1.5), 2, b))
        Ho = O.trans_inv_operator(xxz(O.spin, 1.5), 2, O.translational(L, k=k, N=L // 2))
        dense.append(np.linalg.eigvalsh(Ho.dense())[:2])
    big, _ = ek.batch_lanczos_e0(ops, m=7000, nev=2, tol=1e-12, check_every=5)
    small, _ = ek.batch_lanczos_e0(ops, m=150, nev=2, tol=1e-12, check_every=5)
    for q in range(3):
        assert np.allclose(big[q], dense[q], rtol=0, atol=1e-10 * abs(dense[q][0])), q
        assert np.allclose(big[q], small[q], rtol=0, atol=1e-11 * abs(dense[q][0])), q
