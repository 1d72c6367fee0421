"""Block Lanczos (a block of right-hand sides per operator, many operators in
one batch) against the oracle's dense spectra: the lowest distinct
eigenvalues agree to 1e-9 relative."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def xxz(S, delta):
    return S((1.0, "xx"), (1.0, "yy"), (delta, "zz"))


def distinct(ev, n, tol=1e-8):
    out = []
    for x in np.sort(ev):
        if not out or x - out[-1] > tol * max(1.0, abs(x)):
            out.append(x)
    return np.array(out[:n])


def sectors(ek, O, L, N, delta, ks):
    ops, refs = [], []
    for k in ks:
        b = ek.TranslationalBasis(L=L, N=N, k=k)
        ops.append(ek.trans_inv_operator(xxz(ek.spin, delta), 2, b))
        Ho = O.trans_inv_operator(xxz(O.spin, delta), 2, O.translational(L, k=k, N=N))
        refs.append(np.linalg.eigvalsh(Ho.dense()))
    return ops, refs


def check(ev, refs, nev, tol=1e-9):
    for q, r in enumerate(refs):
        want = distinct(r, nev)
        assert np.allclose(ev[q][:len(want)], want, rtol=0, atol=tol * abs(want[0])), (q, ev[q], want)


def test_all_momentum_sectors_block8(ek, O):
    L = 14
    ops, refs = sectors(ek, O, L, 7, 1.5, range(L))
    ev, info = ek.block_lanczos(ops, block=8, m=24, nev=4, check_every=0)
    assert info["steps"] == 24 and info["matvecs"] == 24 * 8 * L
    check(ev, refs, 4)


def test_explicit_start_blocks_and_tol_stop(ek, O):
    L = 14
    ops, refs = sectors(ek, O, L, 7, 1.0, (0, 3, 7))
    rng = np.random.default_rng(9)
    x0 = [rng.standard_normal((op.size(1), 16)) + 1j * rng.standard_normal((op.size(1), 16))
          for op in ops]
    ev, info = ek.block_lanczos(ops, x0, block=16, m=14, nev=3, tol=1e-12, check_every=2)
    check(ev, refs, 3)
    ev2, _ = ek.block_lanczos(ops, block=16, m=14, nev=3, check_every=0, seed=7)
    assert np.allclose(ev, ev2, rtol=0, atol=1e-9 * abs(ev[0, 0]))


def test_materialized_sectors_match(ek, O):
    L = 14
    ops, refs = sectors(ek, O, L, 7, 1.5, (0, 1, 5, 7))
    for op in ops:
        op.sparse_()
    ev, _ = ek.block_lanczos(ops, block=8, m=24, nev=4, check_every=0)
    check(ev, refs, 4)


def test_projected_ensemble_with_fields(ek, O):
    """Open random-field chains of one size (ProjectedBasis, fast kernel with
    diagonal terms) and a 64-wide block."""
    rng = np.random.default_rng(11)
    L = 14
    ops, refs = [], []
    for _ in range(3):
        h = rng.uniform(-3, 3, L)
        mats = [xxz(ek.spin, 1.0)] * (L - 1) + [hi * ek.spin("z") for hi in h]
        omats = [xxz(O.spin, 1.0)] * (L - 1) + [hi * O.spin("z") for hi in h]
        inds = [[i, i + 1] for i in range(1, L)] + [[i] for i in range(1, L + 1)]
        ops.append(ek.operator(mats, inds, ek.ProjectedBasis(L=L, N=L // 2)))
        refs.append(np.linalg.eigvalsh(O.operator(omats, inds, O.projected(L, N=L // 2)).dense()))
    ev, _ = ek.block_lanczos(ops, block=64, m=20, nev=4, check_every=0)
    check(ev, refs, 4)


def test_generic_kernel_operators(ek, O):
    """AbelianBasis sectors run on the column kernels inside the block engine."""
    L = 16
    ops, refs = [], []
    for k in (0, 2):
        b = ek.basis(L=L, N=8, k=k, z=1)
        ops.append(ek.trans_inv_operator(xxz(ek.spin, 1.5), 2, b))
        Ho = O.trans_inv_operator(xxz(O.spin, 1.5), 2, O.basis(L, N=8, k=k, z=1))
        refs.append(np.linalg.eigvalsh(Ho.dense()))
    ev, _ = ek.block_lanczos(ops, block=8, m=36, nev=2, check_every=0)
    check(ev, refs, 2)


def test_block_rejects_bad_sizes(ek):
    import edkit_b200._lib as E
    b = ek.TranslationalBasis(L=10, N=5, k=0)
    H = ek.trans_inv_operator(xxz(ek.spin, 1.0), 2, b)
    with pytest.raises(E.EDKError):
        ek.block_lanczos([H], block=12, m=2)
    with pytest.raises(E.EDKError):
        ek.block_lanczos([H], block=8, m=100)
