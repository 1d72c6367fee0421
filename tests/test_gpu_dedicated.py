"""The reference's dedicated symmetry bases (ParityBasis, FlipBasis,
ParityFlipBasis, TranslationFlipBasis) on the GPU: tables (I, R) bit-exact and
index() identical to the oracle's restatement of each reference file, and the
sector spectra of XXZ chains adding up to the full spectrum."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

XXZ = ((1.0, "xx"), (1.0, "yy"), (0.7, "zz"))


def pxp(d):
    return all(not (d[i] == 1 and d[(i + 1) % len(d)] == 1) for i in range(len(d)))


def cases(ek, O, L):
    out = []
    for p in (1, -1):
        out.append((f"parity p={p}", ek.ParityBasis(L=L, p=p), O.parity_basis(L, p)))
        out.append((f"parity p={p} N", ek.ParityBasis(L=L, p=p, N=L // 2 - 1),
                    O.parity_basis(L, p, N=L // 2 - 1)))
        out.append((f"parity p={p} f", ek.ParityBasis(L=L, p=p, f=pxp), O.parity_basis(L, p, f=pxp)))
        out.append((f"flip p={p}", ek.FlipBasis(L=L, p=p), O.flip_basis(L, p)))
        out.append((f"flip p={p} N", ek.FlipBasis(L=L, p=p, N=L // 2), O.flip_basis(L, p, N=L // 2)))
        for z in (1, -1):
            out.append((f"parityflip {p} {z}", ek.ParityFlipBasis(L=L, p=p, z=z),
                        O.parityflip_basis(L, p, z)))
            out.append((f"parityflip {p} {z} N", ek.ParityFlipBasis(L=L, p=p, z=z, N=L // 2),
                        O.parityflip_basis(L, p, z, N=L // 2)))
        for k in (0, 1, L // 2, L - 1):
            out.append((f"transflip k={k} p={p}", ek.TranslationFlipBasis(L=L, k=k, p=p),
                        O.transflip_basis(L, k, p)))
        out.append((f"transflip k=1 p={p} N", ek.TranslationFlipBasis(L=L, k=1, p=p, N=L // 2),
                    O.transflip_basis(L, 1, p, N=L // 2)))
        out.append((f"transflip a=2 k=1 p={p}", ek.TranslationFlipBasis(L=L, k=1, p=p, a=2),
                    O.transflip_basis(L, 1, p, a=2)))
    return out


@pytest.mark.parametrize("L", [8, 10])
def test_tables_and_index(ek, O, L):
    states = np.arange(2 ** L, dtype=np.uint64)
    for name, b, o in cases(ek, O, L):
        assert b.size(1) == o.dim, name
        if o.dim == 0:
            continue
        assert np.array_equal(b.I, np.array(o.I)), name
        assert np.array_equal(b.R, np.array(o.R)), name
        pos, coeff = b.index_states(states)
        for s in range(2 ** L):
            co, po = o.index_state(s)
            if co == 0:
                assert pos[s] == 0, (name, s)
            else:
                assert pos[s] == po, (name, s)
                assert abs(coeff[s] - co) <= 1e-14 * abs(co), (name, s, coeff[s], co)


def test_sector_spectra_add_up(ek, O):
    """XXZ ring, L = 10: the union of every sector's spectrum is the full
    spectrum, for each dedicated basis family."""
    L = 10
    inds = [[i, i % L + 1] for i in range(1, L + 1)]
    Hfull = O.operator([O.spin(*XXZ)] * L, inds, O.tensor(L)).dense()
    full = np.sort(np.linalg.eigvalsh(Hfull))
    families = {
        "parity": [ek.ParityBasis(L=L, p=p) for p in (1, -1)],
        "flip": [ek.FlipBasis(L=L, p=p) for p in (1, -1)],
        "parityflip": [ek.ParityFlipBasis(L=L, p=p, z=z) for p in (1, -1) for z in (1, -1)],
        "transflip": [ek.TranslationFlipBasis(L=L, k=k, p=p) for k in range(L) for p in (1, -1)],
    }
    for name, bases in families.items():
        ev = []
        for b in bases:
            if b.size(1) == 0:
                continue
            H = ek.operator([ek.spin(*XXZ)] * L, inds, b)
            M = H.todense()
            assert np.allclose(M, M.conj().T, atol=1e-12), name
            ev.extend(np.linalg.eigvalsh(M))
        assert np.allclose(np.sort(ev), full, atol=1e-10), name


def test_lanczos_on_dedicated_sectors(ek, O):
    """L = 16, N = 8: the lowest E0 over the four ParityFlip sectors equals
    the E0 of the whole fixed-N sector."""
    L = 16
    inds = [[i, i % L + 1] for i in range(1, L + 1)]
    es = []
    for p in (1, -1):
        for z in (1, -1):
            b = ek.ParityFlipBasis(L=L, p=p, z=z, N=8)
            H = ek.operator([ek.spin(*XXZ)] * L, inds, b)
            e, _ = ek.lanczos_e0(H, np.random.default_rng(0).standard_normal(b.size(1)), m=150)
            es.append(e[0])
    Ho = O.operator([O.spin(*XXZ)] * L, inds, O.projected(L, N=8))
    from scipy.sparse.linalg import LinearOperator, eigsh
    op = LinearOperator((Ho.b.dim, Ho.b.dim), matvec=lambda v: Ho.mul(v).real, dtype=np.float64)
    e_all = eigsh(op, k=1, which="SA", tol=1e-14)[0][0]
    assert min(es) >= e_all - 1e-10 * abs(e_all)
    assert abs(min(es) - e_all) < 1e-10 * abs(e_all)


def test_reference_ising_spin_flip_pattern(ek, O):
    """EigenvalueTest.jl:562-575: zz + 0.3 x on TranslationalBasis(k) equals
    the union of TranslationFlipBasis(k, p = +-1) spectra, L = 4..10 — a
    one-site off-diagonal term, so the generic kernel on the symmetry path."""
    for L in range(4, 11, 2):
        for k in range(L):
            ba = ek.TranslationalBasis(L=L, k=k)
            va = np.linalg.eigvalsh((ek.trans_inv_operator(ek.spin((1.0, "zz")), 2, ba) +
                                     ek.trans_inv_operator(ek.spin((0.3, "x")), 1, ba)).todense())
            ve = []
            for p in (1, -1):
                b = ek.TranslationFlipBasis(L=L, k=k, p=p)
                if b.size(1) == 0:
                    continue
                H = ek.trans_inv_operator(ek.spin((1.0, "zz")), 2, b) + \
                    ek.trans_inv_operator(ek.spin((0.3, "x")), 1, b)
                ve.extend(np.linalg.eigvalsh(H.todense()))
            assert np.allclose(np.sort(ve), va, atol=1e-12), (L, k)


def test_reference_xy_parity_pattern(ek, O):
    """EigenvalueTest.jl:253-265: XY on ProjectedBasis(N) equals the union of
    ParityBasis(N, p = +-1) spectra, L = 2..8, every N."""
    for L in range(2, 9):
        for n in range(L + 1):
            ba = ek.ProjectedBasis(L=L, N=n)
            va = np.linalg.eigvalsh(ek.trans_inv_operator(ek.spin((1.0, "xx"), (1.0, "yy")), 2, ba).todense())
            ve = []
            for p in (1, -1):
                b = ek.ParityBasis(L=L, N=n, p=p)
                if b.size(1):
                    ve.extend(np.linalg.eigvalsh(
                        ek.trans_inv_operator(ek.spin((1.0, "xx"), (1.0, "yy")), 2, b).todense()))
            assert np.allclose(np.sort(ve), va, atol=1e-12), (L, n)
