"""Pin the oracle's Schmidt / entropy / DoubleBasis restatements against the
reference's own known answers (test/entanglement_tests.jl,
test/advanced_tests.jl:1-59, test/core_tests.jl entropy values)."""
import math

import numpy as np
import pytest


@pytest.fixture(scope="module")
def OE(O):
    from oracle import entanglement
    return entanglement


def _eigvecs(op):
    H = op.dense()
    H = 0.5 * (H + H.conj().T)
    return np.linalg.eigh(H)[1]


def _colmn_sector(OE, b, H_full):
    """Sector matrix of a dedicated basis built the way colmn! fills it
    (Operator.jl:417-465): column j acts on the representative only, and each
    reached state t lands in row index(b, t) with weight coeff(t) / R[j]."""
    D, L = b.dim, b.L
    Hs = np.zeros((D, D), dtype=np.complex128)
    idx = [OE.index_state(b, t) for t in range(2 ** L)]
    for j in range(D):
        col = H_full[:, b.I[j] - 1]
        for t in np.nonzero(col)[0]:
            c, pos = idx[t]
            if c != 0:
                Hs[pos - 1, j] += col[t] * c / b.R[j]
    return Hs


def _spectrum(OE, b, vecs, cut):
    return sorted(OE.ent_S(vecs[:, i], cut, b) for i in range(vecs.shape[1]))


def test_entropy_helpers(OE):
    """Schmidt.jl:101-139: Shannon with the cutoff break, Renyi-0 count, Renyi-alpha."""
    p = np.array([0.5, 0.25, 0.25, 0.0])
    assert OE.entropy(p) == pytest.approx(1.5 * math.log(2))
    assert OE.entropy(p, alpha=0) == 3
    assert OE.entropy(p, alpha=2) == pytest.approx(-math.log(0.375))
    # product state: zero entropy; Bell pair: log 2
    b = pytest.importorskip("oracle").tensor(2)
    assert OE.ent_S(np.array([1.0, 0, 0, 0]), [1], b) == pytest.approx(0.0, abs=1e-15)
    assert OE.ent_S(np.array([1.0, 0, 0, 1]) / math.sqrt(2), [1], b) == pytest.approx(math.log(2))


def test_momentum_resolves_tensor_entropies(O, OE):
    """entanglement_tests.jl:7-20 (a = 1) and :22-35 (a = 2)."""
    L = 6
    rng = np.random.default_rng(7)
    m = rng.standard_normal((4, 4)) + 1j * rng.standard_normal((4, 4))
    mat = m + m.conj().T
    cut = [1, 2, 3]
    B0 = O.tensor(L)
    S0 = _spectrum(OE, B0, _eigvecs(O.trans_inv_operator(mat, 2, B0)), cut)
    for a in (1, 2):
        Ss = []
        for k in range(L // a):
            B = O.translational(L, k=k, a=a)
            Ss += _spectrum(OE, B, _eigvecs(O.trans_inv_operator(mat, 2, B)), cut)
        assert np.allclose(sorted(Ss), S0, atol=1e-9)


def test_parity_splits_momentum_sectors(O, OE):
    """entanglement_tests.jl:37-60: TranslationParityBasis(+-1) = TranslationalBasis
    at k = 0, pi for three bipartitions."""
    L, h = 6, 0.37
    mat = O.spin((1.0, "xx"), (0.8, "yy"), (0.4, "zz"))
    fld = O.spin((h, "z"))
    for k in (0, L // 2):
        def vecs(B):
            H = O.trans_inv_operator(mat, 2, B).dense() + O.trans_inv_operator(fld, 1, B).dense()
            return np.linalg.eigh(0.5 * (H + H.conj().T))[1]
        Bt = O.translational(L, k=k)
        Bp, Bm = O.transparity(L, k=k, p=1), O.transparity(L, k=k, p=-1)
        vt, vp, vm = vecs(Bt), vecs(Bp), vecs(Bm)
        for inds in ([1, 2, 3], [1, 3], [2, 4, 6]):
            St = _spectrum(OE, Bt, vt, inds)
            Spm = sorted(_spectrum(OE, Bp, vp, inds) + _spectrum(OE, Bm, vm, inds))
            assert np.allclose(St, Spm, atol=1e-9)


def test_spin_flip_splits_momentum_sectors(O, OE):
    """entanglement_tests.jl:62-79: TranslationFlipBasis(+-1) = TranslationalBasis.
    The XXZ chain conserves Sz, so levels of opposite magnetisation are
    degenerate inside a momentum sector and their eigenvectors (hence their
    entropies) are arbitrary; only non-degenerate levels are compared."""
    L = 6
    mat = O.spin((1.0, "xx"), (0.8, "yy"), (0.3, "zz"))
    Hf = O.trans_inv_operator(mat, 2, O.tensor(L)).dense()

    def levels(b, H):
        w, v = np.linalg.eigh(0.5 * (H + H.conj().T))
        return w, v
    ncmp = 0
    for k in range(L):
        Bt = O.translational(L, k=k)
        wt, vt = levels(Bt, O.trans_inv_operator(mat, 2, Bt).dense())
        parts = []
        for p in (1, -1):
            Bf = O.transflip_basis(L, k=k, p=p)
            if Bf.dim:
                parts.append((Bf,) + levels(Bf, _colmn_sector(OE, Bf, Hf)))
        for n in range(len(wt)):
            if np.min(np.abs(np.delete(wt, n) - wt[n]), initial=1.0) < 1e-6:
                continue
            for inds in ([1, 2, 3], [1, 2], [2, 4, 6]):
                St = OE.ent_S(vt[:, n], inds, Bt)
                hits = [OE.ent_S(v[:, j], inds, B) for B, w, v in parts
                        for j in range(len(w)) if abs(w[j] - wt[n]) < 1e-8]
                assert len(hits) == 1 and hits[0] == pytest.approx(St, abs=1e-9)
                ncmp += 1
    assert ncmp > 20


def test_abelian_matches_dedicated(O, OE):
    """entanglement_tests.jl:81-112: basis(...) entropies = dedicated types'."""
    L, N = 6, 3
    mat = O.spin((1.0, "xx"), (0.7, "yy"), (0.2, "zz"))
    Hf = O.trans_inv_operator(mat, 2, O.tensor(L)).dense()
    cases = [
        (O.basis(L, k=1), O.translational(L, k=1)),
        (O.basis(L, p=1), O.parity_basis(L, 1)),
        (O.basis(L, z=1), O.flip_basis(L, 1)),
        (O.basis(L, N=N, k=1), O.translational(L, k=1, N=N)),
        (O.basis(L, N=N, p=1), O.parity_basis(L, 1, N=N)),
        (O.basis(L, k=0, p=1), O.transparity(L, k=0, p=1)),
        (O.basis(L, k=1, z=1), O.transflip_basis(L, k=1, p=1)),
        (O.basis(L, p=1, z=1), O.parityflip_basis(L, 1, 1)),
        (O.basis(L, N=N, k=0, p=1, z=1), O.basis(L, N=N, k=0, p=1, z=1)),
    ]
    cut = [1, 2, 3]

    def nondegenerate(B, H):  # exactly degenerate levels have arbitrary vectors
        w, v = np.linalg.eigh(0.5 * (H + H.conj().T))
        keep = [n for n in range(len(w))
                if np.min(np.abs(np.delete(w, n) - w[n]), initial=1.0) > 1e-6]
        return w[keep], [OE.ent_S(v[:, n], cut, B) for n in keep]
    for Ba, Bb in cases:
        wa, Sa = nondegenerate(Ba, O.trans_inv_operator(mat, 2, Ba).dense())
        Hb = (O.trans_inv_operator(mat, 2, Bb).dense() if hasattr(Bb, "h")
              else _colmn_sector(OE, Bb, Hf))
        wb, Sb = nondegenerate(Bb, Hb)
        assert len(Sa) > 0 and np.allclose(wa, wb) and np.allclose(Sa, Sb, atol=1e-9)


def test_schmidt_norm_and_dimensions(O, OE):
    """A normalised sector vector gives a Schmidt matrix of unit Frobenius norm
    and shape 2^|A| x 2^(L-|A|) for every basis type (Schmidt.jl:39-57)."""
    L = 6
    rng = np.random.default_rng(3)
    bases = [O.tensor(L), O.projected(L, N=3), O.translational(L, k=2),
             O.translational(L, k=1, a=2), O.transparity(L, k=3, p=-1),
             O.basis(L, k=1, p=None, z=1), O.parity_basis(L, -1), O.flip_basis(L, 1),
             O.parityflip_basis(L, 1, -1), O.transflip_basis(L, k=2, p=1)]
    for b in bases:
        v = rng.standard_normal(b.dim) + 1j * rng.standard_normal(b.dim)
        v /= np.linalg.norm(v)
        for cut in ([1, 2], [5, 1, 3]):
            M = OE.schmidt(v, cut, b)
            assert M.shape == (2 ** len(cut), 2 ** (L - len(cut)))
            assert np.linalg.norm(M) == pytest.approx(1.0, abs=1e-12)


def test_symmetrizer_known_answers(O, OE):
    """advanced_tests.jl:1-42: the full-space symmetrizer is the identity, and
    the DoubleBasis action equals symmetrizer * v for every basis pair."""
    L, N = 4, 2
    Bf = O.tensor(L)
    assert np.allclose(OE.symmetrizer(Bf, Bf), np.eye(2 ** L))
    rng = np.random.default_rng(11)
    bases = [Bf, O.projected(L, N=N), O.basis(L, N=N, k=0, p=1), O.parity_basis(L, 1),
             O.flip_basis(L, 1, N=N), O.parityflip_basis(L, 1, 1, N=N),
             O.translational(L, k=0, N=N), O.transparity(L, k=0, p=1, N=N),
             O.transflip_basis(L, k=0, p=1, N=N)]
    for Bt in bases:
        for Bs in bases:
            v = rng.standard_normal(Bs.dim) + 1j * rng.standard_normal(Bs.dim)
            assert np.allclose(OE.double_basis_apply(Bt, Bs, v), OE.symmetrizer(Bt, Bs) @ v,
                               atol=1e-10, rtol=1e-10)


def test_product_entropy_helper_matches_oracle(ek, OE):
    """entropy(s; α, cutoff) of the Python mirror (host arithmetic, no device)
    against the oracle's restatement of Schmidt.jl:101-139."""
    rng = np.random.default_rng(21)
    for n in (1, 5, 64):
        p = np.sort(rng.random(n))[::-1]
        p /= p.sum()
        p[-1:] = 1e-25 if n > 1 else p[-1:]
        for alpha in (0, 0.5, 1, 2):
            assert ek.entropy(p, alpha=alpha) == pytest.approx(OE.entropy(p, alpha=alpha),
                                                               rel=1e-14, abs=1e-15), (n, alpha)
        assert ek.entropy(p, cutoff=0.5) == pytest.approx(OE.entropy(p, cutoff=0.5), abs=1e-15)
