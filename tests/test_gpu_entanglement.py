"""Eigenvector post-processing on the GPU against the oracle's restatements of
src/Schmidt.jl and src/LinearMap.jl: Schmidt matrices for every basis type,
entanglement spectra and entropies, the DoubleBasis map and the symmetrizer.

Tolerances: the Schmidt matrix and the DoubleBasis map are FP64 sums of the
same terms as the reference (1e-12 relative); singular values come from the
Gram matrix, so squared Schmidt values agree to 1e-12 absolute for unit
vectors, entropies to 1e-9."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def OE(O):
    from oracle import entanglement
    return entanglement


def pairs(ek, O, L):
    """(name, product basis, oracle basis) for every basis type."""
    N = L // 2
    out = [
        ("tensor", ek.TensorBasis(L=L), O.tensor(L)),
        ("projected", ek.ProjectedBasis(L=L, N=N), O.projected(L, N=N)),
        ("projected N-1", ek.ProjectedBasis(L=L, N=N - 1), O.projected(L, N=N - 1)),
        ("trans k=0", ek.TranslationalBasis(L=L, k=0), O.translational(L, k=0)),
        ("trans k=1 N", ek.TranslationalBasis(L=L, k=1, N=N), O.translational(L, k=1, N=N)),
        ("trans k=L/2", ek.TranslationalBasis(L=L, k=L // 2), O.translational(L, k=L // 2)),
        ("trans a=2 k=1", ek.TranslationalBasis(L=L, k=1, a=2), O.translational(L, k=1, a=2)),
        ("transpar k=0 p=-1", ek.TranslationParityBasis(L=L, k=0, p=-1),
         O.transparity(L, k=0, p=-1)),
        ("transpar k=pi p=1 N", ek.TranslationParityBasis(L=L, k=L // 2, p=1, N=N),
         O.transparity(L, k=L // 2, p=1, N=N)),
        ("abelian k=1 z", ek.basis(L=L, k=1, z=1), O.basis(L, k=1, z=1)),
        ("abelian N k=0 p", ek.basis(L=L, N=N, k=0, p=-1), O.basis(L, N=N, k=0, p=-1)),
        ("abelian N k=0 p z", ek.basis(L=L, N=N, k=0, p=1, z=-1), O.basis(L, N=N, k=0, p=1, z=-1)),
        ("parity", ek.ParityBasis(L=L, p=-1), O.parity_basis(L, -1)),
        ("flip N", ek.FlipBasis(L=L, p=1, N=N), O.flip_basis(L, 1, N=N)),
        ("parityflip", ek.ParityFlipBasis(L=L, p=1, z=-1), O.parityflip_basis(L, 1, -1)),
        ("transflip k=1", ek.TranslationFlipBasis(L=L, k=1, p=1), O.transflip_basis(L, 1, 1)),
        ("transflip a=2 k=1", ek.TranslationFlipBasis(L=L, k=1, p=-1, a=2),
         O.transflip_basis(L, 1, -1, a=2)),
    ]
    return [c for c in out if c[2].dim > 0]


CUTS = ([1, 2, 3, 4], [5, 1, 3], [2], [1, 2, 3, 4, 5, 6, 7])


def _vec(rng, D, cplx):
    v = rng.standard_normal(D) + (1j * rng.standard_normal(D) if cplx else 0)
    return v / np.linalg.norm(v)


@pytest.mark.parametrize("L", [8, 10])
def test_schmidt_matrix_every_basis(ek, O, OE, L):
    rng = np.random.default_rng(L)
    for name, b, o in pairs(ek, O, L):
        for cplx in (False, True):
            v = _vec(rng, b.size(1), cplx)
            for cut in CUTS:
                M = ek.schmidt(v, cut, b)
                R = OE.schmidt(v, cut, o)
                assert M.shape == R.shape, name
                assert np.abs(M - R).max() <= 1e-12 * max(np.abs(R).max(), 1e-300), (name, cut)


@pytest.mark.parametrize("L", [8, 10])
def test_ent_spec_and_entropies(ek, O, OE, L):
    rng = np.random.default_rng(100 + L)
    for name, b, o in pairs(ek, O, L):
        v = _vec(rng, b.size(1), True)
        for cut in CUTS[:3]:
            s = ek.ent_spec(v, cut, b)
            r = OE.ent_spec(v, cut, o)
            assert len(s) == len(r), name
            assert np.abs(s ** 2 - r ** 2).max() <= 1e-12, (name, cut)
            for alpha in (1, 2, 0.5):
                assert ek.ent_S(v, cut, b, alpha=alpha) == pytest.approx(
                    OE.ent_S(v, cut, o, alpha=alpha), abs=1e-9), (name, cut, alpha)


def test_known_entropies(ek):
    """Product state: S = 0 and rank 1; Bell pairs across the cut: S = n log 2."""
    L = 6
    b = ek.TensorBasis(L=L)
    v = np.zeros(2 ** L)
    v[5] = 1.0
    assert ek.ent_S(v, [1, 2, 3], b) == pytest.approx(0.0, abs=1e-14)
    assert ek.ent_S(v, [1, 2, 3], b, alpha=0) == 1
    # (|00> + |11>)/sqrt 2 on sites (1,4), (2,5), (3,6)
    bell = np.zeros(2 ** L)
    for x in range(8):
        bits = [(x >> 2) & 1, (x >> 1) & 1, x & 1]
        dgt = bits + bits
        bell[int("".join(map(str, dgt)), 2)] = 1.0
    bell /= np.linalg.norm(bell)
    assert ek.ent_S(bell, [1, 2, 3], b) == pytest.approx(3 * math.log(2), abs=1e-12)
    assert ek.ent_S(bell, [1, 2, 3], L) == pytest.approx(3 * math.log(2), abs=1e-12)
    assert ek.ent_S(bell, [1, 2, 3], b, alpha=0) == 8
    assert ek.ent_S(bell, [1, 5], b) == pytest.approx(2 * math.log(2), abs=1e-12)


def test_momentum_sectors_resolve_tensor_entropies(ek):
    """entanglement_tests.jl:7-20 on the device path: the entropies of all
    momentum sectors' eigenvectors equal those of the full space."""
    L = 6
    rng = np.random.default_rng(7)
    m = rng.standard_normal((4, 4)) + 1j * rng.standard_normal((4, 4))
    mat = m + m.conj().T

    def spec(B):
        H = ek.trans_inv_operator(mat, 2, B).todense()
        vecs = np.linalg.eigh(0.5 * (H + H.conj().T))[1]
        return [ek.ent_S(vecs[:, i], [1, 2, 3], B) for i in range(vecs.shape[1])]
    S0 = sorted(spec(ek.TensorBasis(L=L)))
    Ss = sorted(sum((spec(ek.TranslationalBasis(L=L, k=k)) for k in range(L)), []))
    assert np.allclose(Ss, S0, atol=1e-9)


def test_schmidt_device_tensors(ek):
    torch = pytest.importorskip("torch")
    L = 10
    rng = np.random.default_rng(5)
    for b in (ek.TranslationalBasis(L=L, k=3, N=5), ek.ParityFlipBasis(L=L, p=1, z=1)):
        v = _vec(rng, b.size(1), True)
        M_host = ek.schmidt(v, [1, 2, 3, 4, 5], b)
        M_dev = ek.schmidt(torch.from_numpy(v).cuda(), [1, 2, 3, 4, 5], b)
        assert M_dev.is_cuda
        assert np.array_equal(M_dev.cpu().numpy(), M_host)


@pytest.mark.parametrize("L", [6, 8])
def test_double_basis_map(ek, O, OE, L):
    rng = np.random.default_rng(L + 1)
    cs = pairs(ek, O, L)
    pick = [cs[i] for i in (0, 1, 3, 4, 7, 9, 12, 14, 15)]
    for n1, b1, o1 in pick:
        for n2, b2, o2 in pick:
            v = _vec(rng, b2.size(1), True)
            T = ek.DoubleBasis(b1, b2)
            out = T(v)
            ref = OE.double_basis_apply(o1, o2, v)
            assert np.abs(out - ref).max() <= 1e-12 * max(np.abs(ref).max(), 1.0), (n1, n2)


def test_symmetrizer(ek, O, OE):
    """advanced_tests.jl:1-42: the full-space symmetrizer is the identity; the
    DoubleBasis action equals symmetrizer * v; entries match the oracle."""
    L = 6
    Bf = ek.TensorBasis(L=L)
    assert np.allclose(ek.symmetrizer(ek.DoubleBasis(Bf, Bf)), np.eye(2 ** L), atol=1e-15)
    rng = np.random.default_rng(9)
    cs = pairs(ek, O, L)
    for n1, b1, o1 in cs[::3]:
        for n2, b2, o2 in cs[1::3]:
            T = ek.DoubleBasis(b1, b2)
            S = ek.symmetrizer(T)
            assert np.abs(S - OE.symmetrizer(o1, o2)).max() <= 1e-12, (n1, n2)
            v = _vec(rng, b2.size(1), True)
            assert np.allclose(T(v), S @ v, atol=1e-10, rtol=1e-10), (n1, n2)


def test_argument_errors(ek):
    with pytest.raises(ValueError, match="same length"):
        ek.DoubleBasis(ek.TensorBasis(L=3), ek.TensorBasis(L=4))
    b = ek.TensorBasis(L=4)
    with pytest.raises(ValueError, match="Expected a vector of length"):
        ek.DoubleBasis(b, b)(np.zeros(3))
    with pytest.raises(ek.EDKError, match="repeated site"):
        ek.schmidt(np.zeros(16), [1, 1], b)
    with pytest.raises(ek.EDKError, match="out of range"):
        ek.schmidt(np.zeros(16), [5], b)
