"""GPU basis tables and index() against the CPU oracle (bit-exact)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def pxp(v):
    return all(v[i] == 0 or v[i + 1] == 0 for i in range(len(v) - 1))


def same_tables(b, o):
    I, R = b.I, b.R
    Io, Ro = o.tables()
    assert I.shape == Io.shape, (I.shape, Io.shape)
    assert np.array_equal(I, Io)
    assert np.array_equal(R, Ro)  # bit-exact norms


def test_tensor_basis(ek, O):
    b = ek.TensorBasis(L=10)
    assert b.size(1) == 1024
    same_tables(b, O.tensor(10))


@pytest.mark.parametrize("L", [6, 9, 12, 16])
def test_projected_N(ek, O, L):
    for N in range(L + 1):
        same_tables(ek.ProjectedBasis(L=L, N=N), O.projected(L, N=N))


def test_projected_predicate(ek, O):
    for L in (6, 10, 14):
        b = ek.ProjectedBasis(L=L, f=pxp)
        same_tables(b, O.projected(L, f=pxp))
    b = ek.ProjectedBasis(L=12, N=6, f=lambda d: d[0] == 0)
    same_tables(b, O.projected(12, N=6, f=lambda d: d[0] == 0))


@pytest.mark.parametrize("L", [8, 10, 12])
def test_translational(ek, O, L):
    for k in range(L):
        for N in (None, L // 2, L // 2 - 1):
            same_tables(ek.TranslationalBasis(L=L, k=k, N=N), O.translational(L, k=k, N=N))
    for k in range(L // 2):
        same_tables(ek.TranslationalBasis(L=L, k=k, a=2), O.translational(L, k=k, a=2))


def test_translational_predicate(ek, O):
    L = 12
    for k in (0, 3):
        same_tables(ek.TranslationalBasis(L=L, k=k, f=pxp), O.translational(L, k=k, f=pxp))


@pytest.mark.parametrize("L", [8, 10, 12])
def test_transparity(ek, O, L):
    for k in (0, L // 2):
        for p in (1, -1):
            for N in (None, L // 2):
                same_tables(ek.TranslationParityBasis(L=L, k=k, p=p, N=N),
                            O.transparity(L, k=k, p=p, N=N))
    same_tables(ek.TranslationParityBasis(L=L, k=0, p=-1, a=2), O.transparity(L, k=0, p=-1, a=2))


def test_transparity_bad_momentum(ek):
    with pytest.raises(ValueError, match="incompatible with parity"):
        ek.TranslationParityBasis(L=8, k=1, p=1)


@pytest.mark.parametrize("L", [6, 8, 10])
def test_abelian_basis(ek, O, L):
    for kw in ({"k": 0}, {"k": 1}, {"k": 0, "p": 1}, {"k": 0, "p": -1}, {"N": L // 2, "k": 0},
               {"N": L // 2, "k": 1, "z": 1}, {"N": L // 2, "k": 0, "p": -1, "z": -1},
               {"N": L // 2, "k": 2, "a": 2}):
        if "a" in kw and L % kw["a"]:
            continue
        same_tables(ek.basis(L=L, **kw), O.basis(L, **kw))


def test_abelian_2d_symmetries(ek, O):
    """abelian_overhaul_tests.jl:315-387: 3x3 lattice, Tx and Ty generators."""
    Lx, Ly = 3, 3
    sites = [(x, y) for y in range(Ly) for x in range(Lx)]
    Tx = [(x + 1) % Lx + Lx * y + 1 for (x, y) in sites]
    Ty = [x + Lx * ((y + 1) % Ly) + 1 for (x, y) in sites]
    for kx in range(Lx):
        for ky in range(Ly):
            for N in (None, 4):
                same_tables(ek.basis(L=9, N=N, symmetries=[(Tx, kx), (Ty, ky)]),
                            O.basis(9, N=N, symmetries=[(Tx, kx), (Ty, ky)]))


def _check_index(b, o, states):
    pos, coeff = b.index_states(states)
    for s, p, c in zip(states, pos, coeff):
        L = b.L
        dgt = [(int(s) >> (L - 1 - q)) & 1 for q in range(L)]
        co, po = o.index(np.array(dgt))
        if co == 0:
            assert p == 0
        else:
            assert p == po
            assert abs(c - co) <= 1e-15 * abs(co), (s, c, co)


def test_index_matches_oracle(ek, O):
    rng = np.random.default_rng(0)
    L = 12
    states = rng.integers(0, 2 ** L, size=400).astype(np.uint64)
    cases = [
        (ek.TensorBasis(L=L), O.tensor(L)),
        (ek.ProjectedBasis(L=L, N=6), O.projected(L, N=6)),
        (ek.ProjectedBasis(L=L, f=pxp), O.projected(L, f=pxp)),
        (ek.TranslationalBasis(L=L, k=0, N=6), O.translational(L, k=0, N=6)),
        (ek.TranslationalBasis(L=L, k=5), O.translational(L, k=5)),
        (ek.TranslationalBasis(L=L, k=3, a=2), O.translational(L, k=3, a=2)),
        (ek.TranslationParityBasis(L=L, k=6, p=-1), O.transparity(L, k=6, p=-1)),
        (ek.TranslationParityBasis(L=L, k=0, p=1, N=6), O.transparity(L, k=0, p=1, N=6)),
        (ek.basis(L=L, N=6, k=1, z=-1), O.basis(L, N=6, k=1, z=-1)),
        (ek.basis(L=L, k=0, p=-1), O.basis(L, k=0, p=-1)),
    ]
    for b, o in cases:
        _check_index(b, o, states)


def test_translational_L28_tables_bit_exact(ek, O):
    """Config-2 sector: L=28, N=14, k=0 (1,432,860 representatives)."""
    b = ek.TranslationalBasis(L=28, N=14, k=0)
    assert b.size(1) == 1432860
    same_tables(b, O.translational(28, k=0, N=14))


def test_sector_dimensions_L32_and_L26(ek):
    """Exact dimensions (Burnside count; sum over k equals C(L, N))."""
    assert ek.TranslationalBasis(L=32, N=16, k=0).size(1) == 18784170
    dims = [ek.TranslationalBasis(L=26, N=13, k=k).size(1) for k in range(26)]
    assert dims[0] == 400024 and dims[13] == 400024
    assert all(d == 400023 for i, d in enumerate(dims) if i not in (0, 13))
    assert sum(dims) == 10400600
