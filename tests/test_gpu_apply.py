"""GPU matrix-free H*x against the oracle's column-scatter mul (Operator.jl).

Tolerances: FP64 paths <= 1e-12 relative (2-norm); FP32 storage paths
<= 2e-6 relative."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

XXZ = ((1.0, "xx"), (1.0, "yy"), (1.5, "zz"))


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300)


def pairs(ek, O):
    L = 10
    return [
        ("tensor", ek.TensorBasis(L=L), O.tensor(L)),
        ("proj_rank", ek.ProjectedBasis(L=L, N=5), O.projected(L, N=5)),
        ("proj_hash", ek.ProjectedBasis(L=L, N=5, f=lambda d: d[0] == 0 or d[1] == 0),
         O.projected(L, N=5, f=lambda d: d[0] == 0 or d[1] == 0)),
        ("trans0", ek.TranslationalBasis(L=L, k=0, N=5), O.translational(L, k=0, N=5)),
        ("trans_k", ek.TranslationalBasis(L=L, k=3, N=5), O.translational(L, k=3, N=5)),
        ("trans_pi", ek.TranslationalBasis(L=L, k=5), O.translational(L, k=5)),
        ("trans_a2", ek.TranslationalBasis(L=L, k=1, a=2), O.translational(L, k=1, a=2)),
        ("transpar", ek.TranslationParityBasis(L=L, k=0, p=-1, N=5),
         O.transparity(L, k=0, p=-1, N=5)),
        ("transpar_pi", ek.TranslationParityBasis(L=L, k=5, p=1), O.transparity(L, k=5, p=1)),
        ("abelian", ek.basis(L=L, N=5, k=2, z=1), O.basis(L, N=5, k=2, z=1)),
        ("abelian_kp", ek.basis(L=L, k=0, p=-1), O.basis(L, k=0, p=-1)),
    ]


@pytest.fixture(scope="module")
def cases(ek, O):
    return pairs(ek, O)


def test_bond_operator_all_bases(ek, O, cases):
    rng = np.random.default_rng(0)
    for name, b, o in cases:
        H = ek.trans_inv_operator(ek.spin(*XXZ), 2, b)
        Ho = O.trans_inv_operator(O.spin(*XXZ), 2, o)
        assert H.hermitian_gather, name
        D = b.size(1)
        x = rng.standard_normal(D) + 1j * rng.standard_normal(D)
        ref = Ho.mul(x)
        assert rel(H * x, ref) < 1e-12, name
        y64 = H * x.astype(np.complex64)
        assert rel(y64, ref) < 2e-6, name
        if not H.is_complex:
            xr = x.real.copy()
            refr = Ho.mul(xr)
            assert np.max(np.abs(refr.imag)) < 1e-12
            assert rel(H * xr, refr.real) < 1e-12, name
            assert rel(H * xr.astype(np.float32), refr.real) < 2e-6, name


def test_generic_terms_and_fields(ek, O, cases):
    """Mixed term shapes: 1-site fields, 3-site terms, complex couplings."""
    rng = np.random.default_rng(1)
    for name, b, o in cases:
        L = b.L
        if name.startswith(("trans", "abelian")):
            mats = [ek.spin("zxz") * 0.3, ek.spin((1.0, "+-"), (1.0, "-+")) + 0.2 * ek.spin("zz")]
            H = ek.trans_inv_operator(mats[0], 3, b) + ek.trans_inv_operator(mats[1], 2, b)
            Ho = O.trans_inv_operator(O.spin("zxz") * 0.3, 3, o)
            Ho2 = O.trans_inv_operator(O.spin((1.0, "+-"), (1.0, "-+")) + 0.2 * O.spin("zz"), 2, o)
            x = rng.standard_normal(b.size(1)) + 1j * rng.standard_normal(b.size(1))
            ref = Ho.mul(x) + Ho2.mul(x)
        else:
            h = rng.uniform(-3, 3, L)
            mats = [ek.spin((1.0, "xx"), (1.0, "yy"), (1.0, "zz"))] * (L - 1) + \
                   [hi * ek.spin("z") for hi in h] + [0.7 * ek.spin("xy")]
            inds = [[i, i + 1] for i in range(1, L)] + [[i] for i in range(1, L + 1)] + [[3, 7]]
            H = ek.operator(mats, inds, b)
            omats = [O.spin((1.0, "xx"), (1.0, "yy"), (1.0, "zz"))] * (L - 1) + \
                    [hi * O.spin("z") for hi in h] + [0.7 * O.spin("xy")]
            Ho = O.operator(omats, inds, o)
            x = rng.standard_normal(b.size(1)) + 1j * rng.standard_normal(b.size(1))
            ref = Ho.mul(x)
        assert rel(H * x, ref) < 1e-12, name


def test_non_hermitian_uses_scatter(ek, O, cases):
    """A non-Hermitian term (S+ on one site pair) runs the column-scatter form."""
    rng = np.random.default_rng(2)
    for name, b, o in cases:
        m = ek.spin("+z") + 0.5 * ek.spin("zz")
        H = ek.trans_inv_operator(m, 2, b)
        Ho = O.trans_inv_operator(O.spin("+z") + 0.5 * O.spin("zz"), 2, o)
        assert not H.hermitian_gather
        x = rng.standard_normal(b.size(1)) + 1j * rng.standard_normal(b.size(1))
        assert rel(H * x, Ho.mul(x)) < 1e-12, name


def test_non_invariant_operator_uses_scatter(ek, O):
    """A field on one site is not translation invariant: scatter form, same
    matrix as the reference builds."""
    L = 8
    b, o = ek.TranslationalBasis(L=L, k=2), O.translational(L, k=2)
    H = ek.operator([ek.spin("x")], [[3]], b)
    Ho = O.operator([O.spin("x")], [[3]], o)
    assert not H.hermitian_gather
    x = np.random.default_rng(3).standard_normal(b.size(1)) + 0j
    assert rel(H * x, Ho.mul(x)) < 1e-12


def test_mul_bang_accumulates(ek, O):
    """mul!(y, H, x) adds into y (Operator.jl:309-315)."""
    L = 10
    b, o = ek.ProjectedBasis(L=L, N=5), O.projected(L, N=5)
    H = ek.trans_inv_operator(ek.spin(*XXZ), 2, b)
    Ho = O.trans_inv_operator(O.spin(*XXZ), 2, o)
    rng = np.random.default_rng(4)
    x = rng.standard_normal(b.size(1))
    y0 = rng.standard_normal(b.size(1))
    y = y0.copy()
    ek.mul_(y, H, x)
    assert rel(y, y0 + Ho.mul(x).real) < 1e-12
    assert rel(ek.mul(H, x), Ho.mul(x).real) < 1e-12


def test_block_rhs(ek, O):
    """H * M for an nvec-column block (Operator.jl:382-394)."""
    L = 10
    b, o = ek.TranslationalBasis(L=L, k=1, N=5), O.translational(L, k=1, N=5)
    H = ek.trans_inv_operator(ek.spin(*XXZ), 2, b)
    Ho = O.trans_inv_operator(O.spin(*XXZ), 2, o)
    rng = np.random.default_rng(5)
    X = np.asfortranarray(rng.standard_normal((b.size(1), 7)) + 1j * rng.standard_normal((b.size(1), 7)))
    assert rel(H * X, Ho.mul(X)) < 1e-12


def test_dense_matches_oracle(ek, O):
    L = 8
    b, o = ek.TranslationalBasis(L=L, k=3), O.translational(L, k=3)
    H = ek.trans_inv_operator(ek.spin(*XXZ), 2, b)
    Ho = O.trans_inv_operator(O.spin(*XXZ), 2, o)
    assert np.allclose(H.todense(), Ho.dense(), atol=1e-13)


def test_device_pointer_path(ek, O):
    torch = pytest.importorskip("torch")
    L = 12
    b, o = ek.TranslationalBasis(L=L, k=0, N=6), O.translational(L, k=0, N=6)
    H = ek.trans_inv_operator(ek.spin(*XXZ), 2, b)
    Ho = O.trans_inv_operator(O.spin(*XXZ), 2, o)
    x = torch.randn(b.size(1), dtype=torch.float64, device="cuda")
    y = H * x
    assert y.is_cuda
    ref = Ho.mul(x.cpu().numpy()).real
    assert rel(y.cpu().numpy(), ref) < 1e-12


def test_deterministic_gather(ek):
    """The row-gather form has no atomics: two runs are bit-identical."""
    b = ek.TranslationalBasis(L=20, k=0, N=10)
    H = ek.trans_inv_operator(ek.spin(*XXZ), 2, b)
    x = np.random.default_rng(6).standard_normal(b.size(1))
    assert np.array_equal(H * x, H * x)


def test_config2_matvec_properties(ek, O):
    """L=28 N=14 k=0 (D=1,432,860): sampled rows vs the oracle, Hermiticity
    <u,Hv> = <Hu,v>, and linearity."""
    b = ek.TranslationalBasis(L=28, N=14, k=0)
    H = ek.trans_inv_operator(ek.spin((1.0, "xx"), (1.0, "yy"), (1.0, "zz")), 2, b)
    rng = np.random.default_rng(7)
    D = b.size(1)
    u, v = rng.standard_normal(D), rng.standard_normal(D)
    Hu, Hv = H * u, H * v
    assert abs(u @ Hv - Hu @ v) <= 1e-12 * abs(u @ Hv)
    assert rel(H * (2.0 * u - 3.0 * v), 2.0 * Hu - 3.0 * Hv) < 1e-13
    o = O.translational(28, k=0, N=14)
    Ho = O.trans_inv_operator(O.spin((1.0, "xx"), (1.0, "yy"), (1.0, "zz")), 2, o)
    assert rel(Hv, Ho.mul(v).real) < 1e-12


def test_fast_path_matches_generic_kernel(ek, O, monkeypatch):
    """The flip-flop bond-family kernel and the generic kernel agree with each
    other and with the oracle on every lookup kind."""
    rng = np.random.default_rng(8)
    L = 12
    cases = [
        (ek.TensorBasis(L=L), O.tensor(L)),
        (ek.ProjectedBasis(L=L, N=6), O.projected(L, N=6)),
        (ek.ProjectedBasis(L=L, N=6, f=lambda d: d[0] == 0), O.projected(L, N=6, f=lambda d: d[0] == 0)),
        (ek.TranslationalBasis(L=L, k=0, N=6), O.translational(L, k=0, N=6)),
        (ek.TranslationalBasis(L=L, k=5, N=6), O.translational(L, k=5, N=6)),
        (ek.TranslationalBasis(L=L, k=2, a=2), O.translational(L, k=2, a=2)),
        (ek.TranslationParityBasis(L=L, k=6, p=-1, N=6), O.transparity(L, k=6, p=-1, N=6)),
    ]
    j2 = ek.spin((0.5, "xx"), (0.5, "yy"), (0.5, "zz"))
    for b, o in cases:
        H1 = ek.trans_inv_operator(ek.spin(*XXZ), 2, b) + ek.trans_inv_operator(j2, [1, 3], b)
        monkeypatch.setenv("EDK_DISABLE_FAST", "1")
        H2 = ek.trans_inv_operator(ek.spin(*XXZ), 2, b) + ek.trans_inv_operator(j2, [1, 3], b)
        monkeypatch.delenv("EDK_DISABLE_FAST")
        Ho = O.trans_inv_operator(O.spin(*XXZ), 2, o)
        Ho2 = O.trans_inv_operator(O.spin((0.5, "xx"), (0.5, "yy"), (0.5, "zz")), [1, 3], o)
        x = rng.standard_normal(b.size(1)) + 1j * rng.standard_normal(b.size(1))
        ref = Ho.mul(x) + Ho2.mul(x)
        y1, y2 = H1 * x, H2 * x
        assert rel(y1, ref) < 1e-12 and rel(y2, ref) < 1e-12
        if not H1.is_complex:
            assert rel(H1 * x.real.astype(np.float32), ref.real) < 2e-6


def test_materialized_matrix_matches_oracle(ek, O):
    """sparse!(opt): the cached sliced-ELL matrix gives the oracle's product on
    every lookup kind, in FP64 and FP32 storage; clearing it restores the
    matrix-free kernels."""
    rng = np.random.default_rng(9)
    L = 12
    cases = [
        (ek.TensorBasis(L=L), O.tensor(L)),
        (ek.ProjectedBasis(L=L, N=6), O.projected(L, N=6)),
        (ek.ProjectedBasis(L=L, N=6, f=lambda d: d[0] == 0), O.projected(L, N=6, f=lambda d: d[0] == 0)),
        (ek.TranslationalBasis(L=L, k=0, N=6), O.translational(L, k=0, N=6)),
        (ek.TranslationalBasis(L=L, k=5, N=6), O.translational(L, k=5, N=6)),
        (ek.TranslationalBasis(L=L, k=1, a=2), O.translational(L, k=1, a=2)),
        (ek.TranslationParityBasis(L=L, k=6, p=-1, N=6), O.transparity(L, k=6, p=-1, N=6)),
    ]
    j2 = ek.spin((0.5, "xx"), (0.5, "yy"), (0.3, "zz"))
    for b, o in cases:
        H = ek.trans_inv_operator(ek.spin(*XXZ), 2, b) + ek.trans_inv_operator(j2, [1, 3], b)
        Ho = O.trans_inv_operator(O.spin(*XXZ), 2, o)
        Ho2 = O.trans_inv_operator(O.spin((0.5, "xx"), (0.5, "yy"), (0.3, "zz")), [1, 3], o)
        x = rng.standard_normal(b.size(1)) + 1j * rng.standard_normal(b.size(1))
        ref = Ho.mul(x) + Ho2.mul(x)
        y_free = H * x
        n = H.sparse_()
        assert n > 0
        assert rel(H * x, ref) < 1e-12
        assert rel(H * x.astype(np.complex64), ref) < 2e-6
        if not H.is_complex:
            assert rel(H * x.real.copy(), ref.real) < 1e-12
        H.clear_sparse_cache_()
        assert np.array_equal(H * x, y_free)


def test_materialized_open_chain_with_fields(ek, O):
    L = 14
    rng = np.random.default_rng(10)
    h = rng.uniform(-3, 3, L)
    b, o = ek.ProjectedBasis(L=L, N=7), O.projected(L, N=7)
    mats = [ek.spin(*XXZ)] * (L - 1) + [hi * ek.spin("z") for hi in h]
    omats = [O.spin(*XXZ)] * (L - 1) + [hi * O.spin("z") for hi in h]
    inds = [[i, i + 1] for i in range(1, L)] + [[i] for i in range(1, L + 1)]
    H, Ho = ek.operator(mats, inds, b), O.operator(omats, inds, o)
    H.sparse_()
    x = rng.standard_normal(b.size(1))
    assert rel(H * x, Ho.mul(x).real) < 1e-12
    y0 = rng.standard_normal(b.size(1))
    y = y0.copy()
    ek.mul_(y, H, x)
    assert rel(y, y0 + Ho.mul(x).real) < 1e-12


def test_pipelined_host_path_matches_device_path(ek, O):
    """Host buffers with D above the chunk size take the pipelined path (row
    chunks, y streamed back while the next chunk computes): identical to the
    device-pointer result for plain, accumulating, tps > 1 and materialised
    application, and to the oracle."""
    import torch
    L = 22
    b = ek.ProjectedBasis(L=L, N=11)  # D = 705,432
    rng = np.random.default_rng(12)
    h = rng.uniform(-1, 1, L)
    mats = [ek.spin(*XXZ)] * (L - 1) + [hi * ek.spin("z") for hi in h]
    omats = [O.spin(*XXZ)] * (L - 1) + [hi * O.spin("z") for hi in h]
    inds = [[i, i + 1] for i in range(1, L)] + [[i] for i in range(1, L + 1)]
    H = ek.operator(mats, inds, b)
    D = b.size(1)
    x = rng.standard_normal(D)
    ref = O.operator(omats, inds, O.projected(L, N=11)).mul(x).real
    xd = torch.from_numpy(x).cuda()
    for setup in ("fast1", "fast2", "materialized"):
        if setup == "fast2":
            H.configure_("fast", 2)
        if setup == "materialized":
            H.sparse_()
        y_host = H * x
        y_dev = (H * xd).cpu().numpy()
        assert np.array_equal(y_host, y_dev), setup
        assert rel(y_host, ref) < 1e-12, setup
        y0 = rng.standard_normal(D)
        y1 = y0.copy()
        ek.mul_(y1, H, x)
        assert rel(y1, y0 + ref) < 1e-12, setup


def test_materialized_any_operator(ek, O):
    """sparse!(opt) for operators outside the bond-family form (one-site x
    fields, three-site terms) and for symmetry-group and dedicated bases:
    explicit-value sliced ELL, equal to the matrix-free product and the
    oracle in every dtype, with accumulation, block right-hand sides and
    Lanczos / batched Lanczos on top."""
    import torch
    rng = np.random.default_rng(31)
    L = 12
    three = np.kron(np.kron(np.array([[0, 1], [1, 0]]), np.eye(2)), np.array([[0, 1], [1, 0]])) * 0.2
    bonds = [[i, i % L + 1] for i in range(1, L + 1)]
    sites = [[i] for i in range(1, L + 1)]
    triples = [[i, (i % L) + 1, ((i + 1) % L) + 1] for i in range(1, L + 1)]
    cases = []
    b = ek.TranslationalBasis(L=L, k=3)
    o = O.translational(L, k=3)
    cases.append(("trans x-field",
                  ek.operator([ek.spin(*XXZ)] * L + [ek.spin((0.3, "x"))] * L, bonds + sites, b),
                  O.operator([O.spin(*XXZ)] * L + [O.spin((0.3, "x"))] * L, bonds + sites, o)))
    bp = ek.ProjectedBasis(L=L, N=6)
    op_ = O.projected(L, N=6)
    cases.append(("proj 3-site",
                  ek.operator([ek.spin(*XXZ)] * L + [three] * L, bonds + triples, bp),
                  O.operator([O.spin(*XXZ)] * L + [three] * L, bonds + triples, op_)))
    ba = ek.basis(L=L, N=6, k=2, z=1)
    oa = O.basis(L, N=6, k=2, z=1)
    cases.append(("abelian", ek.trans_inv_operator(ek.spin(*XXZ), 2, ba),
                  O.trans_inv_operator(O.spin(*XXZ), 2, oa)))
    for name, H, Ho in cases:
        D = H.size(1)
        x = rng.standard_normal(D) + 1j * rng.standard_normal(D)
        ref = Ho.mul(x)
        y_free = H * x
        n = H.sparse_()
        assert n > 0, name
        y_mat = H * x
        assert rel(y_mat, ref) < 1e-12 and rel(y_mat, y_free) < 1e-13, name
        assert rel(H * x.astype(np.complex64), ref) < 2e-6, name
        y0 = rng.standard_normal(D) + 0j
        y1 = y0.copy()
        ek.mul_(y1, H, x)
        assert rel(y1, y0 + ref) < 1e-12, name
        X = np.asfortranarray(rng.standard_normal((D, 6)) + 1j * rng.standard_normal((D, 6)))
        refX = np.stack([Ho.mul(X[:, j]) for j in range(6)], axis=1)
        H.configure_("generic", 1, block=True)
        assert rel(H * X, refX) < 1e-12, name
        H.configure_("generic", 1, block=False)
        assert rel(H * X, refX) < 1e-12, name
        e, _ = ek.lanczos_e0(H, rng.standard_normal(D), m=min(D, 120))
        w = np.linalg.eigvalsh(Ho.dense())
        assert abs(e[0] - w[0]) < 1e-10 * abs(w[0]), name
    # materialised symmetry-group sectors run batched
    ops, refs = [], []
    for k in (0, 1, 3):
        bk_ = ek.basis(L=L, N=6, k=k, z=1)
        Hk = ek.trans_inv_operator(ek.spin(*XXZ), 2, bk_)
        Hk.sparse_()
        ops.append(Hk)
        refs.append(np.linalg.eigvalsh(O.trans_inv_operator(O.spin(*XXZ), 2,
                                                            O.basis(L, N=6, k=k, z=1)).dense())[0])
    ev, _ = ek.batch_lanczos_e0(ops, m=60, tol=1e-13, check_every=5)
    for q in range(3):
        assert abs(ev[q, 0] - refs[q]) < 1e-10 * abs(refs[q]), q


def test_materialized_wide_states(ek, O):
    """L = 34 (64-bit states) materialised: value mode on the wide kernels."""
    L = 34
    b = ek.TranslationalBasis(L=L, k=0, N=3)
    o = O.translational(L, k=0, N=3)
    H = ek.trans_inv_operator(ek.spin(*XXZ), 2, b)
    Ho = O.trans_inv_operator(O.spin(*XXZ), 2, o)
    x = np.random.default_rng(5).standard_normal(b.size(1))
    ref = Ho.mul(x).real
    H.sparse_()
    assert rel(H * x, ref) < 1e-12
