"""Index-search strategies, kernel choices and the autotuner.

Every combination must give the same rows as EDKit's index() (bit-exact,
checked against the oracle) and the same H*x as the oracle's mul
(<= 1e-12 relative in FP64); the autotuner only changes speed."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

XXZ = ((1.0, "xx"), (1.0, "yy"), (1.5, "zz"))


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300)


def pxp(d):
    return all(not (d[i] == 1 and d[(i + 1) % len(d)] == 1) for i in range(len(d)))


def searchable(ek, O, L=12):
    return [
        ("proj_pred", ek.ProjectedBasis(L=L, f=pxp), O.projected(L, f=pxp)),
        ("trans0", ek.TranslationalBasis(L=L, k=0, N=6), O.translational(L, k=0, N=6)),
        ("trans_k", ek.TranslationalBasis(L=L, k=5), O.translational(L, k=5)),
        ("trans_a2", ek.TranslationalBasis(L=L, k=3, a=2), O.translational(L, k=3, a=2)),
        ("transpar", ek.TranslationParityBasis(L=L, k=6, p=-1), O.transparity(L, k=6, p=-1)),
        ("abelian", ek.basis(L=L, N=6, k=1, z=-1), O.basis(L, N=6, k=1, z=-1)),
    ]


def test_sorted_search_index_bit_exact(ek, O):
    rng = np.random.default_rng(3)
    L = 12
    states = rng.integers(0, 2 ** L, size=600).astype(np.uint64)
    for name, b, o in searchable(ek, O, L):
        p_hash, c_hash = b.index_states(states)
        b.set_search("sorted")
        assert b.get_search() == "sorted"
        p_sort, c_sort = b.index_states(states)
        assert np.array_equal(p_hash, p_sort), name
        assert np.array_equal(c_hash, c_sort), name
        for s, p in zip(states[:80], p_sort[:80]):
            dgt = np.array([(int(s) >> (L - 1 - q)) & 1 for q in range(L)])
            co, po = o.index(dgt)
            assert p == (po if co != 0 else 0), (name, s)
        b.set_search("hash")


def test_sorted_search_wide_states(ek, O):
    """L = 34 > 32: the 64-bit sorted search over the state array."""
    L = 34
    b = ek.TranslationalBasis(L=L, k=0, N=2)
    o = O.translational(L, k=0, N=2)
    oI, oR = o.tables()
    assert np.array_equal(b.I, oI) and np.array_equal(b.R, oR)
    rng = np.random.default_rng(5)
    st = [int(x) - 1 for x in oI] + [int(v) for v in rng.integers(0, 2 ** 40, size=50)]
    st = np.array([v % (1 << L) for v in st], dtype=np.uint64)
    p0, c0 = b.index_states(st)
    b.set_search("sorted")
    p1, c1 = b.index_states(st)
    assert np.array_equal(p0[:len(oI)], np.arange(1, len(oI) + 1))
    assert np.array_equal(p0, p1) and np.array_equal(c0, c1)
    H = ek.trans_inv_operator(ek.spin(*XXZ), 2, b)
    Ho = O.trans_inv_operator(O.spin(*XXZ), 2, o)
    x = rng.standard_normal(b.size(1))
    assert rel(H * x, Ho.mul(x).real) < 1e-12


def test_direct_bases_have_no_search(ek):
    import edkit_b200._lib as E
    for b in (ek.TensorBasis(L=8), ek.ProjectedBasis(L=8, N=4)):
        with pytest.raises(E.EDKError):
            b.set_search("sorted")


def test_every_kernel_choice_matches_oracle(ek, O):
    rng = np.random.default_rng(1)
    for name, b, o in searchable(ek, O):
        H = ek.trans_inv_operator(ek.spin(*XXZ), 2, b)
        Ho = O.trans_inv_operator(O.spin(*XXZ), 2, o)
        D = b.size(1)
        x = rng.standard_normal(D) + 1j * rng.standard_normal(D)
        ref = Ho.mul(x)
        fast = H.n_families > 0 and b.L <= 32 and name != "abelian"
        for search in ("hash", "sorted"):
            b.set_search(search)
            choices = [("generic", 1)] + ([("fast", t) for t in (1, 2, 4)] if fast else [])
            for kernel, tps in choices:
                H.configure_(kernel, tps)
                assert rel(H * x, ref) < 1e-12, (name, search, kernel, tps)
                assert rel(H * x.astype(np.complex64), ref) < 2e-6, (name, search, kernel, tps)
        b.set_search("hash")


def test_threads_per_state_with_fields(ek, O):
    """Fast kernel with diagonal fields and a second bond family, every tps,
    ragged last tile (D not a multiple of the rows per tile)."""
    L = 14
    b = ek.ProjectedBasis(L=L, N=7)
    o = O.projected(L, N=7)
    rng = np.random.default_rng(2)
    h = rng.uniform(-1, 1, L)
    mats = [ek.spin(*XXZ)] * (L - 1) + [ek.spin((0.4, "xx"), (0.4, "yy"))] * (L - 2) + \
        [hi * ek.spin("z") for hi in h]
    omats = [O.spin(*XXZ)] * (L - 1) + [O.spin((0.4, "xx"), (0.4, "yy"))] * (L - 2) + \
        [hi * O.spin("z") for hi in h]
    inds = [[i, i + 1] for i in range(1, L)] + [[i, i + 2] for i in range(1, L - 1)] + \
        [[i] for i in range(1, L + 1)]
    H = ek.operator(mats, inds, b)
    Ho = O.operator(omats, inds, o)
    x = rng.standard_normal(b.size(1))
    ref = Ho.mul(x).real
    for tps in (1, 2, 4):
        H.configure_("fast", tps)
        assert rel(H * x, ref) < 1e-12, tps
        X = rng.standard_normal((b.size(1), 3))
        Y = H * np.asfortranarray(X)
        for j in range(3):
            assert rel(Y[:, j], Ho.mul(X[:, j]).real) < 1e-12, (tps, j)


def test_autotune_installs_a_correct_choice(ek, O):
    L = 16
    b = ek.TranslationalBasis(L=L, k=3, N=8)
    o = O.translational(L, k=3, N=8)
    H = ek.trans_inv_operator(ek.spin(*XXZ), 2, b)
    Ho = O.trans_inv_operator(O.spin(*XXZ), 2, o)
    rng = np.random.default_rng(4)
    x = rng.standard_normal(b.size(1)) + 1j * rng.standard_normal(b.size(1))
    ref = Ho.mul(x)
    r = H.autotune_()
    kinds = {(k, s, t) for k, s, t, _ in r["candidates"]}
    assert ("generic", "hash", 1) in kinds and ("generic", "sorted", 1) in kinds
    assert ("fast", "sorted", 4) in kinds
    assert all(ms > 0 for *_, ms in r["candidates"])
    assert r["ms"] == min(ms for *_, ms in r["candidates"])
    assert b.get_search() == r["search"]
    assert rel(H * x, ref) < 1e-12
    r2 = H.autotune_(materialize=True)
    assert any(k == "materialized" for k, *_ in r2["candidates"])
    assert rel(H * x, ref) < 1e-12
    e, _ = ek.lanczos_e0(H, rng.standard_normal(b.size(1)), m=80)
    E0 = np.linalg.eigvalsh(Ho.dense())[0]
    assert abs(e[0] - E0) < 1e-10 * abs(E0)


def test_batch_lanczos_with_sorted_search(ek, O):
    L = 12
    ops, refs = [], []
    for k in (0, 1, 6):
        b = ek.TranslationalBasis(L=L, N=6, k=k)
        b.set_search("sorted")
        ops.append(ek.trans_inv_operator(ek.spin(*XXZ), 2, b))
        Ho = O.trans_inv_operator(O.spin(*XXZ), 2, O.translational(L, k=k, N=6))
        refs.append(np.linalg.eigvalsh(Ho.dense())[:2])
    ev, _ = ek.batch_lanczos_e0(ops, m=80, nev=2, tol=1e-13, check_every=5)
    for q in range(3):
        assert np.allclose(ev[q], refs[q], rtol=0, atol=1e-10 * abs(refs[q][0])), q


@pytest.mark.parametrize("nvec", [4, 5, 70])
def test_block_rhs_spmm_matches_columns(ek, O, nvec):
    """Several right-hand sides as one SpMM (every hit located once for all
    columns): equal to the column-at-a-time kernels and to the oracle, for
    every dtype, accumulation, strided blocks, and the materialised matrix;
    more than 64 columns run in chunks."""
    import torch
    L = 16
    b = ek.TranslationalBasis(L=L, N=8, k=3)
    o = O.translational(L, k=3, N=8)
    H = ek.trans_inv_operator(ek.spin(*XXZ), 2, b)
    Ho = O.trans_inv_operator(O.spin(*XXZ), 2, o)
    D = b.size(1)
    rng = np.random.default_rng(nvec)
    X = np.asfortranarray(rng.standard_normal((D, nvec)) + 1j * rng.standard_normal((D, nvec)))
    ref = np.stack([Ho.mul(X[:, j]) for j in range(nvec)], axis=1)
    for mat in (False, True):
        if mat:
            H.sparse_()
        H.configure_("fast", 1, block=True)
        Yb = H * X
        H.configure_("fast", 1, block=False)
        Yc = H * X
        H.configure_("fast", 1, block=True)
        assert rel(Yb, ref) < 1e-12 and rel(Yb, Yc) < 1e-13, mat
        assert rel(H * X.astype(np.complex64), ref) < 2e-6, mat
        # accumulate into a strided (ld > D) device block
        Xd = torch.from_numpy(np.ascontiguousarray(X.T)).cuda()       # (nvec, D) row-major
        Xpad = torch.zeros((nvec, D + 7), dtype=torch.complex128, device="cuda")
        Xpad[:, :D] = Xd
        Y0 = torch.from_numpy(np.ascontiguousarray(rng.standard_normal((nvec, D + 7)) + 0j)).cuda()
        Y1 = Y0.clone()
        from edkit_b200 import _lib as E
        E.check(E.load().edk_apply(H._h, E.C128, E.ptr(Xpad), E.ptr(Y1), nvec, D + 7, D + 7, 1,
                                   E.DEVICE))
        got = (Y1 - Y0)[:, :D].cpu().numpy().T
        assert rel(got, ref) < 1e-12, mat
        assert torch.equal(Y1[:, D:], Y0[:, D:])
        H.clear_sparse_cache_()
    # real operator, real dtypes
    Hr = ek.trans_inv_operator(ek.spin(*XXZ), 2, ek.TranslationalBasis(L=L, N=8, k=0))
    Hro = O.trans_inv_operator(O.spin(*XXZ), 2, O.translational(L, k=0, N=8))
    Dr = Hr.size(1)
    Xr = np.asfortranarray(rng.standard_normal((Dr, nvec)))
    refr = np.stack([Hro.mul(Xr[:, j]).real for j in range(nvec)], axis=1)
    assert rel(Hr * Xr, refr) < 1e-12
    assert rel(Hr * Xr.astype(np.float32), refr) < 2e-6


def test_autotune_with_block_rhs(ek, O):
    b = ek.TranslationalBasis(L=18, N=9, k=0)
    H = ek.trans_inv_operator(ek.spin(*XXZ), 2, b)
    r = H.autotune_(nvec=16, materialize=True)
    assert any(r["candidates_block"])
    X = np.asfortranarray(np.random.default_rng(0).standard_normal((b.size(1), 16)))
    Ho = O.trans_inv_operator(O.spin(*XXZ), 2, O.translational(18, k=0, N=9))
    ref = np.stack([Ho.mul(X[:, j]).real for j in range(16)], axis=1)
    assert rel(H * X, ref) < 1e-12


def test_staged_materialized_product(ek, O):
    """The materialised product with its entry stream staged in shared memory
    by bulk copies equals the plain one bit for bit (every dtype, accumulate,
    pipelined host path) and the oracle."""
    import torch
    L = 22
    b = ek.TranslationalBasis(L=L, N=11, k=2)  # D = 32,066: 126 windows
    o = O.translational(L, k=2, N=11)
    H = ek.trans_inv_operator(ek.spin(*XXZ), 2, b)
    Ho = O.trans_inv_operator(O.spin(*XXZ), 2, o)
    D = b.size(1)
    rng = np.random.default_rng(21)
    x = rng.standard_normal(D) + 1j * rng.standard_normal(D)
    ref = Ho.mul(x)
    H.sparse_()
    H.configure_("materialized")
    y_plain = H * x
    y32_plain = H * x.astype(np.complex64)
    H.configure_("materialized_staged")
    y_st = H * x
    assert np.array_equal(y_st, y_plain) and rel(y_st, ref) < 1e-12
    assert np.array_equal(H * x.astype(np.complex64), y32_plain)
    y0 = rng.standard_normal(D) + 0j
    y1 = y0.copy()
    ek.mul_(y1, H, x)
    assert rel(y1, y0 + ref) < 1e-12
    r = H.autotune_(dtype=None, materialize=True)
    assert any(k == "materialized_staged" for k, *_ in r["candidates"])
    assert rel(H * x, ref) < 1e-12
    # a large real sector through the pipelined host path
    b2 = ek.ProjectedBasis(L=22, N=11)
    H2 = ek.trans_inv_operator(ek.spin(*XXZ), 2, b2)
    H2.sparse_()
    x2 = rng.standard_normal(b2.size(1))
    H2.configure_("materialized")
    a = H2 * x2
    H2.configure_("materialized_staged")
    assert np.array_equal(H2 * x2, a)
    assert np.array_equal((H2 * torch.from_numpy(x2).cuda()).cpu().numpy(), a)
