"""The rank-table index search (EDK_SEARCH_RANK) of translation sectors of
fixed N: the bond-family row kernel finds target rows (and, for k != 0, the
shift that sets the phase) by updating the colex rank of the row state and
reading one table entry.  Rows are the ones EDKit's
index() gives, so H*x must equal the hash-table result bit for bit and the
oracle's mul within 1e-12 (FP64)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

XXZ = ((1.0, "xx"), (1.0, "yy"), (1.5, "zz"))


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300)


def j1j2(ek, L, b, h=None):
    mats = [ek.spin(*XXZ)] * L + [ek.spin((0.5, "xx"), (0.5, "yy"), (0.5, "zz"))] * L
    inds = [[i, i % L + 1] for i in range(1, L + 1)] + [[i, (i + 1) % L + 1] for i in range(1, L + 1)]
    if h is not None:
        mats += [h * ek.spin("z")] * L
        inds += [[i] for i in range(1, L + 1)]
    return ek.operator(mats, inds, b)


def pxp(d):
    return all(not (d[i] == 1 and d[(i + 1) % len(d)] == 1) for i in range(len(d)))


@pytest.mark.parametrize("L,N", [(12, 6), (16, 8), (16, 5), (20, 10), (24, 12)])
def test_rank_search_bit_exact_with_hash(ek, O, L, N):
    rng = np.random.default_rng(L + N)
    b = ek.TranslationalBasis(L=L, k=0, N=N)
    ops = [("xxz", ek.trans_inv_operator(ek.spin(*XXZ), 2, b)),
           ("j1j2+h", j1j2(ek, L, b, h=0.3))]
    D = b.size(1)
    for name, H in ops:
        for dt in (np.float64, np.complex128, np.float32):
            x = rng.standard_normal(D).astype(dt)
            if np.iscomplexobj(x):
                x = x + 1j * rng.standard_normal(D)
            for tps in (1, 2, 4):
                H.configure_("fast", tps)
                b.set_search("hash")
                y_hash = H * x
                b.set_search("rank")
                assert b.get_search() == "rank"
                y_rank = H * x
                assert np.array_equal(y_rank, y_hash), (name, dt, tps)
        b.set_search("hash")
    if L <= 16:  # and against the oracle
        o = O.translational(L, k=0, N=N)
        Ho = O.trans_inv_operator(O.spin(*XXZ), 2, o)
        x = rng.standard_normal(D)
        b.set_search("rank")
        H = ops[0][1]
        H.configure_("fast", 1)
        assert rel(H * x, Ho.mul(x).real) < 1e-12


def test_rank_search_with_predicate_and_unit_cell_rejected(ek, O):
    """A predicate drops states (their table entries stay empty); bases the
    table does not serve are refused with EDK_UNSUPPORTED."""
    L = 14
    b = ek.TranslationalBasis(L=L, k=0, N=9, f=pxp)  # 5 up spins, no two adjacent
    o = O.translational(L, k=0, N=9, f=pxp)
    assert b.size(1) == o.dim > 0
    H = ek.trans_inv_operator(ek.spin(*XXZ), 2, b)
    Ho = O.trans_inv_operator(O.spin(*XXZ), 2, o)
    x = np.random.default_rng(3).standard_normal(b.size(1))
    b.set_search("rank")
    H.configure_("fast", 1)
    assert rel(H * x, Ho.mul(x).real) < 1e-12
    for bad in (ek.TranslationalBasis(L=L, k=1), ek.TranslationalBasis(L=L, k=0),
                ek.TranslationParityBasis(L=L, k=0, p=1), ek.ProjectedBasis(L=L, N=7, f=pxp)):
        with pytest.raises(ek.EDKError):
            bad.set_search("rank")


def test_rank_search_lanczos_and_batches(ek, O):
    L = 16
    rng = np.random.default_rng(5)
    refs, ops = [], []
    for N in (7, 8):
        b = ek.TranslationalBasis(L=L, k=0, N=N)
        o = O.translational(L, k=0, N=N)
        b.set_search("rank")
        ops.append(ek.trans_inv_operator(ek.spin(*XXZ), 2, b))
        refs.append(np.linalg.eigvalsh(O.trans_inv_operator(O.spin(*XXZ), 2, o).dense())[:2])
    e, _ = ek.lanczos_e0(ops[1], rng.standard_normal(ops[1].size(1)), m=120, tol=1e-13)
    assert abs(e[0] - refs[1][0]) < 1e-11 * abs(refs[1][0])
    ev, _ = ek.batch_lanczos_e0(ops, m=120, nev=2, tol=1e-13, check_every=5)
    for q in range(2):
        assert np.allclose(ev[q], refs[q], rtol=0, atol=1e-10 * abs(refs[q][0])), q


def test_autotune_offers_rank_search(ek, O):
    L = 18
    b = ek.TranslationalBasis(L=L, k=0, N=9)
    o = O.translational(L, k=0, N=9)
    H = ek.trans_inv_operator(ek.spin(*XXZ), 2, b)
    Ho = O.trans_inv_operator(O.spin(*XXZ), 2, o)
    r = H.autotune_()
    kinds = {(k, s, t) for k, s, t, _ in r["candidates"]}
    assert ("fast", "rank", 1) in kinds
    assert b.get_search() == r["search"]
    x = np.random.default_rng(6).standard_normal(b.size(1))
    assert rel(H * x, Ho.mul(x).real) < 1e-12


@pytest.mark.parametrize("nvec", [5, 64])
def test_rank_search_spmm_bit_exact_with_hash(ek, nvec):
    """Several right-hand sides through one SpMM (which locates rows through
    the hash table whatever the basis' search: there the psi rows, not the
    lookups, set the time): the same block product under either search."""
    L = 20
    b = ek.TranslationalBasis(L=L, k=0, N=10)
    H = j1j2(ek, L, b, h=0.2)
    rng = np.random.default_rng(nvec)
    X = np.asfortranarray(rng.standard_normal((b.size(1), nvec)))
    H.configure_("fast", 1, block=True)
    b.set_search("hash")
    Y_hash = H * X
    b.set_search("rank")
    Y_rank = H * X
    assert np.array_equal(Y_rank, Y_hash)
    H.configure_("fast", 1, block=False)
    assert rel(H * X, Y_hash) < 1e-14
    b.set_search("hash")


def test_block_lanczos_mixes_ranked_and_phased_sectors(ek, O):
    """A block Lanczos batch with a rank-searched k = 0 sector beside k != 0
    sectors runs on the shared translation path and finds the sectors' levels."""
    L = 14
    ops, refs = [], []
    for k in (0, 1, 7):
        b = ek.TranslationalBasis(L=L, k=k, N=7)
        if k == 0:
            b.set_search("rank")
        ops.append(ek.trans_inv_operator(ek.spin(*XXZ), 2, b))
        Ho = O.trans_inv_operator(O.spin(*XXZ), 2, O.translational(L, k=k, N=7))
        w = np.linalg.eigvalsh(Ho.dense())
        distinct = [w[0]] + [x for a, x in zip(w[:-1], w[1:]) if x - a > 1e-8 * abs(w[0])]
        refs.append(distinct[:3])
    ev, _ = ek.block_lanczos(ops, block=8, m=24, nev=3, check_every=0)
    for q in range(3):
        assert np.allclose(ev[q][:3], refs[q], rtol=0, atol=1e-9 * abs(refs[q][0])), q


@pytest.mark.parametrize("L,N,k,a", [(12, 6, 1, 1), (16, 8, 3, 1), (16, 7, 8, 1), (20, 10, 7, 1),
                                     (16, 8, 3, 2)])
def test_rank_search_phased_sectors_bit_exact(ek, O, L, N, k, a):
    """k != 0: the table entry also carries the first-minimum shift M, so the
    phase C[M] equals the one index() gives; H*x bit-identical to the hash path."""
    rng = np.random.default_rng(L * 100 + k)
    b = ek.TranslationalBasis(L=L, k=k, N=N, a=a)
    ops = [("xxz", ek.trans_inv_operator(ek.spin(*XXZ), 2, b))]
    if a == 1:
        ops.append(("j1j2+h", j1j2(ek, L, b, h=0.3)))
    D = b.size(1)
    for name, H in ops:
        for dt in (np.complex128, np.complex64):
            x = (rng.standard_normal(D) + 1j * rng.standard_normal(D)).astype(dt)
            for tps in (1, 2):
                H.configure_("fast", tps)
                b.set_search("hash")
                y_hash = H * x
                b.set_search("rank")
                y_rank = H * x
                assert np.array_equal(y_rank, y_hash), (name, dt, tps)
    o = O.translational(L, k=k, N=N, a=a)
    Ho = O.trans_inv_operator(O.spin(*XXZ), 2, o)
    x = rng.standard_normal(D) + 1j * rng.standard_normal(D)
    b.set_search("rank")
    ops[0][1].configure_("fast", 1)
    assert rel(ops[0][1] * x, Ho.mul(x)) < 1e-12


def test_rank_search_all_momentum_sectors_batched(ek, O):
    """Every momentum sector rank-searched, one batched Lanczos (FP64 and
    mixed) against the sectors' dense spectra."""
    L = 14
    ops, refs = [], []
    for k in range(L):
        b = ek.TranslationalBasis(L=L, k=k, N=7)
        b.set_search("rank")
        ops.append(ek.trans_inv_operator(ek.spin(*XXZ), 2, b))
        Ho = O.trans_inv_operator(O.spin(*XXZ), 2, O.translational(L, k=k, N=7))
        refs.append(np.linalg.eigvalsh(Ho.dense())[:2])
    for prec in ("fp64", "mixed"):
        ev, _ = ek.batch_lanczos_e0(ops, m=150, nev=2, tol=1e-12, check_every=5, precision=prec)
        for q in range(L):
            assert np.allclose(ev[q], refs[q], rtol=0, atol=1e-9 * abs(refs[q][0])), (prec, q)


def test_run_canonicalisation_gives_the_same_rows(ek, monkeypatch):
    """EDK_CANON_RUNS=1 canonicalises k = 0 states by comparing only the
    rotations that start at a domain wall; the representative, hence every
    row and H*x (hash and rank searches), is the same as the full scan's."""
    L = 16
    rng = np.random.default_rng(11)
    b0 = ek.TranslationalBasis(L=L, k=0, N=8)
    H0 = ek.trans_inv_operator(ek.spin(*XXZ), 2, b0)
    x = rng.standard_normal(b0.size(1))
    y0 = H0 * x
    monkeypatch.setenv("EDK_CANON_RUNS", "1")
    b1 = ek.TranslationalBasis(L=L, k=0, N=8)
    monkeypatch.delenv("EDK_CANON_RUNS")
    H1 = ek.trans_inv_operator(ek.spin(*XXZ), 2, b1)
    assert np.array_equal(b1.I, b0.I) and np.array_equal(b1.R, b0.R)
    assert np.array_equal(H1 * x, y0)
    b1.set_search("rank")
    assert np.array_equal(H1 * x, y0)


@pytest.mark.parametrize("L,N,k,p", [(12, 6, 0, 1), (14, 7, 0, -1), (16, 8, 8, 1), (16, 7, 8, -1),
                                     (20, 10, 0, 1)])
def test_rank_search_translation_parity_bit_exact(ek, O, L, N, k, p):
    """TranslationParityBasis: the entry carries the sign of the coefficient
    (P C[M] or C[R], +-1), so H*x is bit-identical to the hash path."""
    rng = np.random.default_rng(L * 10 + N + k)
    b = ek.TranslationParityBasis(L=L, k=k, p=p, N=N)
    ops = [("xxz", ek.trans_inv_operator(ek.spin(*XXZ), 2, b)), ("j1j2+h", j1j2(ek, L, b, h=0.3))]
    D = b.size(1)
    for name, H in ops:
        for dt in (np.float64, np.float32, np.complex128):
            x = rng.standard_normal(D).astype(dt)
            if np.iscomplexobj(x):
                x = x + 1j * rng.standard_normal(D)
            for tps in (1, 2):
                H.configure_("fast", tps)
                b.set_search("hash")
                y_hash = H * x
                b.set_search("rank")
                assert np.array_equal(H * x, y_hash), (name, dt, tps)
    if L <= 16:
        o = O.transparity(L, k=k, p=p, N=N)
        Ho = O.trans_inv_operator(O.spin(*XXZ), 2, o)
        x = rng.standard_normal(D)
        b.set_search("rank")
        ops[0][1].configure_("fast", 1)
        assert rel(ops[0][1] * x, Ho.mul(x).real) < 1e-12
    # batched Lanczos over both parities, rank-searched
    ops2, refs = [], []
    if L <= 14:
        for pp in (1, -1):
            bb = ek.TranslationParityBasis(L=L, k=k, p=pp, N=N)
            bb.set_search("rank")
            ops2.append(ek.trans_inv_operator(ek.spin(*XXZ), 2, bb))
            Ho = O.trans_inv_operator(O.spin(*XXZ), 2, O.transparity(L, k=k, p=pp, N=N))
            refs.append(np.linalg.eigvalsh(Ho.dense())[0])
        ev, _ = ek.batch_lanczos_e0(ops2, m=min(120, min(o.size(1) for o in ops2) - 1), nev=1,
                                    tol=1e-13, check_every=5)
        for q in range(2):
            assert abs(ev[q][0] - refs[q]) <= 1e-10 * abs(refs[q]), q
