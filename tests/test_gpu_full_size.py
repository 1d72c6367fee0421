"""Parity at the workloads' own sizes.

* J1-J2 XXZ L=32, N=16, k=0 (D = 18,784,170): the rank table's large-sector
  entry format (row << 5 | class, used from 2^22 rows on) gives H*x bit for bit
  equal to the hash search; sampled rows of H*x equal the oracle's colmn!
  (TranslationalBasis.jl:310-341 index, Operator.jl:426-465) within 1e-12; the
  tables agree with the oracle's judge (TranslationalBasis.jl:94-114) on a
  seeded sample of 10^6 states of the charge sector and of 2 * 10^5
  representatives (the oracle's full scan of C(32,16) states takes too long
  here).
* XXZ L=28, N=14, k=0 (D = 1,432,860): E0 of the FP64 and mixed GPU Lanczos
  against the oracle's CGS2 Lanczos on the oracle's own matrix, 1e-12.
* XXZ L=26, N=13, Delta=1.5, all 26 momentum sectors: the lowest four levels
  of FP64, mixed and 64-vector block Lanczos agree within 1e-9; sectors k and
  L-k are degenerate; the lowest sector level is the ground state of the
  whole N=13 space (ProjectedBasis, D = 10,400,600).
* The 512-instance random-field ensemble (L in {12,...,20}): every instance
  with L <= 16 against the oracle's matrix (dense spectrum for L = 12, ARPACK
  for L = 14, 16), every instance FP64 batched against mixed batched, 1e-9."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

XXZ1 = ((1.0, "xx"), (1.0, "yy"), (1.0, "zz"))
J2 = ((0.5, "xx"), (0.5, "yy"), (0.5, "zz"))


def test_L32_j1j2_rank_tables_and_rows(ek, O):
    L = 32
    b = ek.TranslationalBasis(L=L, N=16, k=0)
    H = ek.trans_inv_operator(ek.spin(*XXZ1), 2, b) + ek.trans_inv_operator(ek.spin(*J2), [1, 3], b)
    D = b.size(1)
    assert D == 18_784_170
    I, R = b.I, b.R  # 1-based, as EDKit holds them
    assert np.all(np.diff(I) > 0)
    rng = np.random.default_rng(3232)
    # tables against the oracle's judge: sampled representatives ...
    pick = rng.choice(D, 200_000, replace=False)
    acc, Rj = O.trans_judge(L, I[pick], k=0, N=16)
    assert acc.all() and np.array_equal(Rj, R[pick])
    # ... and sampled states of the charge sector: accepted exactly when present
    n = 1_000_000
    bits = np.argsort(rng.random((n, L)), axis=1)[:, :16]
    states = np.zeros(n, np.uint64)
    for c in range(16):
        states |= np.uint64(1) << bits[:, c].astype(np.uint64)
    idx = states.astype(np.int64) + 1
    acc, Rj = O.trans_judge(L, idx, k=0, N=16)
    where = np.searchsorted(I, idx)
    present = (where < D) & (I[np.minimum(where, D - 1)] == idx)
    assert np.array_equal(acc, present) and acc.sum() > 1000
    assert np.array_equal(Rj[acc], R[where[acc]])
    # H*x: the rank table (row << 5 | class entries) equals the hash search
    x = rng.standard_normal(D)
    b.set_search("hash")
    y_hash = H * x
    b.set_search("rank")
    y_rank = H * x
    assert np.array_equal(y_rank, y_hash)
    # sampled rows against the oracle's colmn!
    Bo = O.translational_from_tables(L, I, R)
    Ho = O.operator([O.spin(*XXZ1)] * L + [O.spin(*J2)] * L,
                    [[i, i % L + 1] for i in range(1, L + 1)] +
                    [[i, (i + 1) % L + 1] for i in range(1, L + 1)], Bo)
    rows = np.sort(rng.choice(D, 20_000, replace=False)) + 1
    yo = Ho.rows_hermitian(rows, x)
    assert np.max(np.abs(yo.imag)) <= 1e-12 * np.max(np.abs(yo.real))
    assert np.linalg.norm(y_rank[rows - 1] - yo.real) <= 1e-12 * np.linalg.norm(yo.real)
    # single-precision complex through the same table (the Krylov workload's dtype)
    xc = (x + 1j * rng.standard_normal(D)).astype(np.complex64)
    yc = H * xc
    yref = Ho.rows_hermitian(rows, xc.astype(np.complex128))
    assert np.linalg.norm(yc[rows - 1] - yref) <= 2e-6 * np.linalg.norm(yref)


def test_L28_E0_against_the_oracle_lanczos(ek, O):
    b = ek.TranslationalBasis(L=28, N=14, k=0)
    H = ek.trans_inv_operator(ek.spin(*XXZ1), 2, b)
    b.set_search("rank")
    v0 = np.random.default_rng(1234).standard_normal(b.size(1))
    e64, _ = ek.lanczos_e0(H, v0, m=300, tol=1e-13, check_every=10)
    emx, _ = ek.lanczos_e0(H, v0, m=300, tol=1e-13, check_every=10, precision="mixed",
                           refine_steps=20)
    # the oracle's basis holds the tables the GPU built (bit-exact with the
    # oracle's own scan: test_gpu_basis.py checks this sector)
    Bo = O.translational_from_tables(28, b.I, b.R)
    M = O.trans_inv_operator(O.spin(*XXZ1), 2, Bo).sparse().real  # the nonzeros colmn! scatters
    ref = O.lanczos_e0(lambda v: M @ v, v0, 120, blas=True)[0][0]
    assert abs(e64[0] - ref) <= 1e-12 * abs(ref)
    assert abs(emx[0] - ref) <= 1e-12 * abs(ref)


def test_L26_all_momentum_sectors(ek):
    bond = ek.spin((1.0, "xx"), (1.0, "yy"), (1.5, "zz"))
    bases = [ek.TranslationalBasis(L=26, N=13, k=k) for k in range(26)]
    for b in bases:
        b.set_search("rank")
    ops = [ek.trans_inv_operator(bond, 2, b) for b in bases]
    e64, _ = ek.batch_lanczos_e0(ops, m=300, nev=4, tol=1e-12, check_every=10)
    emx, _ = ek.batch_lanczos_e0(ops, m=300, nev=4, tol=1e-12, check_every=10, precision="mixed")
    scale = np.abs(e64[:, :1])
    assert np.max(np.abs(emx - e64) / scale) <= 1e-9
    for k in range(1, 13):  # k and L - k: complex-conjugate sectors, the same spectrum
        assert np.max(np.abs(e64[k] - e64[26 - k])) <= 1e-10 * scale[k, 0]
    evb, _ = ek.block_lanczos(ops, block=64, m=100, nev=4, check_every=0, seed=2026)
    assert np.max(np.abs(evb - e64) / scale) <= 1e-9
    # the lowest sector level is the ground state of the whole N = 13 space
    P = ek.ProjectedBasis(L=26, N=13)
    HP = ek.trans_inv_operator(bond, 2, P)
    eP, _ = ek.lanczos_e0(HP, m=300, tol=1e-13, check_every=10)
    assert abs(eP[0] - e64[:, 0].min()) <= 1e-10 * abs(eP[0])


def test_random_field_ensemble_512(ek, O):
    import scipy.sparse.linalg as sla
    rng = np.random.default_rng(2024)
    ops, oracle_cases = [], []
    for q in range(512):
        L = int(rng.choice([12, 14, 16, 18, 20]))
        h = rng.uniform(-3, 3, L)
        inds = [[i, i + 1] for i in range(1, L)] + [[i] for i in range(1, L + 1)]
        ops.append(ek.operator([ek.spin(*XXZ1)] * (L - 1) + [hi * ek.spin("z") for hi in h], inds,
                               ek.ProjectedBasis(L=L, N=L // 2)))
        if L <= 16:
            oracle_cases.append((q, L, [O.spin(*XXZ1)] * (L - 1) + [hi * O.spin("z") for hi in h],
                                 inds))
    v0s = [np.random.default_rng(q).standard_normal(op.size(1)) for q, op in enumerate(ops)]
    e64, _ = ek.batch_lanczos_e0(ops, v0s, m=200, nev=4, tol=1e-12, check_every=10)
    emx, _ = ek.batch_lanczos_e0(ops, v0s, m=200, nev=4, tol=1e-12, check_every=10,
                                 precision="mixed")
    scale = np.abs(e64[:, :1])
    assert np.max(np.abs(emx - e64) / scale) <= 1e-9
    for q, L, omats, inds in oracle_cases:
        M = O.operator(omats, inds, O.projected(L, N=L // 2)).sparse().real
        if L <= 12:
            ref = np.linalg.eigvalsh(M.toarray())[:4]
        else:  # ARPACK on the oracle's matrix: a solver independent of the GPU's
            ref = np.sort(sla.eigsh(M, k=4, which="SA", tol=1e-14, v0=np.ones(M.shape[0]))[0])
        assert np.max(np.abs(e64[q] - ref)) <= 1e-9 * abs(ref[0]), (q, L)
    assert len(oracle_cases) > 250
