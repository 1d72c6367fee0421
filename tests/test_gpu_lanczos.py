"""GPU Lanczos ground states and Krylov time evolution against the oracle.

E0 tolerance: FP64 <= 1e-12 relative; mixed precision (FP32 Krylov vectors,
FP64 refinement) <= 1e-9 relative.  Krylov states: the reference's own test
tolerances (timeevolve_tests.jl: 1e-10 / 1e-9)."""
import numpy as np
import pytest
from scipy.linalg import expm

pytestmark = pytest.mark.gpu


def xxz(S, delta):
    return S((1.0, "xx"), (1.0, "yy"), (delta, "zz"))


def test_e0_matches_dense_small(ek, O):
    L = 12
    b = ek.TranslationalBasis(L=L, k=0, N=6)
    H = ek.trans_inv_operator(xxz(ek.spin, 1.0), 2, b)
    Ho = O.trans_inv_operator(xxz(O.spin, 1.0), 2, O.translational(L, k=0, N=6))
    ref = np.linalg.eigvalsh(Ho.dense())
    ev, info = ek.lanczos_e0(H, m=min(b.size(1), 120), nev=3)
    assert np.allclose(ev, ref[:3], rtol=0, atol=1e-12 * abs(ref[0]))
    assert info["steps"] <= b.size(1)


def test_lanczos_coefficients_match_cgs2_oracle(ek, O):
    """alpha/beta of the GPU CGS2 Lanczos equal the restated _lanczos_build!."""
    L = 14
    b = ek.TranslationalBasis(L=L, k=0, N=7)
    H = ek.trans_inv_operator(xxz(ek.spin, 1.0), 2, b)
    Ho = O.trans_inv_operator(xxz(O.spin, 1.0), 2, O.translational(L, k=0, N=7))
    v0 = np.random.default_rng(3).standard_normal(b.size(1))
    ev, info, a, bb = ek.lanczos_e0(H, v0, m=40, return_coeffs=True)
    ea, oa, ob = O.lanczos_e0(lambda v: Ho.mul(v), v0.astype(complex), 40)
    assert np.allclose(a, oa[: len(a)], atol=1e-10)
    assert np.allclose(bb, ob[: len(bb)], atol=1e-10)
    assert abs(ev[0] - ea[0]) < 1e-12 * abs(ea[0])


def test_config1_tensor_l16_e0(ek, O):
    """Open XXZ L=16, Delta=1.5 on the full TensorBasis (D=65536), complex start
    vector, 150-step Lanczos; E0 vs the minimum over fixed-N sectors computed
    with ARPACK on the oracle's matvec (dense 65536^2 is out of reach)."""
    from scipy.sparse.linalg import LinearOperator, eigsh
    L = 16
    b = ek.TensorBasis(L=L)
    inds = [[i, i + 1] for i in range(1, L)]
    H = ek.operator([xxz(ek.spin, 1.5)] * (L - 1), inds, b)
    rng = np.random.default_rng(1234)
    v0 = rng.standard_normal(2 ** L) + 1j * rng.standard_normal(2 ** L)
    v0 /= np.linalg.norm(v0)
    ev, info = ek.lanczos_e0(H, v0, m=150)
    e_sec = []
    for N in (7, 8, 9):
        o = O.projected(L, N=N)
        Ho = O.operator([xxz(O.spin, 1.5)] * (L - 1), inds, o)
        op = LinearOperator((o.dim, o.dim), matvec=lambda v, Ho=Ho: Ho.mul(v).real,
                            dtype=np.float64)
        e_sec.append(eigsh(op, k=1, which="SA", tol=1e-14)[0][0])
    ref = min(e_sec)
    assert abs(ev[0] - ref) < 1e-12 * abs(ref)


def test_mixed_precision_e0(ek, O):
    L = 20
    b = ek.TranslationalBasis(L=L, k=0, N=10)
    H = ek.trans_inv_operator(xxz(ek.spin, 1.0), 2, b)
    v0 = np.random.default_rng(2).standard_normal(b.size(1))
    e64, _ = ek.lanczos_e0(H, v0, m=200, tol=1e-13, check_every=5)
    emx, info = ek.lanczos_e0(H, v0, m=200, tol=1e-13, check_every=5, precision="mixed")
    assert abs(emx[0] - e64[0]) <= 1e-9 * abs(e64[0])
    assert info["steps_low"] > 0


def test_e0_zero_norm_error(ek):
    b = ek.TranslationalBasis(L=8, k=0, N=4)
    H = ek.trans_inv_operator(xxz(ek.spin, 1.0), 2, b)
    with pytest.raises(ek.EDKError, match="zero norm"):
        ek.lanczos_e0(H, np.zeros(b.size(1)), m=10)


def _dense_exp(Hd, psi0, t):
    return expm(-1j * t * Hd) @ psi0


def test_timeevolve_tensor_dense_reference(ek, O):
    """timeevolve_tests.jl:10-36."""
    L = 6
    bond = ek.spin((1.0, "xx"), (1.0, "yy"), (0.7, "zz"))
    H = ek.trans_inv_operator(bond, [1, 2], ek.TensorBasis(L=L))
    Hd = O.trans_inv_operator(O.spin((1.0, "xx"), (1.0, "yy"), (0.7, "zz")), [1, 2],
                              O.tensor(L)).dense()
    rng = np.random.default_rng(11)
    psi0 = rng.standard_normal(2 ** L) + 1j * rng.standard_normal(2 ** L)
    psi0 /= np.linalg.norm(psi0)
    for t in (0.1, 0.5, 1.7, 0.0):
        psi = ek.timeevolve(H, psi0, t, tol=1e-12, m_init=25, m_max=50)
        assert np.linalg.norm(psi - _dense_exp(Hd, psi0, t)) < 1e-10
        assert abs(np.linalg.norm(psi) - 1) < 1e-10
    ts = np.linspace(0, 3, 31)
    psis, diag = ek.timeevolve(H, psi0, ts, tol=1e-12, m_init=25, m_max=50,
                               return_diagnostics=True)
    for i, t in enumerate(ts):
        assert np.linalg.norm(psis[:, i] - _dense_exp(Hd, psi0, t)) < 1e-10
    assert diag.total_times_served == len(ts)


def test_timeevolve_symmetry_sector(ek, O):
    """timeevolve_tests.jl:53-69: TranslationalBasis L=8 N=4 k=0."""
    L = 8
    bond_e = ek.spin((1.0, "+-"), (1.0, "-+"), (0.5, "zz"))
    b = ek.TranslationalBasis(L=L, k=0, N=4)
    H = ek.trans_inv_operator(bond_e, [1, 2], b)
    Hd = O.trans_inv_operator(O.spin((1.0, "+-"), (1.0, "-+"), (0.5, "zz")), [1, 2],
                              O.translational(L, k=0, N=4)).dense()
    rng = np.random.default_rng(12)
    psi0 = rng.standard_normal(b.size(1)) + 1j * rng.standard_normal(b.size(1))
    psi0 /= np.linalg.norm(psi0)
    ts = [0.3, 0.9, 1.4]
    psis = ek.timeevolve(H, psi0, ts, tol=1e-11, m_init=20, m_max=40)
    for i, t in enumerate(ts):
        assert np.linalg.norm(psis[:, i] - _dense_exp(Hd, psi0, t)) < 1e-9


def test_timeevolve_controller_counters(ek, O):
    """timeevolve_tests.jl:71-136: reuse, restart and extension paths, and the
    same counters as the restated controller."""
    L = 6
    bond = ek.spin((1.0, "xx"), (1.0, "yy"), (0.7, "zz"))
    obond = O.spin((1.0, "xx"), (1.0, "yy"), (0.7, "zz"))
    H = ek.trans_inv_operator(bond, [1, 2], ek.TensorBasis(L=L))
    Hd = O.trans_inv_operator(obond, [1, 2], O.tensor(L)).dense()
    rng = np.random.default_rng(13)
    psi0 = rng.standard_normal(2 ** L) + 1j * rng.standard_normal(2 ** L)
    psi0 /= np.linalg.norm(psi0)
    ts = np.linspace(0, 0.4, 25)
    _, d = ek.timeevolve(H, psi0, ts, tol=1e-10, m_init=25, m_max=50, return_diagnostics=True)
    assert d.basis_builds == 1 and d.restarts == 0 and d.matvecs <= d.max_dim_used
    ts = np.linspace(0, 3.0, 15)
    psis, d = ek.timeevolve(H, psi0, ts, tol=1e-12, m_init=5, m_max=40, extend_step=5,
                            return_diagnostics=True)
    _, od = O.timeevolve(lambda v: Hd @ v, psi0, ts, tol=1e-12, m_init=5, m_max=40,
                         extend_step=5)
    assert d.basis_extensions >= 1
    assert d.basis_extensions == od["basis_extensions"] and d.matvecs == od["matvecs"]
    for i, t in enumerate(ts):
        assert np.linalg.norm(psis[:, i] - _dense_exp(Hd, psi0, t)) < 1e-9
    L = 8
    H = ek.trans_inv_operator(bond, [1, 2], ek.TensorBasis(L=L))
    Hd = O.trans_inv_operator(obond, [1, 2], O.tensor(L)).dense()
    psi0 = rng.standard_normal(2 ** L) + 1j * rng.standard_normal(2 ** L)
    psi0 /= np.linalg.norm(psi0)
    ts = np.linspace(0, 20, 11)
    psis, d = ek.timeevolve(H, psi0, ts, tol=1e-10, m_init=6, m_max=6, extend_basis=False,
                            return_diagnostics=True)
    for i, t in enumerate(ts):
        assert np.linalg.norm(psis[:, i] - _dense_exp(Hd, psi0, t)) < 1e-6
    assert d.restarts >= 1 and d.basis_builds >= 2


def test_timeevolve_order_and_errors(ek):
    """timeevolve_tests.jl:166-201: unsorted ts keep caller order; negative
    times and zero-norm states are rejected."""
    L = 6
    bond = ek.spin((1.0, "xx"), (1.0, "yy"), (0.7, "zz"))
    H = ek.trans_inv_operator(bond, [1, 2], ek.TensorBasis(L=L))
    rng = np.random.default_rng(14)
    psi0 = rng.standard_normal(2 ** L) + 1j * rng.standard_normal(2 ** L)
    psi0 /= np.linalg.norm(psi0)
    ts = np.linspace(0, 2, 9)
    a = ek.timeevolve(H, psi0, ts, tol=1e-12, m_init=20, m_max=40)
    perm = [4, 0, 8, 2, 6, 1, 7, 3, 5]
    bsh = ek.timeevolve(H, psi0, ts[perm], tol=1e-12, m_init=20, m_max=40)
    for j, p in enumerate(perm):
        assert np.allclose(bsh[:, j], a[:, p], atol=1e-10)
    with pytest.raises(ValueError):
        ek.timeevolve(H, psi0, -0.3)
    with pytest.raises(ValueError):
        ek.timeevolve(H, psi0, [-0.1, 0.3])
    with pytest.raises(ek.EDKError, match="zero norm"):
        ek.timeevolve(H, np.zeros(2 ** L, complex), 1.0)


def test_timeevolve_mixed_precision_fidelity(ek):
    L = 16
    b = ek.TranslationalBasis(L=L, k=0, N=8)
    H = ek.trans_inv_operator(ek.spin((1.0, "xx"), (1.0, "yy"), (1.0, "zz")), 2, b)
    rng = np.random.default_rng(15)
    psi0 = rng.standard_normal(b.size(1)) + 1j * rng.standard_normal(b.size(1))
    psi0 /= np.linalg.norm(psi0)
    ts = np.linspace(0, 2, 11)
    a = ek.timeevolve(H, psi0, ts, tol=1e-10)
    m = ek.timeevolve(H, psi0, ts, tol=1e-10, precision="mixed")
    for i in range(len(ts)):
        fid = abs(np.vdot(a[:, i], m[:, i])) ** 2
        assert 1 - fid < 1e-8


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_ground_state_vector(ek, O, precision):
    """The returned ground state is normalised, satisfies H psi = E0 psi to the
    residual the eigenvalue allows, and matches the dense eigenvector up to a
    phase — on the batched path (translation sector, complex and real), the
    dedicated-basis path and the generic path (AbelianBasis)."""
    L = 14
    cases = [
        ek.trans_inv_operator(xxz(ek.spin, 1.0), 2, ek.TranslationalBasis(L=L, N=7, k=0)),
        ek.trans_inv_operator(xxz(ek.spin, 1.0), 2, ek.TranslationalBasis(L=L, N=7, k=3)),
        ek.trans_inv_operator(xxz(ek.spin, 1.0), 2, ek.basis(L=L, N=7, k=0, p=1)),
    ]
    for H in cases:
        e0, psi, info = ek.ground_state(H, m=200, tol=1e-13, precision=precision)
        assert abs(np.linalg.norm(psi) - 1) < 1e-12
        r = H * psi - e0 * psi
        assert np.linalg.norm(r) < 1e-6
        M = H.todense()
        w, Vd = np.linalg.eigh(M)
        assert abs(e0 - w[0]) < 1e-10 * abs(w[0])
        assert abs(abs(np.vdot(Vd[:, 0], psi)) - 1) < 1e-9
