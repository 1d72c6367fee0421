"""Failure detection without a GPU fault: bad inputs come back as statuses
with messages, an allocation the device cannot hold comes back as EDK_OOM,
and a bounded device wait that runs out comes back as EDK_TIMEOUT — each
time the context stays usable for the next call.

The reference raises Julia errors for the zero-norm case ("Initial state has
zero norm", TimeEvolution.jl:188); it has no check for non-finite entries,
which these solvers refuse instead of returning NaN eigenvalues."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _xxz(ek, L=12, N=6):
    b = ek.TranslationalBasis(L=L, k=0, N=N)
    return b, ek.trans_inv_operator(ek.spin((1.0, "xx"), (1.0, "yy"), (1.0, "zz")), 2, b)


def _still_works(ek, O, H, L=12, N=6):
    Ho = O.trans_inv_operator(O.spin((1.0, "xx"), (1.0, "yy"), (1.0, "zz")), 2,
                              O.translational(L, k=0, N=N))
    x = np.random.default_rng(5).standard_normal(H.size(1))
    y = H * x
    yo = Ho.mul(x).real.ravel()
    assert np.linalg.norm(y - yo) <= 1e-12 * np.linalg.norm(yo)


def test_non_finite_start_vectors_are_refused(ek, O):
    from edkit_b200 import _lib as E
    b, H = _xxz(ek)
    D = b.size(1)
    v = np.random.default_rng(1).standard_normal(D)
    for bad in (np.nan, np.inf):
        w = v.copy()
        w[D // 2] = bad
        with pytest.raises(ek.EDKError, match="non-finite") as e:
            ek.lanczos_e0(H, w, m=20)
        assert e.value.status == E.INVALID_ARG
        with pytest.raises(ek.EDKError, match="non-finite"):
            ek.lanczos_e0(H, w, m=20, precision="mixed")
        with pytest.raises(ek.EDKError, match="non-finite"):
            ek.batch_lanczos_e0([H, H], [v, w], m=20)
        with pytest.raises(ek.EDKError, match="non-finite"):
            ek.ground_state(H, w, m=20)
        with pytest.raises(ek.EDKError, match="non-finite"):
            ek.timeevolve(H, w.astype(np.complex128), [0.1, 0.2])
    with pytest.raises(ek.EDKError, match="zero norm"):
        ek.batch_lanczos_e0([H, H], [v, np.zeros(D)], m=20)
    _still_works(ek, O, H)


def test_oversized_request_is_oom_and_the_context_survives(ek, O):
    """A Krylov basis of 12,001 complex vectors of the L=28, N=14, k=0 sector
    (1,432,860 rows) needs 275 GB: more than the device holds."""
    from edkit_b200 import _lib as E
    b = ek.TranslationalBasis(L=28, k=0, N=14)
    Hb = ek.trans_inv_operator(ek.spin((1.0, "xx"), (1.0, "yy"), (1.0, "zz")), 2, b)
    psi0 = np.zeros(b.size(1), np.complex128)
    psi0[0] = 1.0
    with pytest.raises(ek.EDKError, match="out of memory") as e:
        ek.KrylovEvolutionCache(Hb, psi0, m_init=10, m_max=12000)
    assert e.value.status == E.OOM
    # the device and the library keep working: the same operator, a small basis
    psi = ek.timeevolve(Hb, psi0, 0.05, m_init=10, m_max=20)
    assert abs(np.linalg.norm(psi) - 1.0) < 1e-10
    _, H = _xxz(ek)
    _still_works(ek, O, H)


def test_bounded_wait_runs_out_and_reports_timeout(ek, O):
    from edkit_b200 import _lib as E
    lib = E.load()
    for polls in (1, 1000, 100000):
        assert lib.edk_selftest_bounded_wait(polls) == E.TIMEOUT
        msg = lib.edk_last_error().decode()
        assert "bounded wait ran out" in msg and str(polls) in msg
    assert lib.edk_selftest_bounded_wait(0) == E.INVALID_ARG
    _, H = _xxz(ek)
    _still_works(ek, O, H)
