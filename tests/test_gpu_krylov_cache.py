"""The resumable Krylov propagator (KrylovEvolutionCache + timeevolve!,
TimeEvolution.jl:166-218, 586-636): a cache advanced across calls gives the
states of the one-shot timeevolve on the same times, keeps its basis,
anchor and diagnostics between calls, and refuses backward times with the
reference's messages (timeevolve_tests.jl covers the same behaviour)."""
import numpy as np
import pytest
from scipy.linalg import expm

pytestmark = pytest.mark.gpu


def _setup(ek, O, L=12):
    bond = ek.spin((1.0, "xx"), (1.0, "yy"), (0.7, "zz"))
    b = ek.TranslationalBasis(L=L, k=0, N=L // 2)
    H = ek.trans_inv_operator(bond, [1, 2], b)
    Hd = O.trans_inv_operator(O.spin((1.0, "xx"), (1.0, "yy"), (0.7, "zz")), [1, 2],
                              O.translational(L, k=0, N=L // 2)).dense()
    rng = np.random.default_rng(31)
    psi0 = rng.standard_normal(b.size(1)) + 1j * rng.standard_normal(b.size(1))
    psi0 /= np.linalg.norm(psi0)
    return H, Hd, psi0


def test_cache_matches_one_shot_and_dense(ek, O):
    H, Hd, psi0 = _setup(ek, O)
    ts = np.linspace(0.0, 6.0, 13)
    kw = dict(tol=1e-12, m_init=6, m_max=12, extend_step=3)
    ref, dref = ek.timeevolve(H, psi0, ts, return_diagnostics=True, **kw)
    cache = ek.KrylovEvolutionCache(H, psi0, **kw)
    assert cache.m == 6 and cache.t_anchor == 0.0
    # one time per call, then the rest as a forward sequence in one call
    cols = [cache.timeevolve_(t) for t in ts[:5]]
    rest = cache.timeevolve_(ts[5:])
    got = np.column_stack(cols + [rest[:, q] for q in range(rest.shape[1])])
    assert np.array_equal(got, ref)  # the same controller decisions, the same arithmetic
    d = cache.diagnostics
    for k in ("basis_builds", "basis_extensions", "restarts", "matvecs", "total_times_served",
              "max_dim_used"):
        assert d[k] == dref[k], k
    assert d.restarts >= 1 and cache.t_anchor > 0.0 and cache.t_latest == ts[-1]
    for q, t in enumerate(ts):
        assert np.linalg.norm(got[:, q] - expm(-1j * t * Hd) @ psi0) < 1e-9


def test_cache_forward_only_and_reuse(ek, O):
    H, Hd, psi0 = _setup(ek, O)
    cache = ek.KrylovEvolutionCache(H, psi0, tol=1e-10, m_init=20, m_max=40)
    a = cache.timeevolve_(0.4)
    builds = cache.diagnostics.basis_builds
    b = cache.timeevolve_(0.4)  # the same time again is allowed (not before the last)
    assert np.array_equal(a, b)
    cache.timeevolve_(0.5)
    assert cache.diagnostics.basis_builds == builds  # served from the same basis
    with pytest.raises(ek.EDKError, match="precedes the last served time"):
        cache.timeevolve_(0.3)
    with pytest.raises(ek.EDKError, match="sorted in ascending order"):
        cache.timeevolve_([0.7, 0.6])
    assert cache.t_latest == 0.5  # a refused call changes nothing
    c = cache.timeevolve_([0.6, 0.9])
    for q, t in enumerate((0.6, 0.9)):
        assert np.linalg.norm(c[:, q] - expm(-1j * t * Hd) @ psi0) < 1e-8


def test_cache_device_states_and_bad_start(ek, O):
    import torch
    H, Hd, psi0 = _setup(ek, O)
    cache = ek.KrylovEvolutionCache(H, torch.from_numpy(psi0).cuda(), tol=1e-11,
                                    m_init=20, m_max=40)
    out = cache.timeevolve_([0.2, 1.1])
    assert out.is_cuda
    for q, t in enumerate((0.2, 1.1)):
        assert np.linalg.norm(out[:, q].cpu().numpy() - expm(-1j * t * Hd) @ psi0) < 1e-9
    with pytest.raises(ek.EDKError, match="zero norm"):
        ek.KrylovEvolutionCache(H, np.zeros_like(psi0))
    bad = psi0.copy()
    bad[3] = np.nan
    with pytest.raises(ek.EDKError, match="non-finite"):
        ek.KrylovEvolutionCache(H, bad)
    with pytest.raises(ek.EDKError, match="m_max must be"):
        ek.KrylovEvolutionCache(H, psi0, m_init=10, m_max=5)
