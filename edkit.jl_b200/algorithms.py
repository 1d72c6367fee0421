"""Lanczos ground state, adaptive Krylov exp(-iHt) and the toolkit helpers.

``timeevolve`` mirrors src/algorithms/TimeEvolution.jl:556-649 (keyword names,
defaults, forward-only errors, column order).  ``lanczos_e0`` is the new
ground-state entry built on the same CGS2 Lanczos builder
(TimeEvolution.jl:250-306).  ``gapratio``/``meangapratio``/``productstate``
mirror src/ToolKit.jl:15-37, 103-109.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as E
from .operator import Operator


def _opts(max_steps, nev, tol, check_every, precision, refine_steps, reorth, complex_vectors):
    o = E.LanczosOpts()
    o.max_steps = int(max_steps)
    o.nev = int(nev)
    o.tol = float(tol)
    o.check_every = int(check_every)
    o.precision = {"fp64": E.PREC_FP64, "mixed": E.PREC_MIXED}[precision]
    o.refine_steps = int(refine_steps)
    o.reorth = 1 if reorth else 0
    o.complex_vectors = 1 if complex_vectors else 0
    return o


def _diag_dict(d: E.LanczosDiag):
    return {f: getattr(d, f) for f, _ in d._fields_}


def lanczos_e0(H: Operator, v0=None, *, m=300, nev=1, tol=0.0, check_every=10,
               precision="fp64", refine_steps=20, reorth=True, complex_vectors=False, seed=0,
               return_coeffs=False):
    """Lowest `nev` eigenvalues of Hermitian H by Lanczos with full CGS2
    reorthogonalisation.  `tol` = 0 runs exactly `m` steps; otherwise the run
    stops once the lowest Ritz values change by less than tol (relative)
    between checks.  precision="mixed" stores the Krylov vectors in FP32 and
    refines the ground state in FP64."""
    D = H.size(1)
    if v0 is None:
        v0 = np.random.default_rng(seed).standard_normal(D)
    dt = E.C128 if np.iscomplexobj(v0) else E.F64
    v0 = np.ascontiguousarray(v0, dtype=np.complex128 if dt == E.C128 else np.float64)
    o = _opts(m, nev, tol, check_every, precision, refine_steps, reorth, complex_vectors)
    ev = np.zeros(nev)
    a = np.zeros(m)
    b = np.zeros(m)
    d = E.LanczosDiag()
    E.check(E.load().edk_lanczos_e0(H._h, C.byref(o), E.ptr(v0), dt, E.HOST, E.ptr(ev), E.ptr(a),
                                    E.ptr(b), C.byref(d)))
    info = _diag_dict(d)
    if return_coeffs:
        n = d.steps
        return ev, info, a[:n], b[:n]
    return ev, info


def ground_state(H: Operator, v0=None, *, m=300, tol=1e-12, check_every=10, precision="fp64",
                 refine_steps=20, complex_vectors=False, seed=0):
    """(E0, psi): the lowest eigenvalue and its normalised Lanczos Ritz vector
    (FP64; complex when H or v0 is).  Same run as lanczos_e0."""
    D = H.size(1)
    if v0 is None:
        v0 = np.random.default_rng(seed).standard_normal(D)
    dt = E.C128 if np.iscomplexobj(v0) else E.F64
    v0 = np.ascontiguousarray(v0, dtype=np.complex128 if dt == E.C128 else np.float64)
    cx = H.is_complex or complex_vectors or dt == E.C128
    psi = np.zeros(D, dtype=np.complex128 if cx else np.float64)
    o = _opts(m, 1, tol, check_every, precision, refine_steps, True, complex_vectors)
    ev = np.zeros(1)
    d = E.LanczosDiag()
    E.check(E.load().edk_lanczos_ground_state(H._h, C.byref(o), E.ptr(v0), dt, E.HOST,
                                              E.ptr(ev), E.ptr(psi),
                                              E.C128 if cx else E.F64, C.byref(d)))
    return float(ev[0]), psi, _diag_dict(d)


def batch_lanczos_e0(ops, v0s=None, *, m=200, nev=1, tol=0.0, check_every=10, precision="fp64",
                     refine_steps=20, reorth=True, seed=0):
    """Lanczos over many independent operators (sectors / instances)."""
    rng = np.random.default_rng(seed)
    if v0s is None:
        v0s = [rng.standard_normal(op.size(1)) for op in ops]
    cx = any(np.iscomplexobj(v) for v in v0s)
    cat = np.concatenate([np.asarray(v, np.complex128 if cx else np.float64) for v in v0s])
    o = _opts(m, nev, tol, check_every, precision, refine_steps, reorth, False)
    hs = (C.c_void_p * len(ops))(*[op._h.value for op in ops])
    ev = np.zeros(len(ops) * nev)
    d = E.LanczosDiag()
    E.check(E.load().edk_batch_lanczos_e0(len(ops), hs, C.byref(o), E.ptr(cat),
                                          E.C128 if cx else E.F64, E.ptr(ev), C.byref(d)))
    return ev.reshape(len(ops), nev), _diag_dict(d)


def block_lanczos(ops, x0s=None, *, block=64, m=100, nev=4, tol=0.0, check_every=10,
                  seed=1234):
    """Block Lanczos over many operators, `block` right-hand sides each.

    Returns (evals[nops, nev], info): the lowest `nev` distinct eigenvalues of
    every operator.  x0s: per operator a D x block start block (complex), or
    None for seeded N(0,1) real and imaginary parts drawn on the device."""
    o = E.BlockLanczosOpts()
    E.load().edk_block_lanczos_default_opts(C.byref(o))
    o.block, o.max_steps, o.nev, o.tol, o.check_every, o.seed = block, m, nev, tol, \
        check_every, seed
    x = None
    if x0s is not None:
        x = np.concatenate([np.asarray(a, np.complex128).ravel(order="F") for a in x0s])
    hs = (C.c_void_p * len(ops))(*[op._h.value for op in ops])
    ev = np.zeros(len(ops) * nev)
    d = E.BlockLanczosDiag()
    E.check(E.load().edk_block_lanczos(len(ops), hs, C.byref(o),
                                       E.ptr(x) if x is not None else None, E.ptr(ev),
                                       C.byref(d)))
    info = {k: getattr(d, k) for k, _ in E.BlockLanczosDiag._fields_}
    return ev.reshape(len(ops), nev), info


class KrylovEvolutionDiagnostics(dict):
    def __getattr__(self, k):
        return self[k]


def _krylov_opts(tol, m_init, m_max, extend_step, nsample, bisect_iters, reuse_basis,
                 extend_basis, normalize_output, precision):
    o = E.KrylovOpts()
    E.load().edk_krylov_default_opts(C.byref(o))
    o.tol, o.m_init, o.m_max, o.extend_step = tol, m_init, m_max, extend_step
    o.nsample, o.bisect_iters = nsample, bisect_iters
    o.reuse_basis, o.extend_basis = int(reuse_basis), int(extend_basis)
    o.normalize_output = int(normalize_output)
    o.precision = {"fp64": E.PREC_FP64, "mixed": E.PREC_MIXED}[precision]
    return o


def _krylov_diag(d):
    return KrylovEvolutionDiagnostics(
        basis_builds=d.basis_builds, basis_extensions=d.basis_extensions, restarts=d.restarts,
        matvecs=d.matvecs, total_times_served=d.total_times_served, max_dim_used=d.max_dim_used,
        accepted_intervals=list(d.accepted_intervals[: min(d.n_intervals, 64)]),
        seconds=d.seconds)


class KrylovEvolutionCache:
    """KrylovEvolutionCache(H, ψ0; kwargs...) — TimeEvolution.jl:166-218.

    A resumable propagator: the Lanczos basis, anchor state and diagnostics
    live on the device between calls of ``timeevolve_``, which serves forward
    times only (TimeEvolution.jl:586-636).  ψ0 is a host array or a CUDA
    tensor; states come back the same way."""

    def __init__(self, H: Operator, psi0, *, tol=1e-10, m_init=30, m_max=60, extend_step=10,
                 nsample=13, bisect_iters=12, reuse_basis=True, extend_basis=True,
                 normalize_output=False, precision="fp64"):
        self.H = H
        self.N = H.size(1)
        self._dev = hasattr(psi0, "data_ptr") and getattr(psi0, "is_cuda", False)
        if self._dev:
            import torch
            psi0 = psi0.to(torch.complex128).contiguous()
            self._device = psi0.device
        else:
            psi0 = np.ascontiguousarray(psi0, dtype=np.complex128)
        if psi0.shape[0] != self.N:
            raise ValueError("psi0 has the wrong length")
        o = _krylov_opts(tol, m_init, m_max, extend_step, nsample, bisect_iters, reuse_basis,
                         extend_basis, normalize_output, precision)
        h = C.c_void_p()
        E.check(E.load().edk_krylov_cache_create(H._h, C.byref(o), E.ptr(psi0),
                                                 E.DEVICE if self._dev else E.HOST, C.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            E.load().edk_krylov_cache_destroy(h)
            self._h = None

    def _info(self):
        ta, tl, m = C.c_double(), C.c_double(), C.c_int32()
        d = E.KrylovDiag()
        E.check(E.load().edk_krylov_cache_info(self._h, C.byref(ta), C.byref(tl), C.byref(m),
                                               C.byref(d)))
        return ta.value, tl.value, m.value, d

    @property
    def t_anchor(self):
        return self._info()[0]

    @property
    def t_latest(self):
        return self._info()[1]

    @property
    def m(self):
        return self._info()[2]

    @property
    def diagnostics(self):
        return _krylov_diag(self._info()[3])

    def timeevolve_(self, t):
        """timeevolve!(cache, t) for a time, or timeevolve!(out, cache, ts) for a
        non-decreasing sequence (columns in the order given)."""
        scalar = np.isscalar(t)
        ts = np.ascontiguousarray(np.atleast_1d(np.asarray(t, dtype=np.float64)))
        if self._dev:
            import torch
            out = torch.empty((len(ts), self.N), dtype=torch.complex128, device=self._device)
        else:
            out = np.zeros((self.N, len(ts)), dtype=np.complex128, order="F")
        E.check(E.load().edk_krylov_cache_evolve(self._h, E.ptr(ts), len(ts), E.ptr(out),
                                                 E.DEVICE if self._dev else E.HOST))
        if self._dev:
            out = out.t()
        return out[:, 0] if scalar else out


def timeevolve(H: Operator, psi0, t, *, return_diagnostics=False, tol=1e-10, m_init=30,
               m_max=60, extend_step=10, nsample=13, bisect_iters=12, reuse_basis=True,
               extend_basis=True, normalize_output=False, precision="fp64"):
    """timeevolve(H, ψ0, t) / timeevolve(H, ψ0, ts) — TimeEvolution.jl:556-577."""
    scalar = np.isscalar(t)
    ts = np.atleast_1d(np.asarray(t, dtype=np.float64))
    if scalar and ts[0] < 0:
        raise ValueError(f"timeevolve!: requested time {t} precedes anchor time 0.0")
    if np.any(ts < 0):
        raise ValueError("timeevolve: all times in ts must be non-negative; backward evolution "
                         "is not supported")
    D = H.size(1)
    on_device = hasattr(psi0, "data_ptr") and getattr(psi0, "is_cuda", False)
    if on_device:
        import torch
        psi0 = psi0.to(torch.complex128).contiguous()
    else:
        psi0 = np.ascontiguousarray(psi0, dtype=np.complex128)
    if psi0.shape[0] != D:
        raise ValueError("psi0 has the wrong length")
    o = _krylov_opts(tol, m_init, m_max, extend_step, nsample, bisect_iters, reuse_basis,
                     extend_basis, normalize_output, precision)
    if on_device:  # states stay in HBM: column q of the (D, nts) view is time ts[q]
        out = torch.empty((len(ts), D), dtype=torch.complex128, device=psi0.device)
    else:
        out = np.zeros((D, len(ts)), dtype=np.complex128, order="F")
    d = E.KrylovDiag()
    E.check(E.load().edk_krylov_evolve(H._h, C.byref(o), E.ptr(psi0), E.ptr(ts), len(ts),
                                       E.ptr(out), E.DEVICE if on_device else E.HOST,
                                       C.byref(d)))
    if on_device:
        out = out.t()
    diag = _krylov_diag(d)
    res = out[:, 0] if scalar else out
    return (res, diag) if return_diagnostics else res


def tridiag_eigen(a, b):
    """eigen(SymTridiagonal(a, b)) with the library's host eigensolver."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    m = len(a)
    bb = np.ascontiguousarray(np.asarray(b, dtype=np.float64)[: max(m - 1, 0)])
    if len(bb) == 0:
        bb = np.zeros(1)
    w = np.zeros(m)
    Q = np.zeros((m, m), order="F")
    if E.load().edk_tridiag_eigen(m, E.ptr(a), E.ptr(bb), E.ptr(w), E.ptr(Q)) != 0:
        raise RuntimeError("tridiagonal eigensolver did not converge")
    return w, Q


# ---------------------------------------------------------------------------
# ToolKit.jl
# ---------------------------------------------------------------------------
def gapratio(E_):
    """Adjacent-gap ratios of a sorted spectrum (ToolKit.jl:15-28)."""
    dE = np.diff(np.asarray(E_, dtype=np.float64))
    a, b = dE[:-1], dE[1:]
    r = np.where(a < b, a / np.where(b == 0, 1, b), np.where(a > b, b / np.where(a == 0, 1, a), 1.0))
    return r


def meangapratio(E_):
    """ToolKit.jl:37."""
    return float(np.sum(gapratio(E_)) / (len(E_) - 2))


def productstate(v, B):
    """Unit vector at the position of digit string v in basis B (ToolKit.jl:103-109)."""
    s = np.zeros(B.size(1))
    _, pos = B.index(np.asarray(v, dtype=np.int64))
    s[pos - 1] = 1.0
    return s
