"""Operators — the Python mirror of src/Operator.jl.

``operator(mats, inds, B)`` merges repeated site lists and drops all-zero
matrices exactly like Operator.jl:56-78; ``trans_inv_operator`` generates the
translated copies of Operator.jl:102-108; ``spin`` parses EDKit's spin strings
(Operator.jl:470-718).  Application (``H * x``, ``mul_`` = ``mul!``, ``mul``)
runs on the GPU through ``edk_apply``; inputs may be numpy arrays (host) or
CUDA tensors (device pointers, no copies).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib as E
from .basis import AbstractBasis, TensorBasis

# ---------------------------------------------------------------------------
# spin strings — Operator.jl:536-718
# ---------------------------------------------------------------------------


def _spin_coeff(D):
    return np.array([math.sqrt(i * (D - i)) for i in range(1, D)])


def _upper(D, vals):
    m = np.zeros((D, D))
    m[np.arange(D - 1), np.arange(1, D)] = vals
    return m


def _spin_dict(c, D):
    if c == "+":
        return _upper(D, _spin_coeff(D))
    if c == "-":
        return _upper(D, _spin_coeff(D)).T.copy()
    if c == "x":
        sp = _upper(D, _spin_coeff(D) / 2)
        return sp + sp.T
    if c == "y":  # i*Sy, kept real (Operator.jl:584-588)
        sp = _upper(D, _spin_coeff(D) / 2)
        return sp - sp.T
    if c == "z":
        J = (D - 1) / 2
        return np.diag([J - i for i in range(D)])
    if c in ("1", "I"):
        return np.eye(D)
    if D != 2:
        raise AssertionError(f"Invalid spin symbol: {c}.")
    if c == "X":
        return np.array([[0.0, 1.0], [1.0, 0.0]])
    if c == "Y":
        return np.array([[0.0, 1.0], [-1.0, 0.0]])
    if c == "Z":
        return np.array([[1.0, 0.0], [0.0, -1.0]])
    raise ValueError(f"Invalid spin symbol: {c}.")


_SPIN_CACHE: dict = {}


def spin(*args, D=2):
    """spin("xx"), spin(c, "xx") or spin((c1, "xx"), (c2, "yy"), ...)."""
    if len(args) == 1 and isinstance(args[0], str):
        s = args[0]
        if not s:
            raise ValueError("Empty spin string.")
        key = (D, s)
        if key not in _SPIN_CACHE:
            ny = sum(1 for ch in s if ch == "y" or (D == 2 and ch == "Y"))
            raw = _spin_dict(s[0], D)
            for ch in s[1:]:
                raw = np.kron(raw, _spin_dict(ch, D))
            sign = (-1) ** (ny // 2) if ny % 2 == 0 else (-1j) ** ny
            m = sign * raw
            if np.iscomplexobj(m) and not np.any(m.imag):
                m = m.real
            _SPIN_CACHE[key] = m
        return _SPIN_CACHE[key].copy()
    if len(args) == 2 and isinstance(args[1], str) and not isinstance(args[0], tuple):
        return args[0] * spin(args[1], D=D)
    if len(args) == 1 and isinstance(args[0], (list, tuple)) and args[0] and \
            isinstance(args[0][0], tuple):
        args = tuple(args[0])
    tot = None
    for c, s in args:
        m = c * spin(s, D=D)
        tot = m if tot is None else tot + m
    return tot


def σ(*idx):
    """Pauli products σ(0..3) (Operator.jl:502-504)."""
    P = [np.eye(2), np.array([[0, 1], [1, 0]], complex), np.array([[0, -1j], [1j, 0]]),
         np.array([[1, 0], [0, -1]], complex)]
    m = P[idx[0]]
    for i in idx[1:]:
        m = np.kron(m, P[i])
    return m


# ---------------------------------------------------------------------------
# Operator
# ---------------------------------------------------------------------------
def _find_base(a, b):
    if b == 1:
        return a
    for i in range(2, a + 1):
        if i ** b == a:
            return i
    raise ValueError(f"Incompatible dimension: ({a}, {b}).")


def _merge(mats, inds):
    """Drop all-zero matrices, merge repeated site lists (Operator.jl:56-78)."""
    if len(mats) != len(inds):
        raise AssertionError(f"Numbers mismatch: {len(mats)} matrices and {len(inds)} indices.")
    M, I = [], []
    for m, ind in zip(mats, inds):
        m = np.asarray(m.toarray() if hasattr(m, "toarray") else m)
        if not np.any(m):
            continue
        ind = [int(v) for v in (ind if np.ndim(ind) else [ind])]
        if ind in I:
            k = I.index(ind)
            M[k] = M[k] + m
        else:
            I.append(ind)
            M.append(np.array(m, copy=True))
    return M, I


def _vec_dtype(a):
    dt = np.dtype(str(a.dtype).replace("torch.", "")) if hasattr(a, "data_ptr") else a.dtype
    return {np.dtype(np.float64): E.F64, np.dtype(np.complex128): E.C128,
            np.dtype(np.float32): E.F32, np.dtype(np.complex64): E.C64}.get(np.dtype(dt))


class Operator:
    """Operator{Tv,Tb}: merged local terms M[n] on sites I[n] over basis B."""

    def __init__(self, M, I, B: AbstractBasis):
        self.M, self.I, self.B = M, I, B
        lib = E.load()
        nsites, sites, nnz, colptr, rowval, nzval = [], [], [], [], [], []
        for m, ind in zip(M, I):
            m = np.asarray(m, dtype=np.complex128)
            nsites.append(len(ind))
            sites.extend(ind)
            cp = [1]
            for c in range(m.shape[1]):
                rows = np.nonzero(m[:, c])[0]
                rowval.extend(int(r) + 1 for r in rows)
                nzval.extend(m[rows, c])
                cp.append(cp[-1] + len(rows))
            colptr.extend(cp)
            nnz.append(cp[-1] - 1)
        self._arr = arr = (
            np.array(nsites, np.int32), np.array(sites, np.int32), np.array(nnz, np.int64),
            np.array(colptr, np.int64), np.array(rowval, np.int64),
            np.ascontiguousarray(np.array(nzval, np.complex128)).view(np.float64))
        h = C.c_void_p()
        E.check(lib.edk_operator_create(B._h, len(M), *(E.ptr(a) for a in arr), C.byref(h)))
        self._h = h
        g, cx, nf, ng = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32()
        E.check(lib.edk_operator_info(h, C.byref(g), C.byref(cx), C.byref(nf), C.byref(ng)))
        self.hermitian_gather = bool(g.value)
        self.is_complex = bool(cx.value)
        self.n_families = nf.value
        self.n_generic = ng.value

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                E.load().edk_operator_destroy(h)
            except Exception:
                pass

    # --- shape / type (Operator.jl:30-33) ---
    def size(self, dim=None):
        return self.B.size(dim)

    @property
    def shape(self):
        return self.B.shape

    def __len__(self):
        return len(self.M)

    def eltype(self):
        return np.complex128 if self.is_complex else np.float64

    # --- arithmetic (Operator.jl:118-134) ---
    def __rmul__(self, c):
        if np.isscalar(c):
            return operator([c * m for m in self.M], self.I, self.B)
        return NotImplemented

    def __truediv__(self, c):
        return operator([m / c for m in self.M], self.I, self.B)

    def __add__(self, other):
        if other is None:
            return self
        return operator(self.M + other.M, self.I + other.I, self.B)

    def __radd__(self, other):
        return self if other is None else other.__add__(self)

    def __neg__(self):
        return Operator([-m for m in self.M], self.I, self.B)

    def __sub__(self, other):
        return self + (-other)

    def adjoint(self):
        return operator([np.conj(m).T for m in self.M], self.I, self.B)

    # --- application ---
    def _out_dtype(self, x):
        dt = _vec_dtype(x)
        if dt is None:
            raise TypeError(f"unsupported vector dtype {x.dtype}")
        if self.is_complex:
            dt = {E.F64: E.C128, E.F32: E.C64}.get(dt, dt)
        return dt

    def _apply(self, x, y, accumulate, dt):
        D = self.B.size(1)
        vec = x.ndim == 1
        nvec = 1 if vec else x.shape[1]
        if hasattr(x, "data_ptr"):  # torch tensor (device or host)
            kind = E.DEVICE if x.is_cuda else E.HOST
            assert x.shape[0] == D
            if not vec:  # torch is row-major: require a column-major (transposed) view
                assert x.stride(0) == 1 and y.stride(0) == 1, "need column-major blocks"
            ldx = D if vec else x.stride(1)
            ldy = D if vec else y.stride(1)
        else:
            kind = E.HOST
            ldx = D if vec else x.strides[1] // x.itemsize
            ldy = D if vec else y.strides[1] // y.itemsize
        E.check(E.load().edk_apply(self._h, dt, E.ptr(x), E.ptr(y), nvec, ldx, ldy,
                                   1 if accumulate else 0, kind))
        return y

    def _prep(self, x):
        if hasattr(x, "data_ptr"):
            return x
        x = np.asarray(x)
        if x.dtype.kind in "iub":
            x = x.astype(np.float64)
        dt = self._out_dtype(x)
        npdt = {E.F64: np.float64, E.C128: np.complex128, E.F32: np.float32,
                E.C64: np.complex64}[dt]
        return np.asfortranarray(x.astype(npdt, copy=False))

    def __mul__(self, x):
        """opt * v / opt * m — Operator.jl:372-394 (fresh zeroed output)."""
        if np.isscalar(x):
            return x * self
        x = self._prep(x)
        dt = self._out_dtype(x)
        if hasattr(x, "data_ptr"):
            import torch
            tdt = {E.F64: torch.float64, E.C128: torch.complex128, E.F32: torch.float32,
                   E.C64: torch.complex64}[dt]
            if x.dtype != tdt:
                x = x.to(tdt)
            y = torch.empty_like(x) if x.ndim == 1 else torch.empty(
                (x.shape[1], x.shape[0]), dtype=tdt, device=x.device).t()
        else:
            y = np.zeros_like(x, order="F")
        return self._apply(x, y, False, dt)

    __matmul__ = __mul__

    def sparse_(self):
        """sparse!(opt): cache the expanded matrix on the device (Operator.jl:269-273);
        later products, Lanczos and Krylov runs on this operator use it.
        Returns the number of stored entries."""
        n = C.c_int64()
        E.check(E.load().edk_operator_materialize(self._h, 1, C.byref(n)))
        self.materialized = True
        return int(n.value)

    def clear_sparse_cache_(self):
        """clear_sparse_cache!() for this operator (Operator.jl:283)."""
        E.check(E.load().edk_operator_materialize(self._h, 0, None))
        self.materialized = False

    _KERNELS = {"fast": 0, "generic": 1, "materialized": 2, "materialized_staged": 3}

    def configure_(self, kernel="fast", tps=1, block=None):
        """Pick the matrix-free kernel by hand: "fast" (bond families, `tps`
        threads per state) or "generic"; `block` True/False forces four or
        more right-hand sides through one SpMM or one column at a time (None:
        automatic).  Every choice gives the same product."""
        E.check(E.load().edk_operator_configure(self._h, self._KERNELS[kernel], int(tps),
                                                -1 if block is None else int(bool(block))))

    def autotune_(self, dtype=None, nvec=1, materialize=False):
        """Time every admissible kernel / threads-per-state / index-search
        combination (and the materialised matrix when `materialize`) on this
        operator and keep the fastest.  Returns the choice and every timing."""
        dt = dtype if dtype is not None else (E.C128 if self.is_complex else E.F64)
        r = E.TuneResult()
        E.check(E.load().edk_operator_autotune(self._h, dt, int(nvec),
                                                E.TUNE_MATERIALIZE if materialize else 0,
                                                C.byref(r)))
        names = {v: k for k, v in self._KERNELS.items()}
        srch = {0: "hash", 1: "sorted", 2: "rank"}
        self.materialized = r.kernel in (E.KERNEL_MATERIALIZED, E.KERNEL_MATERIALIZED_STAGED)
        return {"kernel": names[r.kernel], "search": srch[r.search], "tps": r.tps,
                "block": bool(r.block), "ms": r.ms,
                "candidates": [(names[r.cand_kernel[i]], srch[r.cand_search[i]], r.cand_tps[i],
                                r.cand_ms[i]) for i in range(r.ncand)],
                "candidates_block": [bool(r.cand_block[i]) for i in range(r.ncand)]}

    def todense(self):
        """Array(opt) — Operator.jl:171-196 (H times the identity, small D only)."""
        D = self.B.size(1)
        eye = np.asfortranarray(np.eye(D, dtype=np.complex128 if self.is_complex else np.float64))
        return self * eye


def operator(mats, inds=None, B=None):
    """operator(mats, inds, B) and its convenience forms (Operator.jl:56-88, 727-741)."""
    if isinstance(mats, str):
        mat = spin(mats, D=B.B if isinstance(B, AbstractBasis) else 2)
        return operator([mat], [list(inds)], B)
    if isinstance(mats, np.ndarray) and mats.ndim == 2:
        return operator([mats], [list(inds)], B)
    mats = list(mats)
    if inds is None or isinstance(inds, (AbstractBasis, int)):
        B = inds
        inds = [[i] for i in range(1, (B if isinstance(B, int) else B.L) + 1)]
    inds = [[int(i)] if np.isscalar(i) else [int(v) for v in i] for i in inds]
    if isinstance(B, int):
        base = _find_base(np.asarray(mats[0]).shape[0], len(inds[0]))
        B = TensorBasis(L=B, base=base)
    M, I = _merge(mats, inds)
    return Operator(M, I, B)


def trans_inv_operator(mat, ind, B):
    """trans_inv_operator(mat, ind, B) — Operator.jl:102-116, 749-774."""
    if isinstance(mat, str):
        D = B.B if isinstance(B, AbstractBasis) else 2
        if isinstance(ind, AbstractBasis):  # trans_inv_operator(s, basis)
            B = ind
            ind = len(mat)
        mat = spin(mat, D=D)
    mat = np.asarray(mat)
    if isinstance(ind, int):
        ind = list(range(1, ind + 1))
    ind = np.asarray(list(ind), dtype=np.int64)
    if isinstance(B, int):
        base = _find_base(mat.shape[0], len(ind))
        B = TensorBasis(L=B, base=base)
    L = B.L
    inds = [list(np.mod(ind + i, L) + 1) for i in range(-1, L - 1)]
    M, I = _merge([mat] * L, inds)
    return Operator(M, I, B)


def mul_(target, opt: Operator, v):
    """mul!(target, opt, v): accumulates into target (Operator.jl:309-328)."""
    v = opt._prep(v)
    dt = opt._out_dtype(v)
    if not hasattr(target, "data_ptr"):
        if not (target.flags.f_contiguous or target.ndim == 1):
            raise ValueError("target must be column-major")
        if _vec_dtype(target) != dt:
            raise TypeError("target dtype does not match the product dtype")
    return opt._apply(v, target, True, dt)


def mul(opt: Operator, v):
    """mul(opt, v) — Operator.jl:340-370 (same result as opt * v)."""
    return opt * v
