"""Eigenvector post-processing: Schmidt matrices, entanglement spectra and
entropies of sector vectors, and maps between two bases of one chain.

Mirrors src/Schmidt.jl (``schmidt``, ``ent_spec``, ``entropy``, ``ent_S``) and
src/LinearMap.jl (``DoubleBasis``, ``symmetrizer``) with the reference's names,
keyword arguments and error messages.  The work runs in libedk
(edk_schmidt.cu): the Schmidt matrix and the DoubleBasis map are CUDA kernels,
the singular values come from a Gram matrix (cuBLAS) and a dense Hermitian
eigensolver (cuSOLVER).  Vectors may be numpy arrays (host) or CUDA torch
tensors (device); results of ``schmidt`` and ``DoubleBasis`` come back on the
side the input came from.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as E
from .basis import AbstractBasis, TensorBasis


def _vec(v):
    """(pointer, edk dtype, ptr kind, keep-alive, is_torch, device) of a vector."""
    if hasattr(v, "data_ptr"):
        import torch
        if v.dtype not in (torch.float64, torch.complex128):
            raise TypeError("vectors must be float64 or complex128")
        v = v.contiguous()
        kind = E.DEVICE if v.is_cuda else E.HOST
        return (E.ptr(v), E.C128 if v.is_complex() else E.F64, kind, v, True,
                v.device)
    a = np.asarray(v)
    a = np.ascontiguousarray(a, dtype=np.complex128 if np.iscomplexobj(a) else np.float64)
    return E.ptr(a), (E.C128 if np.iscomplexobj(a) else E.F64), E.HOST, a, False, None


def _sites(Ainds, L):
    a = np.ascontiguousarray([int(i) for i in Ainds], dtype=np.int32)
    return a, len(a)


def _basis_complex(b):
    return bool(getattr(b, "_complex", False))


def schmidt(v, Ainds, b: AbstractBasis):
    """schmidt(v, Ainds, b) — Schmidt.jl:186-336 / AbelianBasis.jl:704-719:
    the matrix S with |v> = S_ij |A_i>|B_j>, shape 2^|A| x 2^(L-|A|)."""
    if len(v) != b.size(1):
        raise ValueError(f"Expected a vector of length {b.size(1)}; got {len(v)}.")
    p, dt, kind, keep, is_t, dev = _vec(v)
    a, nA = _sites(Ainds, b.L)
    cm = dt == E.C128 or _basis_complex(b)
    shape_f = (2 ** nA, 2 ** (b.L - nA))
    if is_t and kind == E.DEVICE:
        import torch
        # column-major dA x dB == row-major dB x dA; return its transpose view
        M = torch.empty(shape_f[1], shape_f[0], dtype=torch.complex128 if cm else torch.float64,
                        device=dev)
        E.check(E.load().edk_schmidt(b._h, dt, p, nA, E.ptr(a), E.ptr(M),
                                     E.C128 if cm else E.F64, E.DEVICE))
        return M.T
    M = np.zeros(shape_f, dtype=np.complex128 if cm else np.float64, order="F")
    E.check(E.load().edk_schmidt(b._h, dt, p, nA, E.ptr(a), E.ptr(M), E.C128 if cm else E.F64,
                                 kind))
    return M


def ent_spec(v, Aind, b: AbstractBasis):
    """ent_spec(v, Aind, b) — Schmidt.jl:84: Schmidt singular values, descending."""
    if len(v) != b.size(1):
        raise ValueError(f"Expected a vector of length {b.size(1)}; got {len(v)}.")
    p, dt, kind, keep, _, _ = _vec(v)
    a, nA = _sites(Aind, b.L)
    n = C.c_int64()
    lib = E.load()
    s = np.zeros(2 ** min(nA, b.L - nA))
    E.check(lib.edk_ent_spec(b._h, dt, p, nA, E.ptr(a), E.ptr(s), C.byref(n), kind))
    return s[:n.value]


def entropy(s, alpha=1, cutoff=1e-20):
    """entropy(s; α, cutoff) — Schmidt.jl:101-139 (host arithmetic on the
    given probabilities, sorted as passed)."""
    if alpha == 1:
        ent = 0.0
        for si in s:
            if not si > cutoff:
                break
            ent -= si * np.log(si)
        return float(ent)
    if alpha == 0:
        n = 0
        for si in s:
            if not si > cutoff:
                break
            n += 1
        return n
    return float(np.log(np.sum(np.asarray(s, dtype=np.float64) ** alpha)) / (1 - alpha))


def ent_S(v, Aind, b, alpha=1, cutoff=1e-20):
    """ent_S(v, Aind, b; α=1, cutoff=1e-20) — Schmidt.jl:150-165.  `b` may be a
    basis or the chain length L (a TensorBasis is inferred from len(v))."""
    if isinstance(b, (int, np.integer)):
        L = int(b)
        base = int(round(len(v) ** (1.0 / L)))
        b = TensorBasis(L=L, base=base)
    if len(v) != b.size(1):
        raise ValueError(f"Expected a vector of length {b.size(1)}; got {len(v)}.")
    p, dt, kind, keep, _, _ = _vec(v)
    a, nA = _sites(Aind, b.L)
    S = C.c_double()
    E.check(E.load().edk_ent_S(b._h, dt, p, nA, E.ptr(a), float(alpha), float(cutoff),
                               C.byref(S), kind))
    return int(S.value) if alpha == 0 else float(S.value)


class DoubleBasis:
    """DoubleBasis(B1, B2) — LinearMap.jl:88-126: the map from coordinates in
    the source basis B2 to coordinates in the target basis B1."""

    def __init__(self, B1: AbstractBasis, B2: AbstractBasis):
        if len(B1) != len(B2):  # check_doublebasis_compatible, LinearMap.jl:38-42
            raise ValueError("DoubleBasis requires bases with the same length.")
        if B1.B != B2.B:
            raise ValueError("DoubleBasis requires bases with the same local base.")
        self.B1, self.B2, self.B = B1, B2, B2.B
        self.dgt = B1.dgt

    def size(self, dim=None):
        s = (self.B1.size(1), self.B2.size(2))
        return s if dim is None else (s[dim - 1] if dim in (1, 2) else 1)

    def __len__(self):
        return len(self.B1)

    def __call__(self, v):
        """(B::DoubleBasis)(v) — LinearMap.jl:140-166."""
        if len(v) != self.size(2):
            raise ValueError(f"Expected a vector of length {self.size(2)}; got {len(v)}.")
        p, dt, kind, keep, is_t, dev = _vec(v)
        if is_t and kind == E.DEVICE:
            import torch
            out = torch.empty(self.size(1), dtype=torch.complex128, device=dev)
        else:
            out = np.zeros(self.size(1), dtype=np.complex128)
        E.check(E.load().edk_double_basis_apply(self.B1._h, self.B2._h, dt, p, E.ptr(out),
                                                kind))
        return out


def symmetrizer(B: DoubleBasis):
    """symmetrizer(B) — LinearMap.jl:183-185: basis_embedding(B1)' *
    basis_embedding(B2), a dense complex size(B1) x size(B2) matrix."""
    M = np.zeros(B.size(), dtype=np.complex128, order="F")
    E.check(E.load().edk_symmetrizer(B.B1._h, B.B2._h, E.ptr(M), E.HOST))
    return M
