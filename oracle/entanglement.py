"""CPU oracle for eigenvector post-processing — TEST INFRASTRUCTURE ONLY.

Plain-Python restatements (small L only) of
  * ``schmidt`` for every basis type   src/Schmidt.jl:186-336,
                                       src/Basis/AbelianBasis.jl:704-719
  * ``ent_spec`` / ``entropy`` / ``ent_S``  src/Schmidt.jl:84-165
  * ``(B::DoubleBasis)(v)`` and ``symmetrizer``  src/LinearMap.jl:57-70, 140-185
following the reference's loops literally: digit vectors, ``circshift!`` by
the unit cell, ``reverse!`` / ``spinflip``, running products of the phase.
The bases are the oracle's own (``oracle.tensor`` ... ``oracle.abelian`` and
the dedicated ``parity_basis`` ... ``transflip_basis``), whose tables are
pinned separately.  Only tests and the bench's CPU legs import this module.
"""
from __future__ import annotations

import math

import numpy as np

from . import (KIND_ABELIAN, KIND_PROJECTED, KIND_TENSOR, KIND_TRANS, KIND_TRANSPAR,
               DedicatedBasis, OBasis)


def _state(dgt):
    s = 0
    for d in dgt:
        s = 2 * s + int(d)
    return s


def _dgt(s, L):
    return [(s >> (L - 1 - q)) & 1 for q in range(L)]


class _Schmidt:
    """SchmidtMatrix + schmidtmatrix/addto! (Schmidt.jl:16-71) with TensorBasis
    subsystem bases: row index = A digits big-endian in Ainds order, column
    index = the remaining sites ascending."""

    def __init__(self, L, Ainds, dtype):
        self.A = [int(i) for i in Ainds]
        self.B = [i for i in range(1, L + 1) if i not in self.A]
        self.M = np.zeros((2 ** len(self.A), 2 ** len(self.B)), dtype=dtype)

    def addto(self, dgt, val):
        ia = _state([dgt[i - 1] for i in self.A])
        ib = _state([dgt[i - 1] for i in self.B])
        self.M[ia, ib] += val


def _circshift(dgt, a):  # Julia circshift!(dgt, a): element i moves to i + a
    return dgt[-a:] + dgt[:-a]


def _abelian_phases(order, q):  # AbelianOperator, AbelianBasis.jl:167-176
    if q == 0:
        return [1.0] * order
    if 2 * q == order:
        return [1.0 if j % 2 == 0 else -1.0 for j in range(order)]
    return [complex(math.cos(2 * math.pi * q / order * j), math.sin(2 * math.pi * q / order * j))
            for j in range(order)]


def _basis_info(b):
    """(kind, L, I 1-based, R) of an oracle basis."""
    if isinstance(b, DedicatedBasis):
        return b.kind, b.L, list(b.I), list(b.R)
    I, R = b.tables()
    kind = {KIND_TENSOR: "tensor", KIND_PROJECTED: "projected", KIND_TRANS: "trans",
            KIND_TRANSPAR: "transpar", KIND_ABELIAN: "abelian"}[b.kind]
    return kind, b.L, list(I), list(R)


def schmidt(v, Ainds, b):
    """schmidt(v, Ainds, b) for every basis type (Schmidt.jl:186-336,
    AbelianBasis.jl:704-719)."""
    kind, L, I, R = _basis_info(b)
    v = np.asarray(v)
    cplx = np.iscomplexobj(v)
    phase_tab = None
    if kind in ("trans", "transpar"):
        phase_tab = b.phase()
        cplx = cplx or np.iscomplexobj(phase_tab) and np.any(np.imag(phase_tab) != 0)
    elif kind == "transflip":
        phase_tab = np.asarray(b.C, dtype=complex)
        cplx = cplx or np.any(np.imag(phase_tab) != 0)
    elif kind == "abelian":
        cplx = cplx or any(not (q == 0 or 2 * q == o) for o, q, _, _ in b.gens)
    if phase_tab is not None and not np.any(np.imag(phase_tab) != 0):
        phase_tab = np.real(phase_tab)
    S = _Schmidt(L, Ainds, np.complex128 if cplx else np.float64)
    for i in range(len(v)):
        dgt = _dgt(I[i] - 1, L)
        if kind in ("tensor", "projected"):  # :186-194
            S.addto(dgt, v[i])
        elif kind == "trans":  # :202-216
            A = b.A
            phase = phase_tab[1] if len(phase_tab) > 1 else phase_tab[0]
            val = v[i] / R[i]
            for _ in range(L // A):
                S.addto(dgt, val)
                dgt = _circshift(dgt, A)
                val *= phase
        elif kind in ("transpar", "transflip"):  # parity_schmidt :249-273
            A, P = b.A, b.P
            phase = phase_tab[1] if len(phase_tab) > 1 else phase_tab[0]
            val = v[i] / R[i]
            for _ in range(L // A):
                S.addto(dgt, val)
                dgt = _circshift(dgt, A)
                val *= phase
            dgt = dgt[::-1] if kind == "transpar" else [1 - d for d in dgt]
            val *= P
            for _ in range(L // A):
                S.addto(dgt, val)
                dgt = _circshift(dgt, A)
                val *= phase
        elif kind == "flip":  # :279-291
            val = v[i] / R[i]
            S.addto(dgt, val)
            S.addto([1 - d for d in dgt], b.P * val)
        elif kind == "parity":  # :296-308
            val = v[i] / R[i]
            S.addto(dgt, val)
            S.addto(dgt[::-1], b.P * val)
        elif kind == "parityflip":  # :313-336
            val = v[i] / R[i]
            S.addto(dgt, val)
            dgt = dgt[::-1]
            val *= b.P
            S.addto(dgt, val)
            dgt = [1 - d for d in dgt]
            val *= b.Z
            S.addto(dgt, val)
            dgt = dgt[::-1]
            val *= b.P
            S.addto(dgt, val)
        elif kind == "abelian":  # AbelianBasis.jl:704-719 with the odometer of :282-289
            gens = b.gens
            cs = [_abelian_phases(o, q) for o, q, _, _ in gens]
            cnt = [0] * len(gens)
            val = v[i] / R[i]
            S.addto(dgt, val)
            order = int(np.prod([g[0] for g in gens]))
            for _ in range(1, order):
                for gi, (o, q, perm, inv) in enumerate(gens):
                    new = list(dgt)
                    for site in range(L):  # apply_perm!: value at site i moves to perm[i]
                        new[perm[site] - 1] = dgt[site]
                    dgt = [1 - d if inv[site] else d for site, d in enumerate(new)]
                    cnt[gi] += 1
                    if cnt[gi] >= o:
                        cnt[gi] = 0
                    else:
                        break
                ph = cs[0][cnt[0]]
                for gi in range(1, len(gens)):
                    ph = ph * cs[gi][cnt[gi]]
                S.addto(dgt, ph * val)
        else:
            raise ValueError(kind)
    return S.M


def ent_spec(v, Ainds, b):  # Schmidt.jl:84
    return np.linalg.svd(schmidt(v, Ainds, b), compute_uv=False)


def entropy(s, alpha=1.0, cutoff=1e-20):  # Schmidt.jl:101-139
    if alpha == 1:
        ent = 0.0
        for si in s:
            if not si > cutoff:
                break
            ent -= si * math.log(si)
        return ent
    if alpha == 0:
        n = 0
        for si in s:
            if not si > cutoff:
                break
            n += 1
        return n
    return math.log(float(np.sum(np.asarray(s) ** alpha))) / (1 - alpha)


def ent_S(v, Ainds, b, alpha=1.0, cutoff=1e-20):  # Schmidt.jl:150-153
    return entropy(ent_spec(v, Ainds, b) ** 2, alpha=alpha, cutoff=cutoff)


# ---------------------------------------------------------------------------
# DoubleBasis (LinearMap.jl)
# ---------------------------------------------------------------------------
def orbit_order(b):
    """orbit_order / order(B) (LinearMap.jl:25 with AbstractBasis.jl:197,
    TranslationalBasis.jl:349, TranslationalParityBasis.jl:241,
    TranslationalFlipBasis.jl:222, ParityBasis.jl:128, FlipBasis.jl:122,
    ParityFlipBasis.jl:152, AbelianBasis.jl:507)."""
    kind, L, _, _ = _basis_info(b)
    return {"tensor": 1, "projected": 1, "trans": L, "transpar": 2 * L, "transflip": 2 * L,
            "parity": 2, "flip": 2, "parityflip": 4}.get(kind) or int(
                np.prod([g[0] for g in b.gens]))


def index_state(b, s):
    """index_nocheck(b, dgt) for the 0-based state s: (coeff, 1-based pos),
    (0, 1) when absent."""
    if isinstance(b, DedicatedBasis):
        return b.index_state(s)
    return b.index(_dgt(s, b.L))


def double_basis_apply(b1, b2, v):  # (B::DoubleBasis)(v), LinearMap.jl:140-166
    L = b1.L
    out = np.zeros(_dim(b1), dtype=np.complex128)
    o1, o2 = orbit_order(b1), orbit_order(b2)
    for j in range(2 ** L):
        c2, p2 = index_state(b2, j)
        if c2 == 0:
            continue
        c1, p1 = index_state(b1, j)
        if c1 == 0:
            continue
        out[p1 - 1] += np.conj(c1 / o1) * (c2 / o2) * v[p2 - 1]
    return out


def basis_embedding(b):  # LinearMap.jl:57-70
    L = b.L
    E = np.zeros((2 ** L, _dim(b)), dtype=np.complex128)
    o = orbit_order(b)
    for j in range(2 ** L):
        c, p = index_state(b, j)
        if c != 0:
            E[j, p - 1] = c / o
    return E


def symmetrizer(b1, b2):  # LinearMap.jl:183-185
    return basis_embedding(b1).conj().T @ basis_embedding(b2)


def _dim(b):
    return b.dim
