"""Bases — the Python mirror of EDKit's basis constructors.

Names, keyword arguments and conventions follow the Julia reference:
  TensorBasis(L=, base=)                        src/Basis/AbstractBasis.jl:234-238
  ProjectedBasis(L=, f=, N=, base=)             src/Basis/ProjectedBasis.jl:244-260
  TranslationalBasis(L=, f=, k=, N=, a=, base=) src/Basis/TranslationalBasis.jl:235-266
  TranslationParityBasis(L=, f=, k=, p=, N=, a=, base=)
                                                src/Basis/TranslationalParityBasis.jl:141-175
  basis(L=, f=, base=, N=, k=, a=, p=, z=, symmetries=)
                                                src/Basis/AbelianBasis.jl:771-847
Tables are built on the GPU by libedk (``edk_basis_create``).  A predicate
``f`` is evaluated on the host over the candidate states and handed to the
library as a bitmap; ``f`` receives one digit vector (``dgt[0]`` = site 1), or
a 2-D array of digit vectors when ``vectorized=True``.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib as E


def _digits(states, L):
    """0-based integer states -> digit rows (site 1 = most significant)."""
    states = np.asarray(states, dtype=np.uint64)
    sh = np.arange(L - 1, -1, -1, dtype=np.uint64)
    return ((states[:, None] >> sh[None, :]) & np.uint64(1)).astype(np.int64)


def _allow_bitmap(f, L, vectorized):
    n = 1 << L
    words = np.zeros((n + 63) // 64, dtype=np.uint64)
    chunk = 1 << 16
    for s0 in range(0, n, chunk):
        st = np.arange(s0, min(n, s0 + chunk), dtype=np.uint64)
        dg = _digits(st, L)
        if vectorized:
            ok = np.asarray(f(dg), dtype=bool)
        else:
            ok = np.fromiter((bool(f(row)) for row in dg), dtype=bool, count=len(st))
        idx = st[ok]
        np.bitwise_or.at(words, (idx >> np.uint64(6)).astype(np.int64),
                         np.uint64(1) << (idx & np.uint64(63)))
    return words


class AbstractBasis:
    """A basis whose tables live on the device (opaque ``edk_basis`` handle)."""

    kind = -1

    def __init__(self, desc: E.BasisDesc, L, base, keep=(), **info):
        lib = E.load()
        h = C.c_void_p()
        E.check(lib.edk_basis_create(C.byref(desc), C.byref(h)))
        self._h = h
        self._keep = keep
        self.L = L
        self.B = base
        self.dgt = np.zeros(L, dtype=np.int64)
        D = C.c_int64()
        E.check(lib.edk_basis_dim(h, C.byref(D)))
        self._D = int(D.value)
        self._I = None
        self._R = None
        self.__dict__.update(info)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                E.load().edk_basis_destroy(h)
            except Exception:
                pass

    def set_search(self, strategy):
        """Index search of a basis with representatives: "hash" (table),
        "sorted" (binary search over the ascending representatives, as
        EDKit's index() does) or "rank" (translation sectors of fixed N: a
        table over the charge sector indexed by colex rank, read by the
        bond-family row kernel); rows and results are identical."""
        E.check(E.load().edk_basis_set_search(self._h, {"hash": 0, "sorted": 1,
                                                         "rank": 2}[strategy]))

    def get_search(self):
        v = C.c_int32()
        E.check(E.load().edk_basis_get_search(self._h, C.byref(v)))
        return {0: "hash", 1: "sorted", 2: "rank"}[v.value]

    # --- AbstractBasis interface (AbstractBasis.jl:95-176) ---
    def size(self, dim=None):
        return (self._D, self._D) if dim is None else (self._D if dim in (1, 2) else 1)

    def __len__(self):
        return self.L

    @property
    def shape(self):
        return (self._D, self._D)

    def _tables(self):
        if self._I is None:
            I = np.zeros(self._D, dtype=np.int64)
            R = np.zeros(self._D, dtype=np.float64)
            E.check(E.load().edk_basis_export(self._h, E.ptr(I), E.ptr(R)))
            self._I, self._R = I, R
        return self._I, self._R

    @property
    def I(self):
        """Representative 1-based indices, as EDKit's ``b.I``."""
        return self._tables()[0]

    @property
    def R(self):
        """Orbit norms, as EDKit's ``b.R`` (ones for onsite bases)."""
        return self._tables()[1]

    def content(self, i):
        return int(self.I[i - 1])

    def norm(self, i):
        return float(self.R[i - 1])

    def eltype(self):
        return np.float64

    def index(self, dgt=None):
        """index(b, dgt) -> (coefficient, 1-based position); absent -> (0, 1)."""
        d = self.dgt if dgt is None else np.asarray(dgt, dtype=np.int64)
        st = np.array([int("".join(str(int(v)) for v in d), 2)], dtype=np.uint64)
        pos, coeff = self.index_states(st)
        if pos[0] == 0:
            return 0, 1
        c = coeff[0]
        c = c.real if c.imag == 0 else c
        return c, int(pos[0])

    def index_states(self, states):
        """Batched index over 0-based integer states (0 = absent in pos)."""
        st = np.ascontiguousarray(states, dtype=np.uint64)
        pos = np.zeros(len(st), dtype=np.int64)
        coeff = np.zeros(len(st), dtype=np.complex128)
        E.check(E.load().edk_basis_index(self._h, len(st), E.ptr(st), E.ptr(pos), E.ptr(coeff),
                                         E.HOST))
        return pos, coeff

    def change(self, i, dgt=None):
        """change!(b, i[, dgt]) — load state i into dgt, return its norm."""
        d = self.dgt if dgt is None else dgt
        s = self.content(i) - 1
        for q in range(self.L - 1, -1, -1):
            d[q] = s & 1
            s >>= 1
        return self.norm(i)


def _desc(kind, L, base=2, a=1, k=0, p=1, N=None, allow=None):
    d = E.BasisDesc()
    d.kind = kind
    d.L = L
    d.base = base
    d.a = a
    d.k = k
    d.p = p
    d.N = -1 if N is None else int(N)
    d.allow = allow.ctypes.data if allow is not None else None
    return d


class TensorBasis(AbstractBasis):
    kind = E.TENSOR

    def __init__(self, *, L, base=2):
        super().__init__(_desc(E.TENSOR, L, base), L, base)

    @property
    def I(self):
        return np.arange(1, self._D + 1, dtype=np.int64)

    def eltype(self):
        return np.int64


class ProjectedBasis(AbstractBasis):
    kind = E.PROJECTED

    def __init__(self, dtype=None, *, L, f=None, N=None, base=2, vectorized=False, **_):
        allow = _allow_bitmap(f, L, vectorized) if f is not None else None
        super().__init__(_desc(E.PROJECTED, L, base, N=N, allow=allow), L, base, (allow,))

    def eltype(self):
        return np.int64


class TranslationalBasis(AbstractBasis):
    kind = E.TRANSLATIONAL

    def __init__(self, dtype=None, *, L, f=None, k=0, N=None, a=1, base=2, vectorized=False, **_):
        if L % a != 0:
            raise AssertionError(f"Length of unit-cell {a} incompatible with L={L}")
        allow = _allow_bitmap(f, L, vectorized) if f is not None else None
        super().__init__(_desc(E.TRANSLATIONAL, L, base, a=a, k=k, N=N, allow=allow), L, base,
                         (allow,), A=a, k=k)
        length = L // a
        kk = (-k) % length
        self._complex = not (kk == 0 or 2 * kk == length)

    def eltype(self):
        return np.complex128 if self._complex else np.float64


class TranslationParityBasis(AbstractBasis):
    kind = E.TRANSPARITY

    def __init__(self, dtype=None, *, L, f=None, k=0, p=1, N=None, a=1, base=2, vectorized=False,
                 **_):
        if L % a != 0:
            raise AssertionError(f"Length of unit-cell {a} incompatible with L={L}")
        length = L // a
        if not (k % length == 0 or (2 * k) % length == 0):
            raise ValueError(f"Momentum {k} incompatible with parity.")
        if p not in (1, -1):
            raise AssertionError("Invalid parity")
        allow = _allow_bitmap(f, L, vectorized) if f is not None else None
        super().__init__(_desc(E.TRANSPARITY, L, base, a=a, k=k, p=p, N=N, allow=allow), L, base,
                         (allow,), A=a, k=k, P=p)


def _compute_period(perm, inv):
    """Order of a site permutation with inversion flags (AbelianBasis.jl:109-130)."""
    L = len(perm)
    pos = list(range(1, L + 1))
    flipped = [False] * L
    for q in range(1, max(2 * L * L, 100) + 1):
        pos2 = [perm[pos[i] - 1] for i in range(L)]
        fl2 = [flipped[i] ^ bool(inv[pos[i] - 1]) for i in range(L)]
        pos, flipped = pos2, fl2
        if pos == list(range(1, L + 1)) and not any(flipped):
            return q
    raise RuntimeError("Period computation failed")


class AbelianBasis(AbstractBasis):
    kind = E.ABELIAN
    _desc_kind = E.ABELIAN

    def __init__(self, *, L, gens, N=None, f=None, base=2, vectorized=False):
        orders = np.array([g[0] for g in gens], dtype=np.int32)
        qs = np.array([g[1] for g in gens], dtype=np.int32)
        perms = np.ascontiguousarray(np.array([g[2] for g in gens], dtype=np.int32).reshape(-1))
        invs = np.ascontiguousarray(np.array([g[3] for g in gens], dtype=np.uint8).reshape(-1))
        use_gosper = base == 2 and N is not None and 0 <= N <= L
        allow = None
        if not use_gosper:
            num = None if N is None else L * (base - 1) - N
            g = f
            if num is not None:
                if vectorized:
                    g = (lambda d: (d.sum(axis=1) == num) & (np.asarray(f(d), bool) if f else True))
                else:
                    g = (lambda d: (int(np.sum(d)) == num) and (f(d) if f else True))
            if g is not None:
                allow = _allow_bitmap(g, L, vectorized)
        d = _desc(self._desc_kind, L, base, N=N if use_gosper else None, allow=allow)
        d.ngen = len(gens)
        d.gen_order = orders.ctypes.data
        d.gen_q = qs.ctypes.data
        d.gen_perm = perms.ctypes.data
        d.gen_inv = invs.ctypes.data
        super().__init__(d, L, base, (orders, qs, perms, invs, allow))
        self._complex = any(not (q == 0 or 2 * q == o) for o, q, _, _ in gens)
        self.G = gens

    def order(self):
        return int(np.prod([g[0] for g in self.G]))

    def eltype(self):
        return np.complex128 if self._complex else np.float64


def basis(dtype=None, *, L, f=None, base=2, N=None, k=None, a=1, p=None, z=None,
          symmetries=None, threaded=None, vectorized=False):
    """basis(...) — AbelianBasis.jl:771-847 (same dispatch and generator order)."""
    if symmetries is not None and (k is not None or p is not None or z is not None):
        raise ValueError("Cannot specify both `symmetries` and `k`/`p`/`z` keywords")
    gens = []
    if k is not None:
        perm = [((i - a - 1) % L) + 1 for i in range(1, L + 1)]
        gens.append((L // a, k, perm, [0] * L))
    if p is not None:
        gens.append((2, 1 if p == -1 else 0, [L - i + 1 for i in range(1, L + 1)], [0] * L))
    if z is not None:
        gens.append((2, 1 if z == -1 else 0, list(range(1, L + 1)), [1] * L))
    for sym in symmetries or []:
        prm = [int(v) for v in sym[0]]
        q = int(sym[1])
        inv = [int(bool(v)) for v in sym[2]] if len(sym) == 3 else [0] * L
        gens.append((_compute_period(prm, inv), q, prm, inv))
    if not gens:
        if f is None and N is None:
            return TensorBasis(L=L, base=base)
        return ProjectedBasis(L=L, f=f, N=N, base=base, vectorized=vectorized)
    return AbelianBasis(L=L, gens=gens, N=N, f=f, base=base, vectorized=vectorized)


# ---------------------------------------------------------------------------
# The reference's dedicated symmetry bases.  Each is the AbelianBasis of its
# generators — reflection P, spin flip Z, translation T^a — and shares its
# conventions exactly: representative = the orbit minimum, norm
# R = sqrt(|G| * n_stab) (ParityBasis/FlipBasis: sqrt 2, or 2 on a fixed
# point; ParityFlipBasis: 2, 2 sqrt 2, 4; TranslationFlipBasis:
# 2len/sqrt(p) [/sqrt 2]), index coefficient = the character of the first
# group element (in P, Z or T-then-Z order) reaching the minimum times R.
# Their charge N counts zeros, as in the reference (sum(dgt) == L - N), and f
# is honoured together with N.
# ---------------------------------------------------------------------------
def _charge_kwargs(L, N, f, vectorized):
    if N is not None and not 0 <= N <= L:
        raise ValueError(f"N = {N} out of range for L = {L}")
    if f is None:
        return dict(N=None if N is None else L - N)  # set bits on the device path
    if N is None:
        return dict(f=f, vectorized=vectorized)
    num = L - N
    if vectorized:
        return dict(f=lambda d: (d.sum(axis=1) == num) & np.asarray(f(d), bool),
                    vectorized=True)
    return dict(f=lambda d: int(np.sum(d)) == num and bool(f(d)), vectorized=False)


def _reflection(L):
    return (2, None, [L - i + 1 for i in range(1, L + 1)], [0] * L)


def _flip(L):
    return (2, None, list(range(1, L + 1)), [1] * L)


def _z2(gen, sign):
    if sign not in (1, -1):
        raise ValueError("Invalid parity")
    return (gen[0], 1 if sign == -1 else 0, gen[2], gen[3])


class ParityBasis(AbelianBasis):
    """ParityBasis (src/Basis/ParityBasis.jl:14-90, index :109-121): reflection
    parity p = +-1."""

    def __init__(self, dtype=None, *, L, p, f=None, N=None, base=2, vectorized=False, **_):
        if base != 2:
            raise ValueError("the GPU path supports base 2 (spin-1/2) only")
        super().__init__(L=L, gens=[_z2(_reflection(L), p)], **_charge_kwargs(L, N, f, vectorized))
        self.P = p

    def eltype(self):
        return np.float64


class FlipBasis(AbelianBasis):
    """FlipBasis (src/Basis/FlipBasis.jl:40-95, index :105-115): spin-flip
    eigenvalue p = +-1; with N only the half-filled sector (2N = L)."""

    def __init__(self, dtype=None, *, L, p, f=None, N=None, base=2, vectorized=False, **_):
        if base != 2:
            raise ValueError("the GPU path supports base 2 (spin-1/2) only")
        if N is not None and 2 * N != L:
            raise ValueError(f"N = {N} not compatible.")
        super().__init__(L=L, gens=[_z2(_flip(L), p)], **_charge_kwargs(L, N, f, vectorized))
        self.P = p

    def eltype(self):
        return np.float64


class ParityFlipBasis(AbelianBasis):
    """ParityFlipBasis (src/Basis/ParityFlipBasis.jl:37-94, index :104-125):
    reflection parity p and spin flip z, both +-1."""

    def __init__(self, dtype=None, *, L, p, z, f=None, N=None, base=2, vectorized=False, **_):
        if base != 2:
            raise ValueError("the GPU path supports base 2 (spin-1/2) only")
        if N is not None and 2 * N != L:
            raise ValueError(f"N = {N} not compatible.")
        super().__init__(L=L, gens=[_z2(_reflection(L), p), _z2(_flip(L), z)],
                         **_charge_kwargs(L, N, f, vectorized))
        self.P, self.Z = p, z

    def eltype(self):
        return np.float64


class TranslationFlipBasis(AbelianBasis):
    """TranslationFlipBasis (src/Basis/TranslationalFlipBasis.jl:50-156, index
    :172-213): momentum k with unit cell a, spin-flip eigenvalue p; its norms
    are the reference's 2len/sqrt(period) [/sqrt 2] expressions."""

    _desc_kind = E.TRANSFLIP

    def __init__(self, dtype=None, *, L, k=0, p=1, f=None, N=None, a=1, base=2,
                 vectorized=False, **_):
        if base != 2:
            raise ValueError("the GPU path supports base 2 (spin-1/2) only")
        if L % a:
            raise ValueError(f"Length of unit-cell {a} incompatible with L={L}")
        if N is not None and 2 * N != L:
            raise ValueError(f"N = {N} not compatible.")
        # the generator below rotates against the reference's circshift!, so
        # its quantum number is -k (phases exp(-i 2pi k' n / len), k' = mod(-k, len))
        perm = [((i - a - 1) % L) + 1 for i in range(1, L + 1)]
        super().__init__(L=L, gens=[(L // a, (-k) % (L // a), perm, [0] * L), _z2(_flip(L), p)],
                         **_charge_kwargs(L, N, f, vectorized))
        self.K, self.P, self.A = k, p, a


def binomial(n, k):
    return math.comb(n, k)
