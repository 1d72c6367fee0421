"""CPU oracle for the EDKit hot path — TEST INFRASTRUCTURE ONLY.

This package restates the reference algorithms on the CPU so that the CUDA
library can be checked against them.  Only ``tests/``, ``__graft_entry__.smoke``
and ``bench.py``'s CPU legs may import it.  The product library never calls it.

* ``liboracle.so`` (``edk_oracle.cpp``): basis tables, ``index``, column-scatter
  ``mul`` with thread-private outputs, dense ``Array(opt)``.
* this module: ``spin`` strings (src/Operator.jl:470-718), operator term merging
  (src/Operator.jl:56-116), ``basis(...)`` generator assembly
  (src/Basis/AbelianBasis.jl:771-847), the CGS2 Lanczos builder and the adaptive
  Krylov controller (src/algorithms/TimeEvolution.jl:166-649), gap ratios
  (src/ToolKit.jl:15-37) and ``productstate`` (src/ToolKit.jl:103-109).

Parity status: the reference is Julia and Julia is absent here, so the oracle is
pinned by the reference's own known-answer tests (dimensions, Gosper sequences,
the nnz pin, spectral identities against independent dense constructions), not
by running the reference.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

PRED = C.CFUNCTYPE(C.c_int, C.POINTER(C.c_int64), C.c_int, C.c_void_p)


def build():
    """Compile liboracle.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        vp, i64, i32, dp = C.c_void_p, C.c_int64, C.c_int, C.POINTER(C.c_double)
        L.orc_last_error.restype = C.c_char_p
        L.orc_tensor.restype = vp
        L.orc_tensor.argtypes = [i32, i32]
        L.orc_projected.restype = vp
        L.orc_projected.argtypes = [i32, i32, i32, PRED, vp, i32, i32]
        L.orc_translational.restype = vp
        L.orc_translational.argtypes = [i32, i32, i32, i32, i32, PRED, vp, i32, i32]
        L.orc_transparity.restype = vp
        L.orc_transparity.argtypes = [i32, i32, i32, i32, i32, i32, PRED, vp, i32, i32]
        L.orc_abelian.restype = vp
        L.orc_abelian.argtypes = [i32, i32, i32, i32, vp, vp, vp, vp, PRED, vp, i32]
        L.orc_free.argtypes = [vp]
        L.orc_dim.restype = i64
        L.orc_dim.argtypes = [vp]
        L.orc_kind.restype = i32
        L.orc_kind.argtypes = [vp]
        L.orc_len.restype = i32
        L.orc_len.argtypes = [vp]
        L.orc_export.argtypes = [vp, vp, vp]
        L.orc_phase.argtypes = [vp, vp]
        L.orc_index.argtypes = [vp, vp, dp, dp, C.POINTER(i64)]
        L.orc_operator_create.restype = vp
        L.orc_operator_create.argtypes = [vp, i32, vp, vp, vp, vp, vp, vp]
        L.orc_operator_free.argtypes = [vp]
        L.orc_mul.argtypes = [vp, vp, vp, i64, i32]
        L.orc_mul_serial.argtypes = [vp, vp, vp, i64]
        L.orc_mul_cols.argtypes = [vp, vp, vp, i64, i64, i64, i32]
        L.orc_dense.argtypes = [vp, vp]
        L.orc_gosper_next.restype = C.c_uint64
        L.orc_gosper_next.argtypes = [C.c_uint64]
        L.orc_apply_perm_benes.restype = C.c_uint64
        L.orc_apply_perm_benes.argtypes = [vp, i32, C.c_uint64]
        L.orc_translational_tables.restype = vp
        L.orc_translational_tables.argtypes = [i32, i32, i32, i32, i64, vp, vp]
        L.orc_trans_judge.argtypes = [i32, i32, i32, i32, i32, i64, vp, vp, vp]
        L.orc_rows_hermitian.argtypes = [vp, i64, vp, vp, vp]
        L.orc_coo.restype = i64
        L.orc_coo.argtypes = [vp, vp, vp, vp]
        L.orc_num_threads.restype = i32
        L.orc_set_threads.argtypes = [i32]
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


# ---------------------------------------------------------------------------
# spin strings — src/Operator.jl:470-718
# ---------------------------------------------------------------------------
def _spin_coeff(D):  # :536
    return np.array([math.sqrt(i * (D - i)) for i in range(1, D)])


def _spin_dict(c, D):  # :617-631
    if c == "+":
        m = np.zeros((D, D)); m[np.arange(D - 1), np.arange(1, D)] = _spin_coeff(D); return m
    if c == "-":
        m = np.zeros((D, D)); m[np.arange(1, D), np.arange(D - 1)] = _spin_coeff(D); return m
    if c in "xy":
        sp = np.zeros((D, D)); sp[np.arange(D - 1), np.arange(1, D)] = _spin_coeff(D) / 2
        return sp + sp.T if c == "x" else sp - sp.T
    if c == "z":
        J = (D - 1) / 2
        return np.diag(np.array([J - i for i in range(D)]))
    if c in "1I":
        return np.eye(D)
    assert D == 2, f"Invalid spin symbol: {c}."
    if c == "X":
        return np.array([[0.0, 1.0], [1.0, 0.0]])
    if c == "Y":
        return np.array([[0.0, 1.0], [-1.0, 0.0]])
    if c == "Z":
        return np.array([[1.0, 0.0], [0.0, -1.0]])
    raise ValueError(f"Invalid spin symbol: {c}.")


def spin(*args, D=2):
    """spin("xx") or spin((c1, "xx"), (c2, "yy"), ...) — Operator.jl:691-718."""
    if len(args) == 1 and isinstance(args[0], str):
        s = args[0]
        ny = sum(1 for ch in s if ch == "y" or (D == 2 and ch == "Y"))
        raw = _spin_dict(s[0], D)
        for ch in s[1:]:
            raw = np.kron(raw, _spin_dict(ch, D))
        sign = (-1) ** (ny // 2) if ny % 2 == 0 else (-1j) ** ny
        return sign * raw
    if len(args) == 2 and not isinstance(args[0], tuple) and isinstance(args[1], str):
        return args[0] * spin(args[1], D=D)
    tot = None
    for c, s in args:
        m = c * spin(s, D=D)
        tot = m if tot is None else tot + m
    return tot


# ---------------------------------------------------------------------------
# Operator construction — Operator.jl:56-116
# ---------------------------------------------------------------------------
def merge_terms(mats, inds):
    """operator(mats, inds, B): drop all-zero matrices, merge equal site lists."""
    M, I = [], []
    for m, ind in zip(mats, inds):
        m = np.asarray(m)
        if not np.any(m):
            continue
        ind = [int(v) for v in ind]
        if ind in I:
            k = I.index(ind)
            M[k] = M[k] + m
        else:
            I.append(ind)
            M.append(m.copy())
    return M, I


def trans_inv_terms(mat, ind, L):
    """trans_inv_operator(mat, ind, B) site lists — Operator.jl:102-108."""
    if isinstance(ind, int):
        ind = list(range(1, ind + 1))
    ind = np.asarray(ind)
    inds = [list(np.mod(ind + i, L) + 1) for i in range(-1, L - 1)]
    return merge_terms([mat] * L, inds)


# ---------------------------------------------------------------------------
# Bases
# ---------------------------------------------------------------------------
KIND_TENSOR, KIND_PROJECTED, KIND_TRANS, KIND_TRANSPAR, KIND_ABELIAN = range(5)


class OBasis:
    def __init__(self, handle, L, base, keep=None):
        if not handle:
            raise RuntimeError(lib().orc_last_error().decode())
        self.h = handle
        self.L = L
        self.base = base
        self._keep = keep

    def __del__(self):
        try:
            lib().orc_free(self.h)
        except Exception:
            pass

    @property
    def kind(self):
        return lib().orc_kind(self.h)

    @property
    def dim(self):
        return int(lib().orc_dim(self.h))

    def tables(self):
        D = self.dim
        I = np.zeros(D, np.int64)
        R = np.zeros(D, np.float64)
        if self.kind == KIND_TENSOR:
            return np.arange(1, D + 1, dtype=np.int64), np.ones(D)
        lib().orc_export(self.h, _ptr(I), _ptr(R))
        if self.kind == KIND_PROJECTED:
            R[:] = 1.0
        return I, R

    def phase(self):
        n = lib().orc_len(self.h)
        C = np.zeros(2 * n)
        lib().orc_phase(self.h, _ptr(C))
        return C[0::2] + 1j * C[1::2]

    def index(self, dgt):
        d = np.ascontiguousarray(dgt, dtype=np.int64)
        re, im, pos = C.c_double(), C.c_double(), C.c_int64()
        lib().orc_index(self.h, _ptr(d), C.byref(re), C.byref(im), C.byref(pos))
        return complex(re.value, im.value), int(pos.value)


def _pred(f):
    if f is None:
        return PRED(), None
    def cb(dgt, L, ud):
        return 1 if f(np.ctypeslib.as_array(dgt, shape=(L,))) else 0
    fn = PRED(cb)
    return fn, fn


def tensor(L, base=2):
    return OBasis(lib().orc_tensor(L, base), L, base)


def projected(L, N=None, f=None, base=2, threaded=True, gosper=True):
    fn, keep = _pred(f)
    h = lib().orc_projected(L, base, -1 if N is None else N, fn, None, int(threaded), int(gosper))
    return OBasis(h, L, base, keep)


def translational(L, k=0, N=None, a=1, f=None, base=2, threaded=True, gosper=True):
    fn, keep = _pred(f)
    h = lib().orc_translational(L, base, k, -1 if N is None else N, a, fn, None,
                                int(threaded), int(gosper))
    ob = OBasis(h, L, base, keep)
    ob.A = a
    return ob


def translational_from_tables(L, I, R, k=0, a=1, base=2):
    """TranslationalBasis over given tables (1-based I, R) — for sectors too
    large to scan here; check the tables with trans_judge."""
    I = np.ascontiguousarray(I, dtype=np.int64)
    R = np.ascontiguousarray(R, dtype=np.float64)
    h = lib().orc_translational_tables(L, base, k, a, len(I), _ptr(I), _ptr(R))
    return OBasis(h, L, base, (I, R))


def trans_judge(L, idx, k=0, N=None, a=1, base=2):
    """The TranslationalBasis judge (TranslationalBasis.jl:94-114) on 1-based
    indices: (accepted, norm) per index."""
    idx = np.ascontiguousarray(idx, dtype=np.int64)
    acc = np.zeros(len(idx), np.uint8)
    R = np.zeros(len(idx), np.float64)
    lib().orc_trans_judge(L, base, k, -1 if N is None else N, a, len(idx), _ptr(idx), _ptr(acc),
                          _ptr(R))
    return acc.astype(bool), R


def transparity(L, k=0, p=1, N=None, a=1, f=None, base=2, threaded=True, gosper=True):
    fn, keep = _pred(f)
    h = lib().orc_transparity(L, base, k, p, -1 if N is None else N, a, fn, None,
                              int(threaded), int(gosper))
    ob = OBasis(h, L, base, keep)
    ob.A, ob.P = a, p
    return ob


def abelian_generators(L, k=None, a=1, p=None, z=None, symmetries=None):
    """Generator list assembled like basis(...) — AbelianBasis.jl:791-834."""
    gens = []  # (order, q, perm, inv)
    if k is not None:
        perm = [((i - a - 1) % L) + 1 for i in range(1, L + 1)]
        gens.append((L // a, k, perm, [0] * L))
    if p is not None:
        gens.append((2, 1 if p == -1 else 0, [L - i + 1 for i in range(1, L + 1)], [0] * L))
    if z is not None:
        gens.append((2, 1 if z == -1 else 0, list(range(1, L + 1)), [1] * L))
    for sym in symmetries or []:
        prm = list(sym[0]); q = sym[1]
        inv = list(sym[2]) if len(sym) == 3 else [0] * L
        gens.append((_compute_period(prm, inv), q, prm, [int(bool(v)) for v in inv]))
    return gens


def _compute_period(perm, inv):  # AbelianBasis.jl:109-130
    L = len(perm)
    pos = list(range(1, L + 1))
    flipped = [False] * L
    for p in range(1, max(2 * L * L, 100) + 1):
        new_pos = [perm[pos[i] - 1] for i in range(L)]
        new_fl = [flipped[i] ^ bool(inv[pos[i] - 1]) for i in range(L)]
        pos, flipped = new_pos, new_fl
        if pos == list(range(1, L + 1)) and not any(flipped):
            return p
    raise RuntimeError("Period computation failed")


def abelian(L, N=None, k=None, a=1, p=None, z=None, symmetries=None, f=None, base=2,
            threaded=True):
    gens = abelian_generators(L, k=k, a=a, p=p, z=z, symmetries=symmetries)
    if not gens:
        raise ValueError("abelian() needs at least one generator")
    orders = np.array([g[0] for g in gens], np.int32)
    ks = np.array([g[1] for g in gens], np.int32)
    perms = np.array([g[2] for g in gens], np.int32).reshape(-1)
    invs = np.array([g[3] for g in gens], np.uint8).reshape(-1)
    fn, keep = _pred(f)
    h = lib().orc_abelian(L, base, -1 if N is None else N, len(gens), _ptr(orders), _ptr(ks),
                          _ptr(perms), _ptr(invs), fn, None, int(threaded))
    ob = OBasis(h, L, base, (keep, orders, ks, perms, invs))
    ob.gens = gens
    return ob


def basis(L, N=None, k=None, a=1, p=None, z=None, symmetries=None, f=None, base=2):
    """basis(...) dispatch — AbelianBasis.jl:771-847."""
    if symmetries is not None and (k is not None or p is not None or z is not None):
        raise ValueError("Cannot specify both `symmetries` and `k`/`p`/`z` keywords")
    if k is None and p is None and z is None and not symmetries:
        if f is None and N is None:
            return tensor(L, base)
        return projected(L, N=N, f=f, base=base)
    return abelian(L, N=N, k=k, a=a, p=p, z=z, symmetries=symmetries, f=f, base=base)


# ---------------------------------------------------------------------------
# Operator application
# ---------------------------------------------------------------------------
# ---------------------------------------------------------------------------
# Dedicated Z2 / translation+flip bases, restated in plain Python from the
# reference (small L only: every one of the base^L states is judged).
# Each returns (I 1-based ascending, R) and an index(state) -> (coeff, pos)
# following the reference's own index function.
# ---------------------------------------------------------------------------
def _dgt(s, L):
    return [(s >> (L - 1 - q)) & 1 for q in range(L)]


def _rev(s, L):  # _int_reverse, AbstractBasis.jl:417-425 (base 2)
    return int(format(s, f"0{L}b")[::-1], 2)


def _bsearch(I, x):  # binary_search, ProjectedBasis.jl:71-81 (0 when absent)
    import bisect
    j = bisect.bisect_left(I, x)
    return j + 1 if j < len(I) and I[j] == x else 0


def _charge_ok(dgt, L, N, f):
    if f is not None and not f(np.array(dgt)):
        return False
    return N is None or sum(dgt) == L - N  # EDKit digit convention


class DedicatedBasis:
    def __init__(self, L, I, R, index_fn, kind, **info):
        self.L, self.I, self.R, self._index = L, I, R, index_fn
        self.dim = len(I)
        self.kind = kind  # "parity" | "flip" | "parityflip" | "transflip"
        for k, v in info.items():
            setattr(self, k, v)

    def index_state(self, s):
        return self._index(self, s)


def parity_basis(L, p, N=None, f=None):
    """ParityBasis: judge ParityBasis.jl:40-57, index :109-121."""
    I, R = [], []
    for s in range(2 ** L):
        dgt = _dgt(s, L)
        if not _charge_ok(dgt, L, N, f):
            continue
        i, In = s + 1, _rev(s, L) + 1
        if In < i:
            continue
        if In == i:
            if p != 1:
                continue
            R.append(2.0)
        else:
            R.append(math.sqrt(2))
        I.append(i)

    def index(b, s):
        Ia, Ib = s + 1, _rev(s, L) + 1
        i, n = (_bsearch(b.I, Ib), p) if Ib < Ia else (_bsearch(b.I, Ia), 1)
        return (0.0, 1) if i == 0 else (n * b.R[i - 1], i)
    return DedicatedBasis(L, I, R, index, "parity", P=p)


def flip_basis(L, p, N=None, f=None):
    """FlipBasis: judge FlipBasis.jl:40-55 (partner MAX - i), index :105-115."""
    MAX = 2 ** L + 1
    I, R = [], []
    for s in range(2 ** L):
        dgt = _dgt(s, L)
        if not _charge_ok(dgt, L, N, f):
            continue
        i = s + 1
        In = MAX - i
        if In < i:
            continue
        if In == i:
            if p != 1:
                continue
            R.append(2.0)
        else:
            R.append(math.sqrt(2))
        I.append(i)

    def index(b, s):
        Ia = s + 1
        Ib = MAX - Ia
        i, n = (_bsearch(b.I, Ib), p) if Ib < Ia else (_bsearch(b.I, Ia), 1)
        return (0.0, 1) if i == 0 else (n * b.R[i - 1], i)
    return DedicatedBasis(L, I, R, index, "flip", P=p)


def parityflip_basis(L, p, z, N=None, f=None):
    """ParityFlipBasis: double_parity_check ParityFlipBasis.jl:37-55 with the
    norm table [2, 2sqrt(2), 0, 4], index :104-125."""
    MAX = 2 ** L + 1
    C = [2.0, 2 * math.sqrt(2), 0.0, 4.0]
    I, R = [], []
    for s in range(2 ** L):
        dgt = _dgt(s, L)
        if not _charge_ok(dgt, L, N, f):
            continue
        i = s + 1
        Ip = _rev(s, L) + 1
        if Ip < i:
            continue
        Iz = MAX - i
        if Iz < i:
            continue
        Ipz = MAX - Ip
        if Ipz < i:
            continue
        n = 1
        if Ip == i:
            if p != 1:
                continue
            n += 1
        if Iz == i:
            if z != 1:
                continue
            n += 1
        if Ipz == i:
            if p * z != 1:
                continue
            n += 1
        I.append(i)
        R.append(C[n - 1])

    def index(b, s):
        I0 = s + 1
        Ip = _rev(s, L) + 1
        Iz = (2 ** L - 1 - s) + 1
        Ipz = (2 ** L - 1 - (Ip - 1)) + 1
        Ir = min(I0, Iz, Ip, Ipz)
        i = _bsearch(b.I, Ir)
        if i == 0:
            return (0.0, 1)
        r = b.R[i - 1]
        if Ir == I0:
            return (r, i)
        if Ir == Ip:
            return (p * r, i)
        if Ir == Iz:
            return (z * r, i)
        return (p * z * r, i)
    return DedicatedBasis(L, I, R, index, "parityflip", P=p, Z=z)


def _phase_factor(k, length):  # TranslationalBasis.jl:277-285
    if k == 0:
        return [1.0] * length
    if 2 * k == length:
        return [1.0 if i % 2 == 0 else -1.0 for i in range(length)]
    return [complex(math.cos(-2 * math.pi / length * k * i), math.sin(-2 * math.pi / length * k * i))
            for i in range(length)]


def transflip_basis(L, k=0, p=1, N=None, a=1, f=None):
    """TranslationFlipBasis: judge TranslationalFlipBasis.jl:50-91 (norms
    vcat(N1, N2), N2 = 2len/sqrt(i), N1 = N2/sqrt 2), index :132-171."""
    length = L // a
    K = (-k) % length
    MAX = 2 ** L + 1
    N2 = [2 * length / math.sqrt(i) for i in range(1, length + 1)]
    N1 = [x / math.sqrt(2) for x in N2]
    Ctab = N1 + N2
    mask = (1 << L) - 1
    I, R = [], []
    for s in range(2 ** L):
        dgt = _dgt(s, L)
        if not _charge_ok(dgt, L, N, f):
            continue
        i = s + 1
        Rr, Qp = length, False
        In = MAX - i
        if In < i:
            continue
        if In == i:
            Qp = True
            if p != 1:
                continue
        ok = True
        st = s
        for n in range(1, length):
            st = ((st >> a) | (st << (L - a))) & mask  # circshift!(dgt, a): digits move right
            In1 = st + 1
            In2 = MAX - In1
            if In1 < i or In2 < i:
                ok = False
                break
            if In2 == i:
                if (p == 1) != ((n * K) // (length // 2) % 2 == 0):
                    ok = False
                    break
                Qp = True
            if In1 == i:
                if (n * K) % length != 0:
                    ok = False
                    break
                Rr = n
                break
        if not ok:
            continue
        I.append(i)
        R.append(Ctab[length + Rr - 1] if Qp else Ctab[Rr - 1])
    Cph = _phase_factor(K, length)

    def index(b, s):  # one loop over rotations, both minima, first strict
        Ia0 = s + 1
        Iam, Rm, Ibm, M = Ia0, 0, (2 ** L - 1 - s) + 1, 0
        st = s
        for i in range(1, length):
            st = ((st >> a) | (st << (L - a))) & mask
            Ia1 = st + 1
            if Ia1 == Ia0:
                break
            if Ia1 < Iam:
                Iam, Rm = Ia1, i
            Ib1 = (2 ** L - 1 - st) + 1
            if Ib1 < Ibm:
                Ibm, M = Ib1, i
        if Ibm < Iam:
            i, n = _bsearch(b.I, Ibm), p * Cph[M]
        else:
            i, n = _bsearch(b.I, Iam), Cph[Rm]
        return (0.0, 1) if i == 0 else (n * b.R[i - 1], i)
    return DedicatedBasis(L, I, R, index, "transflip", P=p, C=Cph, A=a)


class OOperator:
    """Operator{Tv,Tb}: merged local terms + basis (Operator.jl:24-28)."""

    def __init__(self, mats, inds, b: OBasis):
        M, I = merge_terms(mats, inds)
        self.mats, self.inds, self.b = M, I, b
        nsites, sites, nnz, colptr, rowval, nzval = [], [], [], [], [], []
        for m, ind in zip(M, I):
            m = np.asarray(m, dtype=np.complex128)
            nsites.append(len(ind)); sites.extend(ind)
            dim = m.shape[0]
            cp = [1]
            for c in range(dim):
                rows = np.nonzero(m[:, c])[0]
                for r in rows:
                    rowval.append(r + 1); nzval.append(m[r, c])
                cp.append(cp[-1] + len(rows))
            colptr.extend(cp); nnz.append(cp[-1] - 1)
        self._arr = (np.array(nsites, np.int32), np.array(sites, np.int32),
                     np.array(nnz, np.int64), np.array(colptr, np.int64),
                     np.array(rowval, np.int64),
                     np.ascontiguousarray(np.array(nzval, np.complex128)).view(np.float64))
        a = self._arr
        self.h = lib().orc_operator_create(b.h, len(M), _ptr(a[0]), _ptr(a[1]), _ptr(a[2]),
                                           _ptr(a[3]), _ptr(a[4]), _ptr(a[5]))

    def __del__(self):
        try:
            lib().orc_operator_free(self.h)
        except Exception:
            pass

    @property
    def dim(self):
        return self.b.dim

    def mul(self, x, nthreads=0):
        """mul(opt, v) / mul(opt, m): threaded scatter, thread-private outputs."""
        x = np.asarray(x)
        vec = x.ndim == 1
        X = np.asfortranarray(x.reshape(self.dim, -1).astype(np.complex128))
        Y = np.zeros_like(X, order="F")
        lib().orc_mul(self.h, _ptr(X), _ptr(Y), X.shape[1], int(nthreads))
        return Y[:, 0] if vec else Y

    def mul_cols(self, x, j0, j1, nthreads=0):
        """Partial mul(opt, v) over input columns j0..j1 (1-based, inclusive)."""
        X = np.asfortranarray(np.asarray(x).reshape(self.dim, -1).astype(np.complex128))
        Y = np.zeros_like(X, order="F")
        lib().orc_mul_cols(self.h, _ptr(X), _ptr(Y), X.shape[1], int(j0), int(j1), int(nthreads))
        return Y

    def sparse(self):
        """H as a scipy CSR matrix of the entries colmn! scatters (duplicates
        summed, the way the scatter accumulates them)."""
        import scipy.sparse as sp
        n = lib().orc_coo(self.h, None, None, None)
        r = np.zeros(n, np.int64)
        c = np.zeros(n, np.int64)
        v = np.zeros(2 * n, np.float64)
        lib().orc_coo(self.h, _ptr(r), _ptr(c), _ptr(v))
        M = sp.coo_matrix((v[0::2] + 1j * v[1::2], (r - 1, c - 1)),
                          shape=(self.dim, self.dim)).tocsr()
        M.sum_duplicates()
        return M

    def rows_hermitian(self, rows, x):
        """(H*x)[rows] (1-based rows) of a Hermitian operator, each from the
        conjugated column colmn! builds (orc_rows_hermitian)."""
        rows = np.ascontiguousarray(rows, dtype=np.int64)
        X = np.ascontiguousarray(np.asarray(x, dtype=np.complex128))
        Y = np.zeros(len(rows), np.complex128)
        lib().orc_rows_hermitian(self.h, len(rows), _ptr(rows), _ptr(X), _ptr(Y))
        return Y

    def mul_serial(self, x, y=None):
        """mul!(y, opt, x): single-threaded, accumulates into y."""
        x = np.asarray(x)
        vec = x.ndim == 1
        X = np.asfortranarray(x.reshape(self.dim, -1).astype(np.complex128))
        Y = np.zeros_like(X, order="F") if y is None else np.asfortranarray(
            np.asarray(y, np.complex128).reshape(self.dim, -1)).copy()
        lib().orc_mul_serial(self.h, _ptr(X), _ptr(Y), X.shape[1])
        return Y[:, 0] if vec else Y

    def dense(self):
        D = self.dim
        M = np.zeros((D, D), np.complex128, order="F")
        lib().orc_dense(self.h, _ptr(M))
        return M


def operator(mats, inds, b):
    return OOperator(mats, inds, b)


def trans_inv_operator(mat, ind, b):
    M, I = trans_inv_terms(mat, ind, b.L)
    return OOperator(M, I, b)


# ---------------------------------------------------------------------------
# Toolkit — ToolKit.jl
# ---------------------------------------------------------------------------
def gapratio(E):  # :15-28
    dE = np.diff(np.asarray(E, dtype=np.float64))
    r = np.zeros(len(dE) - 1)
    for i in range(len(r)):
        if dE[i] < dE[i + 1]:
            r[i] = dE[i] / dE[i + 1]
        elif dE[i] > dE[i + 1]:
            r[i] = dE[i + 1] / dE[i]
        else:
            r[i] = 1.0
    return r


def meangapratio(E):  # :37
    return float(np.sum(gapratio(E)) / (len(E) - 2))


def productstate(v, b: OBasis):  # :103-109
    s = np.zeros(b.dim)
    _, pos = b.index(np.asarray(v, np.int64))
    s[pos - 1] = 1.0
    return s


# ---------------------------------------------------------------------------
# Lanczos with CGS2 full reorthogonalisation — TimeEvolution.jl:250-306
# ---------------------------------------------------------------------------
def lanczos_build(apply, v1, m, dtype=np.complex128):
    """Run `m` steps of _lanczos_build! from v1 (normalised here).

    Returns (alpha, beta, V, m_used, breakdown).  beta[j] is the coupling
    between v_j and v_{j+1}; on lucky breakdown beta[m_used-1] = 0.
    """
    N = v1.shape[0]
    V = np.zeros((N, m + 1), dtype=dtype)
    V[:, 0] = v1 / np.linalg.norm(v1)
    alpha = np.zeros(m); beta = np.zeros(m)
    for j in range(m):
        vj = V[:, j]
        w = np.asarray(apply(vj), dtype=dtype)
        if j > 0:
            w = w - beta[j - 1] * V[:, j - 1]
        aj = float(np.real(np.vdot(vj, w)))
        alpha[j] = aj
        w = w - aj * vj
        for _ in range(2):
            for i in range(j + 1):
                s = np.vdot(V[:, i], w)
                w = w - s * V[:, i]
        bj = float(np.linalg.norm(w))
        beta[j] = bj
        if bj <= math.sqrt(np.finfo(np.float64).eps) * max(1.0, abs(aj)):
            beta[j] = 0.0
            return alpha[: j + 1], beta[: j + 1], V[:, : j + 2], j + 1, True
        V[:, j + 1] = w * (1.0 / bj)
    return alpha, beta, V, m, False


def tridiag_eigvals(alpha, beta):
    """eigen(SymTridiagonal(alpha, beta[1:m-1])).values — TimeEvolution.jl:311-323."""
    from scipy.linalg import eigh_tridiagonal
    m = len(alpha)
    if m == 1:
        return np.array([alpha[0]])
    return eigh_tridiagonal(alpha, beta[: m - 1], eigvals_only=True)


def tridiag_eigen(alpha, beta):
    from scipy.linalg import eigh_tridiagonal
    m = len(alpha)
    if m == 1:
        return np.array([alpha[0]]), np.ones((1, 1))
    return eigh_tridiagonal(alpha, beta[: m - 1])


def lanczos_build_blas(apply, v1, m, dtype=np.float64):
    """The same m steps with each of the two full sweeps taken as one block
    projection (w -= V (V^H w), through BLAS) instead of one column at a time:
    the same subspace in exact arithmetic, fast enough for sectors of a
    million rows.  Returns (alpha, beta, m_used)."""
    N = v1.shape[0]
    V = np.zeros((m + 1, N), dtype=dtype)  # row j = v_j
    V[0] = v1 / np.linalg.norm(v1)
    alpha = np.zeros(m); beta = np.zeros(m)
    for j in range(m):
        w = np.array(apply(V[j]), dtype=dtype)
        if j > 0:
            w -= beta[j - 1] * V[j - 1]
        aj = float(np.real(np.vdot(V[j], w)))
        alpha[j] = aj
        w -= aj * V[j]
        Vj = V[: j + 1]
        for _ in range(2):
            w -= (Vj.conj() @ w) @ Vj
        bj = float(np.linalg.norm(w))
        beta[j] = bj
        if bj <= math.sqrt(np.finfo(np.float64).eps) * max(1.0, abs(aj)):
            beta[j] = 0.0
            return alpha[: j + 1], beta[: j + 1], j + 1
        V[j + 1] = w * (1.0 / bj)
    return alpha, beta, m


def lanczos_e0(apply, v1, m, nev=1, blas=False):
    """E0 (and the lowest nev Ritz values) after m CGS2 Lanczos steps
    (blas=True: the block-projection form of the same sweeps, real vectors
    when v1 is real)."""
    if blas:
        dt = np.complex128 if np.iscomplexobj(v1) else np.float64
        a, b, _ = lanczos_build_blas(apply, v1, m, dt)
    else:
        a, b, _, mu, _ = lanczos_build(apply, v1, m)
    return tridiag_eigvals(a, b)[:nev], a, b


# ---------------------------------------------------------------------------
# Adaptive Krylov exp(-iHt) — TimeEvolution.jl:166-649
# ---------------------------------------------------------------------------
class KrylovCache:
    def __init__(self, apply, psi0, tol=1e-10, m_init=30, m_max=60, extend_step=10, nsample=13,
                 bisect_iters=12, reuse_basis=True, extend_basis=True, normalize_output=False):
        psi0 = np.asarray(psi0, dtype=np.complex128)
        N = psi0.shape[0]
        if N <= 0:
            raise ValueError("Initial state must be non-empty")
        if m_init < 1:
            raise ValueError("m_init must be ≥ 1")
        if m_max < m_init:
            raise ValueError("m_max must be ≥ m_init")
        m_max = min(m_max, N)
        m_init = min(m_init, m_max)
        if nsample < 2:
            raise ValueError("nsample must be ≥ 2")
        if bisect_iters < 0:
            raise ValueError("bisect_iters must be ≥ 0")
        if extend_step < 1:
            raise ValueError("extend_step must be ≥ 1")
        nrm = float(np.linalg.norm(psi0))
        if not nrm > 0:
            raise ValueError("Initial state has zero norm")
        self.apply, self.N = apply, N
        self.t_anchor = 0.0; self.t_latest = 0.0
        self.psi_anchor = psi0.copy(); self.norm_anchor = nrm
        self.V = np.zeros((N, m_max + 1), np.complex128)
        self.V[:, 0] = self.psi_anchor / nrm
        self.alpha = np.zeros(m_max); self.beta = np.zeros(m_max); self.m = 0
        self.tol, self.m_init, self.m_max = tol, m_init, m_max
        self.extend_step, self.nsample, self.bisect_iters = extend_step, nsample, bisect_iters
        self.reuse_basis, self.extend_basis, self.normalize_output = (
            reuse_basis, extend_basis, normalize_output)
        self.diag = dict(basis_builds=0, basis_extensions=0, restarts=0, matvecs=0,
                         total_times_served=0, max_dim_used=0, accepted_intervals=[])
        self._build(self.m_init)
        self._reduced()
        self.diag["basis_builds"] += 1
        self.diag["max_dim_used"] = max(self.diag["max_dim_used"], self.m)

    def _build(self, m_target):  # _lanczos_build! :250-306
        V, a, b = self.V, self.alpha, self.beta
        m_target = min(int(m_target), self.m_max)
        for j in range(self.m, m_target):
            vj = V[:, j]
            w = np.asarray(self.apply(vj), np.complex128).copy()
            self.diag["matvecs"] += 1
            if j > 0:
                w -= b[j - 1] * V[:, j - 1]
            aj = float(np.real(np.vdot(vj, w)))
            a[j] = aj
            w -= aj * vj
            for _ in range(2):
                for i in range(j + 1):
                    s = np.vdot(V[:, i], w)
                    w -= s * V[:, i]
            bj = float(np.linalg.norm(w))
            b[j] = bj
            if bj <= math.sqrt(np.finfo(np.float64).eps) * max(1.0, abs(aj)):
                self.m = j + 1
                b[j] = 0.0
                return True
            self.m = j + 1
            if j + 1 < V.shape[1]:
                V[:, j + 1] = w * (1.0 / bj)
        return False

    def _reduced(self):  # _build_reduced! :311-323
        lam, Q = tridiag_eigen(self.alpha[: self.m], self.beta[: self.m])
        self.lam, self.Q = lam, Q
        self.Qe1 = Q[0, :].copy(); self.Qem = Q[self.m - 1, :].copy()

    def coeffs(self, tau):  # _reduced_coeffs :329-338
        ph = np.exp(-1j * tau * self.lam) * self.Qe1
        return self.Q @ ph

    def monitor(self, tau):  # _defect_monitor :341-350
        bm = self.beta[self.m - 1]
        if bm == 0:
            return 0.0
        acc = np.sum(self.Qem * np.exp(-1j * tau * self.lam) * self.Qe1)
        return float(abs(bm) * abs(acc))

    def reconstruct(self, tau):  # _reconstruct_state! :352-362
        c = self.coeffs(tau)
        psi = (self.V[:, : self.m] @ c) * self.norm_anchor
        if self.normalize_output:
            n = np.linalg.norm(psi)
            if n > 0:
                psi = psi / n
        return psi

    def _nsample(self, tau_try):  # :383-394
        base_n = self.nsample
        if self.m <= 1:
            return base_n
        om = float(self.lam[-1] - self.lam[0])
        if om <= 0:
            return base_n
        n_nyq = math.ceil(4 * om * tau_try / math.pi) + 1
        return min(max(max(base_n, n_nyq), base_n), 513)

    def _max_valid(self, tau_try):  # :396-429
        if not tau_try > 0:
            return 0.0
        if abs(self.beta[self.m - 1]) <= self.tol:
            return float(tau_try)
        n_eff = self._nsample(tau_try)
        xs = np.linspace(0.0, tau_try, n_eff)
        for k in range(n_eff):
            eta = self.monitor(xs[k])
            if not np.isfinite(eta) or eta > self.tol:
                if k == 0:
                    return 0.0
                lo, hi = float(xs[k - 1]), float(xs[k])
                for _ in range(self.bisect_iters):
                    mid = 0.5 * (lo + hi)
                    if self.monitor(mid) > self.tol:
                        hi = mid
                    else:
                        lo = mid
                return lo
        return float(tau_try)

    def _extend(self):  # :434-447
        if not self.extend_basis or self.m >= self.m_max:
            return False
        old = self.m
        self._build(min(self.m + self.extend_step, self.m_max))
        if self.m > old:
            self._reduced()
            self.diag["basis_extensions"] += 1
            self.diag["max_dim_used"] = max(self.diag["max_dim_used"], self.m)
            return True
        return False

    def _restart(self, tau_valid):  # :449-477
        psi = self.reconstruct(tau_valid)
        self.t_anchor += float(tau_valid)
        self.psi_anchor = psi
        nrm = float(np.linalg.norm(psi))
        if not nrm > 0:
            raise RuntimeError("Restart failed: anchor state has zero norm")
        self.norm_anchor = nrm
        self.alpha[:] = 0; self.beta[:] = 0; self.m = 0
        self.V[:, 0] = psi / nrm
        self._build(self.m_init)
        self._reduced()
        self.diag["basis_builds"] += 1
        self.diag["restarts"] += 1
        self.diag["max_dim_used"] = max(self.diag["max_dim_used"], self.m)

    def ensure(self, tau_target):  # :486-520
        rem = float(tau_target)
        if rem <= 0:
            return
        while True:
            tv = self._max_valid(rem)
            if tv >= rem:
                return
            if self.extend_basis and self.m < self.m_max:
                if self._extend():
                    continue
            if tv <= 0:
                if self.m < self.m_max and self._extend():
                    continue
                raise RuntimeError(f"KrylovEvolutionCache: basis at m={self.m} is not valid at τ=0; "
                                   "consider increasing m_max or loosening tol")
            self.diag["accepted_intervals"].append(tv)
            self._restart(tv)
            rem -= tv

    def evolve_to(self, t):  # timeevolve!(cache, t) :586-597
        tf = float(t)
        if tf < self.t_latest:
            raise RuntimeError("backward evolution is not supported")
        tau = tf - self.t_anchor
        if tau < 0:
            raise RuntimeError("requested time precedes anchor time")
        self.ensure(tau)
        psi = self.reconstruct(tf - self.t_anchor)
        self.t_latest = tf
        self.diag["total_times_served"] += 1
        return psi


def timeevolve(apply, psi0, ts, **kw):
    """timeevolve(H, ψ0, ts) multi-time form — TimeEvolution.jl:563-577."""
    scalar = np.isscalar(ts)
    if scalar:
        if ts < 0:
            raise ValueError("negative time")
        cache = KrylovCache(apply, psi0, **kw)
        return cache.evolve_to(ts), cache.diag
    ts = np.asarray(ts, dtype=np.float64)
    if np.any(ts < 0):
        raise ValueError("timeevolve: all times in ts must be non-negative; backward evolution is not supported")
    cache = KrylovCache(apply, psi0, **kw)
    perm = np.argsort(ts, kind="stable")
    out = np.zeros((cache.N, len(ts)), np.complex128)
    for i, p in enumerate(perm):
        out[:, p] = cache.evolve_to(ts[p])
    return out, cache.diag
