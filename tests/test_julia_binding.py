"""The Julia binding (edkit.jl_b200/julia/EDKitB200.jl) against the C ABI.

Julia is not installed here, so the binding is checked the way it reaches the
library:
  * its structs have the fields, order and widths of the ctypes mirror of
    include/edk.h (CPU);
  * the descriptors it fills for symmetry-group bases — basis(...) with k / p /
    z (an AbelianBasis, AbelianBasis.jl:771-847) and the dedicated
    ParityBasis / FlipBasis / ParityFlipBasis / TranslationFlipBasis — from the
    reference's own fields (the AbelianOperator's orders, phase tables,
    permutations and inversion flags; P, Z, C, A) build bases whose tables and
    index() agree with the oracle (GPU).  gen_q / mom_K below restate the
    binding's functions of the same names."""
import ctypes as C
import math
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
JL = os.path.join(ROOT, "edkit.jl_b200", "julia", "EDKitB200.jl")

_JL_TYPES = {"Int32": C.c_int32, "Int64": C.c_int64, "Float64": C.c_double, "UInt64": C.c_uint64,
             "Ptr{Int32}": C.c_void_p, "Ptr{Int64}": C.c_void_p, "Ptr{Float64}": C.c_void_p,
             "Ptr{UInt8}": C.c_void_p, "Ptr{UInt64}": C.c_void_p}


def _jl_struct(name):
    src = open(JL).read()
    m = re.search(r"(?:mutable )?struct " + name + r"\n(.*?)\n(?:    " + name + r"\(\)|end)", src,
                  re.S)
    assert m, name
    fields = []
    for line in m.group(1).splitlines():
        for part in line.split(";"):
            part = part.strip()
            if "::" not in part:
                continue
            fname, ftype = [x.strip() for x in part.split("::")]
            t = re.match(r"NTuple\{(\d+), (\w+)\}", ftype)
            fields.append((fname, (_JL_TYPES[t.group(2)], int(t.group(1))) if t else
                           (_JL_TYPES[ftype], 1)))
    return fields


@pytest.mark.parametrize("jl,py", [("BasisDesc", "BasisDesc"), ("LanczosOpts", "LanczosOpts"),
                                   ("LanczosDiag", "LanczosDiag"), ("KrylovOpts", "KrylovOpts"),
                                   ("KrylovDiag", "KrylovDiag"),
                                   ("BlockLanczosOpts", "BlockLanczosOpts"),
                                   ("BlockLanczosDiag", "BlockLanczosDiag"),
                                   ("TuneResult", "TuneResult")])
def test_julia_structs_match_the_abi(jl, py):
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "edk_lib_only", os.path.join(ROOT, "edkit.jl_b200", "_lib.py"))
    E = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(E)
    want = getattr(E, py)._fields_
    got = _jl_struct(jl)
    assert [n for n, _ in got] == [n for n, _ in want]
    for (n, (t, cnt)), (_, wt) in zip(got, want):
        if cnt > 1:
            assert C.sizeof(wt) == cnt * C.sizeof(t), n
        else:
            assert C.sizeof(wt) == C.sizeof(t), n


def test_julia_binding_maps_every_symmetry_basis():
    src = open(JL).read()
    for t in ("TensorBasis", "ProjectedBasis", "TranslationalBasis", "TranslationParityBasis",
              "AbelianBasis", "ParityBasis", "FlipBasis", "ParityFlipBasis",
              "TranslationFlipBasis"):
        assert re.search(r"b isa " + t + r"\b", src), t
    for sym in ("edk_krylov_cache_create", "edk_krylov_cache_evolve", "edk_krylov_cache_destroy"):
        assert sym in src


# ---- the binding's generator extraction (EDKitB200.jl basis_desc) -------------
def gen_q(c, order):
    """gen_q: quantum number from the phase table c[j] = exp(2pi i q j / order)."""
    if order == 1:
        return 0
    z = complex(c[1])
    return round(math.atan2(z.imag, z.real) * order / (2 * math.pi)) % order


def mom_K(Ctab, length):
    """mom_K: internal momentum K from C[j] = exp(-2pi i K j / len)."""
    if len(Ctab) <= 1:
        return 0
    z = complex(Ctab[1])
    return round(-math.atan2(z.imag, z.real) * length / (2 * math.pi)) % length


def phase_table(order, q):
    """The AbelianOperator's phase table (AbelianBasis.jl:169-176)."""
    if q == 0:
        return [1.0] * order
    if 2 * q == order:
        return [1.0 if j % 2 == 0 else -1.0 for j in range(order)]
    return [complex(math.cos(2 * math.pi * q * j / order), math.sin(2 * math.pi * q * j / order))
            for j in range(order)]


def _desc_from_gens(E, kind, L, gens, I, R):
    d = E.BasisDesc()
    d.kind, d.L, d.base, d.a, d.k, d.p, d.N = kind, L, 2, 1, 0, 1, -1
    order = np.array([g[0] for g in gens], np.int32)
    q = np.array([g[1] for g in gens], np.int32)
    perm = np.ascontiguousarray(np.array([g[2] for g in gens], np.int32).reshape(-1))
    inv = np.ascontiguousarray(np.array([g[3] for g in gens], np.uint8).reshape(-1))
    I = np.ascontiguousarray(I, np.int64)
    R = np.ascontiguousarray(R, np.float64)
    d.ngen = len(gens)
    d.gen_order, d.gen_q = order.ctypes.data, q.ctypes.data
    d.gen_perm, d.gen_inv = perm.ctypes.data, inv.ctypes.data
    d.D, d.I, d.R = len(I), I.ctypes.data, R.ctypes.data
    return d, (order, q, perm, inv, I, R)


def _check_against_oracle(E, d, L, index_fn, I, R):
    lib = E.load()
    h = C.c_void_p()
    E.check(lib.edk_basis_create(C.byref(d), C.byref(h)))
    try:
        D = C.c_int64()
        E.check(lib.edk_basis_dim(h, C.byref(D)))
        assert D.value == len(I)
        Ig = np.zeros(len(I), np.int64)
        Rg = np.zeros(len(I), np.float64)
        E.check(lib.edk_basis_export(h, E.ptr(Ig), E.ptr(Rg)))
        assert np.array_equal(Ig, I) and np.array_equal(Rg, R)
        states = np.arange(2 ** L, dtype=np.uint64)
        pos = np.zeros(len(states), np.int64)
        coeff = np.zeros(len(states), np.complex128)
        E.check(lib.edk_basis_index(h, len(states), E.ptr(states), E.ptr(pos), E.ptr(coeff),
                                    E.HOST))
        for s in range(2 ** L):
            c0, p0 = index_fn(s)
            if c0 == 0:
                assert pos[s] == 0, s
            else:
                assert pos[s] == p0, s
                assert abs(coeff[s] - c0) <= 1e-13 * max(1.0, abs(c0)), s
    finally:
        lib.edk_basis_destroy(h)


def _odgt(s, L):
    return [(s >> (L - 1 - i)) & 1 for i in range(L)]


CASES = [dict(L=10, N=5, k=1), dict(L=10, N=5, k=0, p=-1), dict(L=10, k=5, z=1),
         dict(L=12, N=6, k=3, z=-1), dict(L=10, N=5, p=1, z=-1)]


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
def test_basis_dispatch_desc_like_the_binding(ek, O, case):
    """basis(L, N, k, p, z) is an AbelianBasis; the binding reads its generator
    orders, phase tables, permutations and inversion flags."""
    from edkit_b200 import _lib as E
    L = case["L"]
    kw = {k: v for k, v in case.items() if k != "L"}
    ob = O.basis(L, **kw)
    I, R = ob.tables()
    gens = [(o, gen_q(phase_table(o, q), o), perm, inv) for (o, q, perm, inv) in ob.gens]
    assert [g[1] for g in gens] == [g[1] for g in ob.gens]
    d, keep = _desc_from_gens(E, E.ABELIAN, L, gens, I, R)
    _check_against_oracle(E, d, L, lambda s: ob.index(_odgt(s, L)), I, R)


@pytest.mark.gpu
@pytest.mark.parametrize("kind,args", [("parity", dict(L=10, p=-1, N=5)),
                                       ("flip", dict(L=10, p=1)),
                                       ("parityflip", dict(L=10, p=1, z=-1, N=5)),
                                       ("transflip", dict(L=10, k=3, p=-1, N=5)),
                                       ("transflip", dict(L=12, k=0, p=1, a=2))])
def test_dedicated_bases_desc_like_the_binding(ek, O, kind, args):
    """ParityBasis / FlipBasis / ParityFlipBasis / TranslationFlipBasis carry
    P, Z, C and A; the binding turns them into generators."""
    from edkit_b200 import _lib as E
    L = args["L"]
    refl = [L - i + 1 for i in range(1, L + 1)]
    ident = list(range(1, L + 1))
    if kind == "parity":
        ob = O.parity_basis(L, args["p"], N=args.get("N"))
        gens, dk = [(2, 1 if ob.P == -1 else 0, refl, [0] * L)], E.ABELIAN
    elif kind == "flip":
        ob = O.flip_basis(L, args["p"], N=args.get("N"))
        gens, dk = [(2, 1 if ob.P == -1 else 0, ident, [1] * L)], E.ABELIAN
    elif kind == "parityflip":
        ob = O.parityflip_basis(L, args["p"], args["z"], N=args.get("N"))
        gens = [(2, 1 if ob.P == -1 else 0, refl, [0] * L),
                (2, 1 if ob.Z == -1 else 0, ident, [1] * L)]
        dk = E.ABELIAN
    else:
        ob = O.transflip_basis(L, k=args["k"], p=args["p"], N=args.get("N"), a=args.get("a", 1))
        length = L // ob.A
        perm = [((i - ob.A - 1) % L) + 1 for i in range(1, L + 1)]
        gens = [(length, mom_K(ob.C, length), perm, [0] * L),
                (2, 1 if ob.P == -1 else 0, ident, [1] * L)]
        dk = E.TRANSFLIP
    I, R = np.asarray(ob.I, np.int64), np.asarray(ob.R, np.float64)
    d, keep = _desc_from_gens(E, dk, L, gens, I, R)
    _check_against_oracle(E, d, L, ob.index_state, I, R)
