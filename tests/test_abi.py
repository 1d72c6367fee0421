"""CPU-side checks of the C ABI: libedk.so loads and exports every function
declared in include/edk.h; argument validation that needs no device."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "edk.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(edk_[A-Za-z0-9_]+)\s*\(", src)))


def test_header_declares_expected_api():
    names = declared_functions()
    for n in ("edk_basis_create", "edk_operator_create", "edk_apply", "edk_lanczos_e0",
              "edk_krylov_evolve", "edk_batch_lanczos_e0", "edk_last_error"):
        assert n in names


def test_library_exports_every_declared_symbol(ek):
    lib = C.CDLL(os.path.join(ROOT, "edkit.jl_b200", "libedk.so"))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, f"missing exports: {missing}"


def test_python_binding_covers_header(ek):
    from edkit_b200 import _lib
    assert sorted(_lib.EXPORTS) == declared_functions()


def test_version_string(ek):
    assert "sm_100a" in ek.version()


def test_null_arguments_rejected(ek):
    from edkit_b200 import _lib as E
    lib = E.load()
    assert lib.edk_basis_create(None, None) == E.INVALID_ARG
    assert "NULL" in lib.edk_last_error().decode()
    assert lib.edk_apply(None, 0, None, None, 1, 1, 1, 0, 0) == E.INVALID_ARG


def test_base3_rejected_as_unsupported(ek):
    from edkit_b200 import _lib as E
    d = E.BasisDesc()
    d.kind, d.L, d.base, d.a, d.N = E.TENSOR, 4, 3, 1, -1
    h = C.c_void_p()
    assert E.load().edk_basis_create(C.byref(d), C.byref(h)) == E.UNSUPPORTED
    assert "base 2" in E.load().edk_last_error().decode()


def test_tridiagonal_eigensolver_host(ek):
    """The host eigensolver used by Lanczos/Krylov (no device needed)."""
    rng = np.random.default_rng(0)
    for m in (1, 2, 5, 40, 200):
        a, b = rng.standard_normal(m), rng.standard_normal(max(m - 1, 1))
        w, Q = ek.tridiag_eigen(a, b)
        T = np.diag(a) + (np.diag(b[: m - 1], 1) + np.diag(b[: m - 1], -1) if m > 1 else 0)
        assert np.allclose(w, np.linalg.eigvalsh(T), atol=1e-12)
        assert np.allclose(T @ Q, Q * w, atol=1e-10)
        assert np.allclose(Q.T @ Q, np.eye(m), atol=1e-12)


def test_spin_and_merge_match_oracle(ek, O):
    for s in ("xx", "yy", "zz", "x1z", "+-", "-+", "XYZ", "yyy", "Y"):
        assert np.allclose(ek.spin(s), O.spin(s)), s
    m = ek.spin((1.0, "xx"), (1.0, "yy"), (0.5, "zz"))
    assert np.allclose(m, O.spin((1.0, "xx"), (1.0, "yy"), (0.5, "zz")))
    from edkit_b200.operator import _merge
    M, I = _merge([m, m, 0 * m, m], [[1, 2], [2, 3], [3, 4], [1, 2]])
    assert I == [[1, 2], [2, 3]] and np.allclose(M[0], 2 * m)


def test_gapratio_and_meangapratio(ek):
    E = [0.0, 1.0, 3.0, 6.0]
    assert np.allclose(ek.gapratio(E), [0.5, 2 / 3])
    assert abs(ek.meangapratio(E) - 7 / 12) < 1e-15
    assert np.allclose(ek.gapratio([0.0, 1.0, 2.0]), [1.0])
