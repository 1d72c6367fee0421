"""edk_basis_index_noalloc: index() through the C ABI without device allocation.

Callers that cannot allocate device memory at the point of a lookup (host
callbacks that forbid allocation, processes whose device memory another
component has reserved) use this entry point; it must give
exactly what edk_basis_index gives, call after call, from its shared fixed
scratch.  This file is collected last so that a failure here leaves every
other test already run."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _index(lib, E, b, states, noalloc):
    st = np.ascontiguousarray(states, dtype=np.uint64)
    pos = np.full(len(st), -7, dtype=np.int64)
    coeff = np.full(len(st), np.nan, dtype=np.complex128)
    if noalloc:
        E.check(lib.edk_basis_index_noalloc(b._h, len(st), E.ptr(st), E.ptr(pos), E.ptr(coeff)))
    else:
        E.check(lib.edk_basis_index(b._h, len(st), E.ptr(st), E.ptr(pos), E.ptr(coeff), E.HOST))
    return pos, coeff


def test_noalloc_index_matches_index_twice(ek):
    from edkit_b200 import _lib as E
    lib = E.load()
    rng = np.random.default_rng(21)
    bases = [ek.TranslationalBasis(L=16, k=3, N=8), ek.ProjectedBasis(L=14, N=7),
             ek.TranslationParityBasis(L=12, k=0, p=-1)]
    for b in bases:
        for call in range(2):  # two calls in a row share the same scratch
            n = 65536 if call == 0 else 1000
            states = rng.integers(0, 2 ** b.L, size=n).astype(np.uint64)
            p0, c0 = _index(lib, E, b, states, noalloc=False)
            p1, c1 = _index(lib, E, b, states, noalloc=True)
            assert np.array_equal(p0, p1)
            assert np.array_equal(c0, c1)  # same kernel, bit-identical coefficients
            assert np.count_nonzero(p1) > 0


def test_noalloc_rejects_oversized_batch(ek):
    from edkit_b200 import _lib as E
    lib = E.load()
    b = ek.ProjectedBasis(L=10, N=5)
    st = np.zeros(65537, dtype=np.uint64)
    pos = np.zeros(65537, dtype=np.int64)
    coeff = np.zeros(65537, dtype=np.complex128)
    assert lib.edk_basis_index_noalloc(b._h, 65537, E.ptr(st), E.ptr(pos), E.ptr(coeff)) == \
        E.INVALID_ARG
    assert "65536" in lib.edk_last_error().decode()
