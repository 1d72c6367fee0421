"""Generate tests/golden/edk_golden.npz: seeded fixtures of the CPU oracle.

EDKit.jl stores no golden vectors and cannot run here (Julia is absent), so
these fixtures come from the oracle (oracle/, the C++/numpy restatement of
the reference, itself pinned by the reference's known-answer tests).  They
pin two things: the oracle does not drift (tests/test_golden.py regenerates
and compares), and the CUDA library reproduces the tables bit for bit and
H*x / E0 within tolerance without running the oracle (tests/test_gpu_golden.py).

    python tests/golden/make_golden.py      # rewrites edk_golden.npz
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
PATH = os.path.join(HERE, "edk_golden.npz")

XXZ = ((1.0, "xx"), (1.0, "yy"), (1.5, "zz"))

# (name, basis kind, keyword arguments of the product constructor)
CASES = [
    ("tensor_L10", "TensorBasis", {"L": 10}),
    ("projected_L12_N6", "ProjectedBasis", {"L": 12, "N": 6}),
    ("trans_L14_N7_k0", "TranslationalBasis", {"L": 14, "N": 7, "k": 0}),
    ("trans_L14_N7_k3", "TranslationalBasis", {"L": 14, "N": 7, "k": 3}),
    ("trans_L12_N6_k1_a2", "TranslationalBasis", {"L": 12, "N": 6, "k": 1, "a": 2}),
    ("transpar_L14_N7_k0_pm", "TranslationParityBasis", {"L": 14, "N": 7, "k": 0, "p": -1}),
    ("transpar_L12_k6_p", "TranslationParityBasis", {"L": 12, "k": 6, "p": 1}),
    ("abelian_L12_N6_k2_z", "basis", {"L": 12, "N": 6, "k": 2, "z": 1}),
]


def oracle_basis(O, kind, kw):
    L = kw["L"]
    if kind == "TensorBasis":
        return O.tensor(L)
    if kind == "ProjectedBasis":
        return O.projected(L, N=kw.get("N"))
    if kind == "TranslationalBasis":
        return O.translational(L, k=kw.get("k", 0), N=kw.get("N"), a=kw.get("a", 1))
    if kind == "TranslationParityBasis":
        return O.transparity(L, k=kw.get("k", 0), p=kw.get("p", 1), N=kw.get("N"))
    return O.basis(L, N=kw.get("N"), k=kw.get("k"), p=kw.get("p"), z=kw.get("z"))


def generate():
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    import oracle as O
    out = {}
    for i, (name, kind, kw) in enumerate(CASES):
        b = oracle_basis(O, kind, kw)
        I, R = b.tables()
        H = O.trans_inv_operator(O.spin(*XXZ), 2, b)
        rng = np.random.default_rng(1000 + i)
        D = b.dim
        x = rng.standard_normal(D) + 1j * rng.standard_normal(D)
        y = H.mul(x)
        E0 = np.linalg.eigvalsh(H.dense())[0]
        out[name + "/I"] = np.asarray(I, dtype=np.int64)
        out[name + "/R"] = np.asarray(R, dtype=np.float64)
        out[name + "/x"] = x
        out[name + "/y"] = np.asarray(y, dtype=np.complex128)
        out[name + "/E0"] = np.array([E0])
    return out


if __name__ == "__main__":
    np.savez_compressed(PATH, **generate())
    print(PATH, os.path.getsize(PATH), "bytes")
