"""The CUDA library against the committed golden fixtures, without running the
oracle: basis tables bit-exact, H*x within 1e-12 relative (FP64), E0 from the
device Lanczos within 1e-10 relative."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def _cases():
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "make_golden", os.path.join(HERE, "golden", "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    return mg


def test_library_matches_golden_fixtures(ek):
    mg = _cases()
    g = np.load(mg.PATH)
    for name, kind, kw in mg.CASES:
        b = getattr(ek, kind)(**kw)
        assert np.array_equal(b.I, g[name + "/I"]), name
        assert np.array_equal(b.R, g[name + "/R"]), name
        H = ek.trans_inv_operator(ek.spin(*mg.XXZ), 2, b)
        x, y = g[name + "/x"], g[name + "/y"]
        assert np.linalg.norm(H * x - y) <= 1e-12 * np.linalg.norm(y), name
        e, _ = ek.lanczos_e0(H, np.real(x), m=min(120, b.size(1) - 1), tol=1e-13)
        E0 = g[name + "/E0"][0]
        assert abs(e[0] - E0) <= 1e-10 * abs(E0), (name, e[0], E0)
