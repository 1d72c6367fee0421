"""The committed golden fixtures (tests/golden/edk_golden.npz) are what the
oracle computes today: basis tables exactly, H*x and E0 to rounding."""
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def test_oracle_reproduces_golden_fixtures(O):
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "make_golden", os.path.join(HERE, "golden", "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    fresh = mg.generate()
    stored = np.load(mg.PATH)
    assert sorted(stored.files) == sorted(fresh)
    for name, _, _ in mg.CASES:
        assert np.array_equal(stored[name + "/I"], fresh[name + "/I"]), name
        assert np.array_equal(stored[name + "/R"], fresh[name + "/R"]), name
        assert np.array_equal(stored[name + "/x"], fresh[name + "/x"]), name
        y0, y1 = stored[name + "/y"], fresh[name + "/y"]
        assert np.linalg.norm(y0 - y1) <= 1e-13 * np.linalg.norm(y0), name
        assert abs(stored[name + "/E0"][0] - fresh[name + "/E0"][0]) <= 1e-12 * abs(y0).max(), name
