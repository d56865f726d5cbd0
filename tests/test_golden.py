"""The oracle reproduces the committed golden fixtures (tests/golden, made by make_golden.py):
integer outputs exactly, FP64 trajectories to 1e-9 m."""
import os

import numpy as np
import pytest

import importlib.util

HERE = os.path.dirname(os.path.abspath(__file__))
spec = importlib.util.spec_from_file_location("make_golden", os.path.join(HERE, "golden", "make_golden.py"))
mg = importlib.util.module_from_spec(spec)
spec.loader.exec_module(mg)


@pytest.mark.parametrize("name", sorted(mg.CASES))
def test_oracle_matches_golden(oracle_lib, name):
    ref = np.load(os.path.join(HERE, "golden", f"{name}.npz"))
    got = mg.generate(name)
    for key in ("morton", "sorted_ids", "lbvh_child", "pairs", "final_stats"):
        assert np.array_equal(got[key], ref[key]), key
    assert np.abs(got["trajectory"] - ref["trajectory"]).max() < 1e-9
