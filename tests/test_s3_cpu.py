"""The C++ stage-3 restatement (oracle/s3_cpu.cpp, the CPU baseline's stage 3)
against the FP64 oracle fixtures: it must run the same algorithm, so it lands
within float32 distance of the FP64 result, like the CUDA path."""
import importlib.util
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# largest vertex deviation from the FP64 oracle as a fraction of the ground
# truth's bounding-box diagonal; measured 4.3e-8 (config 1) and 7.2e-5
# (thin shells, ~45,000 contact blocks) -- the CUDA path's were 4.4e-8 and
# 4.9e-5 .. 5.6e-5
TOL = {"c1": 1e-6, "shell8k": 1.5e-4}


def _case(name):
    spec = importlib.util.spec_from_file_location("make_s3_oracle", os.path.join(GOLDEN, "make_s3_oracle.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    V, F, _, _ = m.case_input(name)
    return V, F, np.load(os.path.join(GOLDEN, f"s3_{name}.npz"))


@pytest.mark.parametrize("name", ["c1", "shell8k"])
def test_s3_cpu_matches_fp64_oracle(name):
    from oracle import s3_cpu

    V, F, fx = _case(name)
    st = {}
    got, gf = s3_cpu.process(V, F, fx["v"], fx["f"], int(fx["steps"]), stats=st)
    assert np.array_equal(gf, fx["f"])
    diag = float(np.linalg.norm(V.max(0) - V.min(0)))
    err = np.abs(got - fx["q"]).max() / diag
    moved = np.abs(fx["q"] - fx["v"]).max() / diag
    assert moved > 3 * err
    assert err < TOL[name], err
    # the thin shells are in contact; the last detection's block count is the
    # oracle's to within the threshold cases
    assert abs(st["blocks"] - int(fx["trace"][-1, 4])) <= 1e-3 * max(int(fx["trace"][-1, 4]), 1000)


def test_s3_cpu_config2_input_one_step():
    """Config 2's stage-3 input (20,604 faces against the 2,097,152-face torus,
    ~1.6M contact blocks), one step.  Measured: vertex error median 4.8e-6,
    max 3.4e-4 of the diagonal, against a move of median 9.7e-5, max 1.4e-3
    (CCD-limited steps taken slightly longer or shorter move every vertex)."""
    from oracle import s3_cpu

    V, F, fx = _case("c2step")
    st = {}
    got, _ = s3_cpu.process(V, F, fx["v"], fx["f"], int(fx["steps"]), stats=st)
    diag = float(np.linalg.norm(V.max(0) - V.min(0)))
    err = np.linalg.norm(got - fx["q"], axis=1) / diag
    move = np.linalg.norm(fx["q"] - fx["v"], axis=1) / diag
    assert np.median(err) < 0.25 * np.median(move)
    assert err.max() < 1e-3
    assert abs(st["blocks"] - int(fx["trace"][-1, 4])) <= 1e-3 * int(fx["trace"][-1, 4])
