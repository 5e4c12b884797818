"""The learned warm start's CPU restatement (oracle/mlp_oracle.py), pinned: its analytic gradient against central
differences, its BF16 rounding against known values. (The network has no counterpart in the reference.)"""
import numpy as np

from oracle import mlp_oracle as mo


def test_parameter_count_matches_header():
    import os
    import re
    h = open(os.path.join(os.path.dirname(__file__), "..", "include", "beamlab_gpu.h")).read()
    assert int(re.search(r"#define BL_GPU_MLP_PARAMS (\d+)", h).group(1)) == mo.N_PARAMS == 11468


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.0078125, 3.14159265, -2.5e-3, 65504.0, 1.0 + 2 ** -9], np.float32)
    r = mo.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0078125  # (1 + 2^-8: a tie, to even; 1 + 2^-7 exact)
    assert abs(r[3] - 3.140625) < 1e-7
    assert np.all(np.abs(r - x) <= np.abs(x) * 2 ** -8)
    assert np.all((r.view(np.uint32) & 0xFFFF) == 0)


def test_analytic_gradient_matches_central_differences():
    rng = np.random.default_rng(3)
    p = rng.normal(0, 0.25, mo.N_PARAMS)
    x = rng.normal(0, 1, (48, mo.N_IN))
    t = rng.normal(0, 1, (48, mo.N_OUT))
    w = rng.uniform(0, 1, (48, mo.N_OUT))
    _, g = mo.loss_and_grad(p, x, t, w, round_bf16=False)
    idx = np.concatenate([rng.choice(mo.N_PARAMS, 60, replace=False), [0, mo.N_PARAMS - 1]])
    cd = mo.central_difference(p, x, t, w, idx)
    assert np.max(np.abs(cd - g[idx])) <= 1e-6 * np.max(np.abs(g[idx]))
