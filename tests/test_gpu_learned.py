"""The implicit FEM step's solvers beside the reference's Cholesky, and the learned warm start (no counterparts in
the reference): the network's forward and gradient kernels against the CPU restatement (oracle/mlp_oracle.py), the
solves' residuals (<= 1e-6 relative, measured on a copy of each assembled system), the fallback to the Cholesky, and
what the trained network gains over PCG without it."""
import numpy as np
import pytest

from beamlab_b200 import rigs, world_from_rig
from oracle import mlp_oracle as mo

pytestmark = pytest.mark.gpu


def plate(n=20, seed=1, **kw):
    return world_from_rig(rigs.shell_plate(n, seed=seed), **kw)


def test_mlp_forward_matches_oracle():
    w = plate()
    w.mlp_init(7)
    p = w.mlp_weights()
    x = np.random.default_rng(1).normal(0, 1, (257, 36)).astype(np.float32)
    y = w.mlp_forward(x)
    yo, _ = mo.forward(p, x)  # (the BF16 weights and layer inputs, accumulated in float64)
    err, scale = np.abs(y - yo), np.max(np.abs(yo))
    # FP32 tensor-core sums against float64 ones: now and then an activation lands on the other side of a BF16
    # rounding boundary (one BF16 ulp, 2^-8), so the worst entry is held loosely and almost all tightly
    assert np.max(err) <= 1e-5 + 3e-3 * scale
    assert np.quantile(err, 0.99) <= 1e-5 + 1e-4 * scale
    w.close()


def test_mlp_gradient_matches_oracle_on_two_calls():
    w = plate()
    rng = np.random.default_rng(2)
    p = rng.normal(0, 0.2, mo.N_PARAMS).astype(np.float32)
    w.set_mlp_weights(p)
    x = rng.normal(0, 1, (200, 36)).astype(np.float32)
    t = rng.normal(0, 1, (200, 12)).astype(np.float32)
    wt = rng.uniform(0, 1, (200, 12)).astype(np.float32)
    g1, l1 = w.mlp_gradient(x, t, wt)
    g2, l2 = w.mlp_gradient(x, t, wt)
    assert np.array_equal(g1, g2) and l1 == l2  # (deterministic: sums in a fixed order)
    lo, go = mo.loss_and_grad(p, x, t, wt)
    err, scale = np.abs(g1 - go), np.max(np.abs(go))
    assert np.max(err) <= 3e-3 * scale  # (as the forward: a rare BF16 rounding-boundary flip of an activation)
    assert np.quantile(err, 0.99) <= 1e-4 * scale
    assert abs(l1 - lo) <= 1e-3 * lo
    w.close()


def test_cholesky_solution_residual():
    """The reference's solve, as this path runs it: |A dv - rhs| / |rhs| of every substep's solution."""
    w = plate(63, fem_check_residual=True)
    for _ in range(5):
        w.step_substeps(20)
    st = w.fem_stats()
    assert 0 < st["max_residual"] <= 1e-6
    w.close()


def test_pcg_meets_tolerance_and_follows_cholesky():
    ref = plate()
    w = plate(fem_solver="pcg", pcg_max_iters=3000, fem_check_residual=True)
    for _ in range(10):
        ref.step_substeps(20)
        w.step_substeps(20)
    st = w.fem_stats()
    assert st["pcg_solves"] == 200 and st["pcg_fallbacks"] == 0
    assert st["max_residual"] <= 1.0001e-6
    d = np.abs(w.bodies()[0].nodes()["p"].astype(np.float64) - ref.bodies()[0].nodes()["p"])
    assert d.max() <= 1e-5
    w.close()
    ref.close()


def test_pcg_fallback_is_the_cholesky():
    """A solve that misses the tolerance within its budget leaves the system to the Cholesky: the same states, bit
    for bit, as the Cholesky alone."""
    ref = plate()
    w = plate(fem_solver="pcg", pcg_max_iters=3)
    for _ in range(3):
        ref.step_substeps(20)
        w.step_substeps(20)
    st = w.fem_stats()
    assert st["pcg_solves"] == 60 and st["pcg_fallbacks"] == 60
    assert np.array_equal(w.bodies()[0].nodes()["p"].view(np.uint32), ref.bodies()[0].nodes()["p"].view(np.uint32))
    w.close()
    ref.close()


def test_learned_warm_start_gain():
    """Train the network on the Cholesky's solves of one plate load (200 substeps, 88,200 node samples), then solve
    200 substeps of another load three ways: from zero, from the last solution (the warm start without the network),
    and from the learned guess (the energy-norm best combination of the network's dv and the last solution). The
    learned start must beat the start from zero and be no worse than the last solution alone; what it gains over the
    latter is printed (measured: about nothing - the network adds little beyond the warm start it is given)."""
    rec = plate(seed=1)
    rec.mlp_record(200 * 441)
    for _ in range(10):
        rec.step_substeps(20)
    assert rec.mlp_samples() == 200 * 441
    rec.mlp_record(0)
    first = rec.mlp_train(1, batch=4096, lr=2e-3, seed=0)
    last = rec.mlp_train(12, batch=4096, lr=1e-3, seed=1)
    assert last < first
    weights = rec.mlp_weights()
    rec.close()
    iters = {}
    for solver in ("pcg", "pcg_previous", "pcg_learned"):
        w = plate(seed=2, fem_solver=solver, pcg_max_iters=3000, fem_check_residual=True)
        if solver == "pcg_learned":
            w.set_mlp_weights(weights)
        for _ in range(10):
            w.step_substeps(20)
        st = w.fem_stats()
        assert st["pcg_fallbacks"] == 0 and st["max_residual"] <= 1.0001e-6
        iters[solver] = st["pcg_iterations"] / st["pcg_solves"]
        w.close()
    print("mean CG iterations:", iters, "learned over previous:", iters["pcg_learned"] / iters["pcg_previous"])
    assert iters["pcg_learned"] < iters["pcg"]
    assert iters["pcg_learned"] <= 1.02 * iters["pcg_previous"]
