"""The GPU's implicit FEM shell step against the reference's (golden fixtures from the reference, tests/golden): node
positions within 1e-4 m over hundreds of substeps of the clamped plate under gravity and a point load, no failed
factorization, no clamp. (The element kernels' atan2 / sin / cos differ from libm's in the last bit and the
substitutions sum in another order, so this is a tolerance, not bitwise.)"""
import numpy as np
import pytest

from beamlab_b200 import rigs, world_from_rig
from conftest import golden

pytestmark = pytest.mark.gpu

TOL = 1e-4  # m


@pytest.mark.parametrize("name,n", [("plate20_s1", 20), ("plate63_s1", 63)])
def test_gpu_plate_matches_reference(name, n):
    g = golden(name)
    w = world_from_rig(rigs.shell_plate(n, seed=1))
    h = w.bodies()[0]
    frame = int(g["frame_substeps"])
    snaps = [int(x) for x in g["snap_frames"]]
    for f in range(1, max(snaps) + 1):
        w.step_substeps(frame)
        if f in snaps:
            p = np.ascontiguousarray(h.nodes()["p"]).astype(np.float64)
            d = np.abs(p - g[f"pos_f{f}"]).max()
            assert d <= TOL, f"frame {f}: max |dp| {d:.3g} m"
            fem = h.fem()
            assert np.abs(fem["xd"] - g[f"xd_f{f}"]).max() <= TOL
    st = h.state()
    assert st["fem_failures"] == 0 and st["fem_clamps"] == 0
    w.close()


def test_gpu_factorization_schedules_agree():
    """The block Cholesky's levels launched one by one, the tree's top in one cluster launch (of 1 and of the largest
    cluster the device runs), or the whole tree in it: the same per-column and per-target work in the same order, so
    the plate's state is bitwise the same after 60 substeps."""
    runs = []
    for top, cl in ((10 ** 6, 0), (-1, 0), (-1, 1), (0, 0), (40, 2)):
        w = world_from_rig(rigs.shell_plate(20, seed=3), fem_top_level=top, fem_cluster=cl)
        for _ in range(3):
            w.step_substeps(20)
        fem = w.bodies()[0].fem()
        runs.append((np.ascontiguousarray(w.bodies()[0].nodes()["p"]).copy(), fem["xd"].copy(), fem["w"].copy()))
        assert w.bodies()[0].state()["fem_failures"] == 0
        w.close()
    for r in runs[1:]:
        for a, b in zip(runs[0], r):
            assert np.array_equal(a.view(np.uint8), b.view(np.uint8))
