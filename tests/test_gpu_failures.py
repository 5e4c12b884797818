"""The failure paths, made to happen without faulting the GPU:

* the beams kernel's bounded wait on its own bulk copies, set to run out at once (bulk_wait_s = 0):
  BL_GPU_DEVERR_TIMEOUT is raised, the copies in flight land, and the device stays usable (a world stepped next on it
  is bitwise the oracle's);
* a contact pair list too small for an island's pairs (max_pairs): BL_GPU_DEVERR_PAIRS, and the island's contacts are
  skipped - the bodies step as if they did not collide;
* a frame whose assembled system is not positive definite (a section with a negative axial factor): the factorization
  fails, the step falls back to the explicit forces for that component (frame_fem.cpp:2900-2909), as in the reference:
  the same failure count and the nodes within the FEM tolerance of the reference's."""
import numpy as np
import pytest

from beamlab_b200 import rigs, world_from_rig

pytestmark = pytest.mark.gpu

DEVERR_PAIRS, DEVERR_TIMEOUT = 1 << 2, 1 << 6


def bits(a):
    a = np.ascontiguousarray(a, np.float32).copy()
    a[np.isnan(a)] = np.nan
    return a.view(np.uint32)


def test_bulk_copy_wait_runs_out_and_the_device_stays_usable(port_lib):
    from oracle.oracle import PortWorld, build_world
    w = world_from_rig(rigs.truss_car(1), bulk_wait_s=0.0)
    w.step_substeps(1)
    st = w.stats()
    assert st["device_errors"] & DEVERR_TIMEOUT
    assert np.all(np.isfinite(w.bodies()[0].nodes()["p"]))  # (the state comes back: no CUDA error)
    w.close()
    rig = rigs.truss_car(1)
    g = world_from_rig(rig)
    c = build_world(PortWorld, rig)
    for _ in range(5):
        g.step_substeps(20)
        c.step_substeps(20)
    assert np.array_equal(bits(g.bodies()[0].nodes()["p"]), bits(c.nodes(0)["pos"]))
    assert g.stats()["device_errors"] == 0
    g.close()


def test_pair_list_overflow_skips_the_island():
    rig = rigs.crash_pair(2, speed_a=12.0, speed_b=12.0, gap=0.5)
    small = world_from_rig(rig, max_pairs=8)
    apart = world_from_rig(rig, inter_body_collisions=False)
    for _ in range(6):
        small.step_substeps(33)
        apart.step_substeps(33)
    st = small.stats()
    assert st["device_errors"] & DEVERR_PAIRS and st["contacts"] == 0 and st["pair_searches"] > 0
    for b in range(2):
        x, y = small.bodies()[b].nodes(), apart.bodies()[b].nodes()
        assert np.array_equal(bits(x["p"]), bits(y["p"])) and np.array_equal(bits(x["v"]), bits(y["v"])), f"body {b}"
    small.close()
    apart.close()


def test_failed_factorization_falls_back_as_the_reference(ref_lib):
    from oracle.oracle import RefWorld, build_world
    sec = rigs.tube_section()
    sec["axial"] = -50.0  # (the members pull where they are pushed: the step's system is indefinite)
    rig = rigs.frame_ladder(12, section=sec)
    w = world_from_rig(rig)
    ref = build_world(RefWorld, rig, multithreaded=False)
    for f in range(4):
        w.step_substeps(10)
        ref.step_substeps(10)
        d = np.abs(np.ascontiguousarray(w.bodies()[0].nodes()["p"]).astype(np.float64) - ref.nodes(0)["pos"]).max()
        assert d <= 1e-4, f"frame {f}: max |dp| {d:.3g} m"
    fails = w.bodies()[0].state()["fem_failures"]
    assert fails > 0 and fails == ref.fem_info(0)["solve_failures"]
    w.close()
