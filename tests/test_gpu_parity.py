"""The CUDA path against the oracle: bitwise equal node and beam states after thousands of substeps, through the C ABI
(beamlab_b200.World -> include/beamlab_gpu.h)."""
import numpy as np
import pytest

from beamlab_b200 import rigs
from conftest import golden
from gpu_adapter import GpuWorld
from test_oracle import CASES, bits, run_against_golden

pytestmark = pytest.mark.gpu


def assert_same(gw, ow, nbodies, what=""):
    for b in range(nbodies):
        a, c = gw.nodes(b), ow.nodes(b)
        dp = np.abs(a["pos"].astype(np.float64) - c["pos"]).max() if len(a["pos"]) else 0.0
        assert np.array_equal(bits(a["pos"]), bits(c["pos"])), f"{what} body {b}: positions differ (max {dp:.3g} m)"
        assert np.array_equal(bits(a["vel"]), bits(c["vel"])), f"{what} body {b}: velocities differ"
        assert np.array_equal(bits(a["inv_mass"]), bits(c["inv_mass"]))
        ga, oa = gw.beams(b), ow.beams(b)
        for k in ("L", "max_pos", "max_neg", "strength", "stress"):
            assert np.array_equal(bits(ga[k]), bits(oa[k])), f"{what} body {b}: beam {k} differs"
        assert np.array_equal(ga["flags"], oa["flags"])
        sa, so = gw.body(b), ow.body(b)
        for k in ("max_speed", "sleeping", "static_contacts", "broken_beams", "sleep_timer"):
            assert sa[k] == so[k], f"{what} body {b}: {k} {sa[k]} != {so[k]}"
        assert np.array_equal(bits(sa["aabb_min"]), bits(so["aabb_min"])) and np.array_equal(bits(sa["aabb_max"]), bits(so["aabb_max"]))


@pytest.mark.parametrize("name", sorted(CASES))
def test_gpu_matches_golden(name):
    """2,000 substeps of the truss car into the wall and of the stress rig: bitwise the reference's fixtures."""
    run_against_golden(GpuWorld(CASES[name]()), name)


@pytest.mark.parametrize("make", [lambda: rigs.truss_car(2, speed=30.0), lambda: rigs.stress_rig(11),
                                  lambda: rigs.fleet(12, seed=5, median_nodes=800, min_nodes=60, max_nodes=4000,
                                                     terrain_size=300.0, terrain_samples=257, skins=False,
                                                     wheels=False)])
def test_gpu_matches_oracle_live(port_lib, make):
    from oracle.oracle import PortWorld, build_world
    rig = make()
    gw, ow = GpuWorld(rig), build_world(PortWorld, rig)
    for f in range(30):
        n = 20 + (f % 3)
        gw.step_substeps(n)
        ow.step_substeps(n)
        if f in (0, 7, 29):
            assert_same(gw, ow, len(rig["bodies"]), f"frame {f}")


def test_gpu_sleep_and_repair(port_lib):
    """A body at rest falls asleep in the oracle's frame; a node made non-finite is repaired as the oracle does."""
    from oracle.oracle import PortWorld, build_world
    rig = rigs.truss_car(3, speed=0.0, dims=(4, 2, 2))
    rig["bodies"].append(rigs.truss_car(4, speed=5.0, dims=(6, 3, 3))["bodies"][0])
    rig["bodies"][1]["pos"][:, 2] += 5.0
    gw, ow = GpuWorld(rig), build_world(PortWorld, rig)
    for w in (gw, ow):
        w.step_substeps(20)
        nd = w.nodes(1)
        pos, vel = nd["pos"].copy(), nd["vel"].copy()
        pos[7] = np.nan
        vel[11] = (500.0, 0.0, 0.0)
        w.set_nodes(1, pos, vel)
    slept = False
    for f in range(90):
        gw.step_substeps(33)
        ow.step_substeps(33)
        if f in (0, 1, 89):
            assert_same(gw, ow, 2, f"frame {f}")
        slept |= gw.body(0)["sleeping"]
    assert slept and gw.h[1].state()["repaired_nodes"] >= 2


def test_gpu_frames_and_streams(port_lib):
    """Frames of any length (each captured once as a graph, then replayed), on the world's stream or a caller's."""
    import torch
    from oracle.oracle import PortWorld, build_world
    rig = rigs.stress_rig(3)
    gw, ow = GpuWorld(rig), build_world(PortWorld, rig)
    s = torch.cuda.Stream()
    for f, n in enumerate([1, 2, 33, 1, 17, 33, 33, 5]):
        gw.step_substeps(n, stream=s if f % 2 else None)
        ow.step_substeps(n)
    assert_same(gw, ow, 3, "mixed frames")
    st = gw.w.stats()
    assert st["total_substeps"] == 125 and st["kernel_launches"] == 3 * 125 + 3 * 8 and st["device_errors"] == 0


def _wall_crash(seed, shuffle=False):
    """A 30 x 6 x 6 truss (1,080 nodes) with weak beams at 30 m/s into the wall: beams yield and break all over its
    front. shuffle: its beams in a seeded random order (each node's beams far apart in memory)."""
    rig = rigs.truss_car(seed, speed=30.0, dims=(30, 6, 6))
    b = rig["bodies"][0]
    b["deform"][:] = 8e3
    b["strength"][:] = 2.5e4
    if shuffle:
        perm = np.random.default_rng(seed).permutation(len(b["k"]))
        for k in ("ab", "k", "d", "strength", "deform", "beam_type", "beam_flags"):
            b[k] = np.ascontiguousarray(b[k][perm])
    return rig


@pytest.mark.parametrize("shuffle,beam_kernel", [(False, 0), (True, 0), (False, 1)])
def test_gpu_crash_yield_and_break_match_oracle(port_lib, shuffle, beam_kernel):
    """Thousands of beams yield and hundreds break in a 30 m/s crash - with the beams in builder order and shuffled,
    the beam arrays streamed by bulk copies or loaded plainly - and the state stays bitwise the oracle's."""
    from oracle.oracle import PortWorld, build_world
    from beamlab_b200.world import SoftBody
    rig = _wall_crash(5, shuffle)
    gw, ow = GpuWorld(rig, beam_kernel=beam_kernel), build_world(PortWorld, rig)
    for f in range(12):
        gw.step_substeps(25)
        ow.step_substeps(25)
        if f in (3, 6, 11):
            assert_same(gw, ow, 1, f"frame {f}")
    rest = SoftBody.from_arrays(rig["bodies"][0]).beams["L"]
    yielded = np.count_nonzero(gw.beams(0)["L"] != rest)
    assert gw.body(0)["broken_beams"] > 100 and yielded > 1000, (gw.body(0)["broken_beams"], yielded)


@pytest.mark.parametrize("split", [False, True])
def test_gpu_air_drag_matches_reference(ref_lib, split):
    """RoR's per-node air drag against each part's mean velocity and Cd A drag on the parts' means
    (SoftBody::clear_forces, softbody.cpp:334-378): the truss car - one part - and the 30 m/s crash whose broken
    beams split it into parts (labelled again when they are 8 substeps old), bitwise the compiled reference's."""
    from oracle.oracle import RefWorld, build_world
    rig = _wall_crash(5) if split else rigs.truss_car(1)
    rig["bodies"][0]["params"].update({"air_drag": 0.05, "aero_cda": 0.8})
    gw, rw = GpuWorld(rig), build_world(RefWorld, rig, multithreaded=False)
    for f in range(12):
        gw.step_substeps(25)
        rw.step_substeps(25)
        if f in (2, 7, 11):
            assert_same(gw, rw, 1, f"frame {f}")
