"""Contacts between bodies on the GPU against the reference (World::rebuild_pairs / near_pairs / pair_detect /
collide_pairs, world.cpp:1851-3023).

The pair lists (every island's node-triangle pairs after each search, in the reference's order) must equal the
reference's element for element, and the node states bit for bit: the pair search is integer and comparison work,
and the contact response runs each island's pairs in the reference's order with its float operations in its order.
Fixtures: tests/golden/make_golden_contacts.py (the reference, parity build)."""
import numpy as np
import pytest

from beamlab_b200 import rigs, world_from_rig
from conftest import golden

pytestmark = pytest.mark.gpu

CASES = {
    "crash_slow_s1": lambda: rigs.crash_pair(1, speed_a=3.0, speed_b=0.0, gap=0.1),
    "crash_fast_s2": lambda: rigs.crash_pair(2, speed_a=12.0, speed_b=12.0, gap=0.5),
    "crash_mixed_s3": lambda: rigs.crash_pair(3, speed_a=25.0, speed_b=3.0, gap=0.6),
    "crash_hull_s4": lambda: rigs.crash_pair(4, speed_a=10.0, speed_b=4.0, gap=0.2, hull=True),
}


def bits(a):
    a = np.ascontiguousarray(a, np.float32).copy()
    a[np.isnan(a)] = np.nan  # (one NaN for all payloads)
    return a.view(np.uint32)


@pytest.mark.parametrize("whole_max", [6144, 0], ids=["whole", "chunks"])
@pytest.mark.parametrize("name", list(CASES))
def test_pairs_and_states_equal_reference_fixture(name, whole_max):
    """Both ways an island's contacts run - whole (their order over the island) and 512 at a time - give the
    reference's states."""
    g = golden(name)
    w = world_from_rig(CASES[name](), contact_whole_max=whole_max)
    snaps = set(int(x) for x in g["snap_frames"])
    total_pairs = 0
    for f, n in enumerate(g["frames"]):
        w.step_substeps(int(n))
        got, want = w.pairs(), g[f"pairs_f{f}"]
        assert got.shape == want.shape, f"frame {f}: {len(got)} pairs, the reference {len(want)}"
        assert np.array_equal(got, want), f"frame {f}: pair lists differ"
        total_pairs += len(want)
        if f in snaps:
            for b in range(2):
                nd = w.bodies()[b].nodes()
                assert np.array_equal(bits(nd["p"]), bits(g[f"pos{b}_f{f}"])), f"frame {f} body {b}: positions differ"
                assert np.array_equal(bits(nd["v"]), bits(g[f"vel{b}_f{f}"])), f"frame {f} body {b}: velocities differ"
    st = w.stats()
    assert total_pairs > 0 and st["contacts"] > 0 and st["pair_searches"] > 0
    assert st["device_errors"] == 0
    w.close()


@pytest.mark.parametrize("name", ["crash_mixed_s3", "crash_hull_s4"])
def test_2000_substeps_equal_live_reference(ref_lib, name):
    """2,013 substeps (61 frames of 33) of a crash: every node state bitwise the reference's (the tolerance the
    contract allows is 1e-4 m; the path reaches equality)."""
    from oracle.oracle import RefWorld, build_world
    rig = CASES[name]()
    w = world_from_rig(rig)
    r = build_world(RefWorld, rig, multithreaded=False)
    for _ in range(61):
        w.step_substeps(33)
        r.step_substeps(33)
    for b in range(2):
        nd, rn = w.bodies()[b].nodes(), r.nodes(b)
        assert np.max(np.abs(nd["p"].astype(np.float64) - rn["pos"])) <= 1e-4
        assert np.array_equal(bits(nd["p"]), bits(rn["pos"])) and np.array_equal(bits(nd["v"]), bits(rn["vel"]))
        s, t = w.bodies()[b].state(), r.body(b)
        assert np.array_equal(s["aabb_min"], t["aabb_min"]) and s["max_speed"] == t["max_speed"]  # (values: -0 == +0)
    w.close()
    r.close()


def test_contacts_off_keeps_bodies_apart_from_pairs():
    """WorldSettings::inter_body_collisions off: no islands, no pairs, the bodies pass through each other."""
    rig = rigs.crash_pair(1, speed_a=3.0, speed_b=0.0, gap=0.1)
    w = world_from_rig(rig, inter_body_collisions=False)
    w.step_substeps(33)
    st = w.stats()
    assert len(w.pairs()) == 0 and st["contacts"] == 0 and st["pair_searches"] == 0
    w.close()


def test_sleeping_body_woken_by_contact_matches_reference(ref_lib):
    """A truss resting on the ground falls asleep (its sleep speed raised to 0.5 m/s), another dropped from 20 m lands
    on it and wakes it (SoftBody::wake_request through the contact between them): the sleeping flags frame by frame
    and the final states bitwise the reference's."""
    from oracle.oracle import RefWorld, build_world
    rig = rigs.drop_pair(1, height=20.0, dims=(6, 2, 3))
    rig["bodies"][0]["params"]["sleep_speed"] = 0.5
    w = world_from_rig(rig)
    ref = build_world(RefWorld, rig, multithreaded=False)
    got, want = [], []
    for f in range(130):
        w.step_substeps(33)
        ref.step_substeps(33)
        got.append(bool(w.bodies()[0].state()["sleeping"]))
        want.append(bool(ref.body(0)["sleeping"]))
    assert got == want
    assert any(want) and not want[-1]  # (it slept, and was woken)
    for b in range(2):
        nd = w.bodies()[b].nodes()
        r = ref.nodes(b)
        assert np.array_equal(bits(nd["p"]), bits(r["pos"])) and np.array_equal(bits(nd["v"]), bits(r["vel"])), f"body {b}"
    w.close()


def test_fleet_pairs_crashing_at_once_equal_reference(ref_lib):
    """Eight islands in contact at once: a fleet of 16 lattice vehicles with skins and wheels laid out in head-on pairs
    (rigs.fleet(layout="pairs")) over a heightfield, 8 frames of 33 substeps on the GPU and by the compiled reference:
    after every frame the pair lists equal the reference's element for element (the islands' lists in the reference's
    order) and every node's position and velocity is bitwise the reference's."""
    from oracle.oracle import RefWorld, build_world
    rig = rigs.fleet(16, seed=5, median_nodes=900, min_nodes=300, max_nodes=3000, terrain_size=400.0, terrain_samples=513,
                     layout="pairs")
    w = world_from_rig(rig)
    r = build_world(RefWorld, rig, multithreaded=False)
    total = 0
    for f in range(8):
        w.step_substeps(33)
        r.step_substeps(33)
        got, want = w.pairs(), r.pairs()
        assert got.shape == want.shape and np.array_equal(got, want), f"frame {f}: pair lists differ ({len(got)} vs {len(want)})"
        total += len(want)
        for b in range(len(rig["bodies"])):
            g, ref = w.bodies()[b].nodes(), r.nodes(b)
            assert np.array_equal(bits(g["p"]), bits(ref["pos"])), f"frame {f} vehicle {b}: positions differ"
            assert np.array_equal(bits(g["v"]), bits(ref["vel"])), f"frame {f} vehicle {b}: velocities differ"
    st = w.stats()
    assert total > 0 and st["contacts"] > 1000 and st["pair_searches"] > 0 and st["device_errors"] == 0
    touched = sum(1 for b in range(16) if w.bodies()[b].state()["body_contacts"] > 0)
    assert touched >= 8, f"only {touched} of 16 vehicles in contact in the last substep"  # (the pairs crash; some rebound)
    w.close()
    r.close()


def test_fleet_contacts_whole_equal_chunks():
    """The fleet's islands (many over 512 contacts in a substep) run whole and 512 at a time: the same node states bit
    for bit, frame after frame."""
    rig = rigs.fleet(16, seed=5, median_nodes=900, min_nodes=300, max_nodes=3000, terrain_size=400.0, terrain_samples=513,
                     layout="pairs")
    a = world_from_rig(rig)
    b = world_from_rig(rig, contact_whole_max=0)
    for f in range(8):
        a.step_substeps(33)
        b.step_substeps(33)
        for k in range(len(rig["bodies"])):
            x, y = a.bodies()[k].nodes(), b.bodies()[k].nodes()
            assert np.array_equal(bits(x["p"]), bits(y["p"])) and np.array_equal(bits(x["v"]), bits(y["v"])), f"frame {f} vehicle {k}"
    sa, sb = a.stats(), b.stats()
    assert sa["contacts"] == sb["contacts"] > 1000 and sa["device_errors"] == sb["device_errors"] == 0
    a.close()
    b.close()


def test_fleet_pairs_4000_substeps_equal_reference(ref_lib):
    """The 16-vehicle crashing fleet over the configuration's horizon: 122 frames of 33 substeps (4,026) on the GPU and
    by the compiled reference - the crashes, the rebounds and the vehicles rolling on after them. Every 11th frame the
    pair lists equal the reference's; at the end every node's position and velocity is bitwise the reference's."""
    from oracle.oracle import RefWorld, build_world
    rig = rigs.fleet(16, seed=5, median_nodes=900, min_nodes=300, max_nodes=3000, terrain_size=400.0, terrain_samples=513,
                     layout="pairs")
    w = world_from_rig(rig)
    r = build_world(RefWorld, rig, multithreaded=False)
    for f in range(122):
        w.step_substeps(33)
        r.step_substeps(33)
        if f % 11 == 0:
            got, want = w.pairs(), r.pairs()
            assert got.shape == want.shape and np.array_equal(got, want), f"frame {f}: pair lists differ ({len(got)} vs {len(want)})"
    for b in range(len(rig["bodies"])):
        g, ref = w.bodies()[b].nodes(), r.nodes(b)
        assert np.array_equal(bits(g["p"]), bits(ref["pos"])), f"vehicle {b}: positions differ"
        assert np.array_equal(bits(g["v"]), bits(ref["vel"])), f"vehicle {b}: velocities differ"
    st = w.stats()
    assert st["contacts"] > 1000 and st["device_errors"] == 0
    w.close()
    r.close()
