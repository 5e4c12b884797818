"""The batched fleet at full size against the reference, and the batched path against the plain per-instance one.

* fleet256 - the bench's workload (256 lattice vehicles in 128 head-on pairs, 943,132 nodes, 8,870,418 beams,
  collision skins, wheels, a 2048^2-sample heightfield) - stepped five 33-substep frames (the first crashes) on the GPU
  and by the reference compiled from its sources (oracle/_ref, parity build): every node's position and velocity
  bitwise equal, every body's bounds and top speed.
* a small fleet in one World (one kernel per phase over all bodies, frames as CUDA graphs) and each of its vehicles in
  a World of its own with its frames' kernels launched one by one: bitwise equal."""
import numpy as np
import pytest

from beamlab_b200 import rigs, world_from_rig

pytestmark = pytest.mark.gpu


def bits(a):
    a = np.ascontiguousarray(a, np.float32).copy()
    a[np.isnan(a)] = np.nan  # (one NaN for all payloads)
    return a.view(np.uint32)


def test_fleet256_full_size_equals_reference(ref_lib):
    from oracle.oracle import RefWorld, build_world
    rig = rigs.fleet(256, seed=3, layout="pairs")
    gw = world_from_rig(rig)
    rw = build_world(RefWorld, rig, multithreaded=False)
    for _ in range(5):
        gw.step_substeps(33)
        rw.step_substeps(33)
    hs = gw.bodies()
    moved = 0.0
    for b in range(len(rig["bodies"])):
        g, r = hs[b].nodes(), rw.nodes(b)
        assert np.array_equal(bits(g["p"]), bits(r["pos"])), f"vehicle {b}: positions differ"
        assert np.array_equal(bits(g["v"]), bits(r["vel"])), f"vehicle {b}: velocities differ"
        sg, sr = hs[b].state(), rw.body(b)
        assert np.array_equal(bits(sg["aabb_min"]), bits(sr["aabb_min"])) and np.array_equal(bits(sg["aabb_max"]), bits(sr["aabb_max"]))
        assert sg["max_speed"] == sr["max_speed"] and sg["static_contacts"] == sr["static_contacts"]
        moved = max(moved, float(np.abs(r["pos"] - rig["bodies"][b]["pos"]).max()))
    assert moved > 0.1  # (the vehicles drive: up to 30 m/s for 83 ms)
    st = gw.stats()
    assert st["device_errors"] == 0 and st["contacts"] > 0  # (the pairs that meet within 83 ms crash)
    gw.close()
    rw.close()


def test_batched_equals_plain_per_instance():
    rig = rigs.fleet(6, seed=9, median_nodes=600, min_nodes=200, max_nodes=1500, terrain_size=300.0, terrain_samples=257)
    batched = world_from_rig(rig)
    alone = [world_from_rig({"settings": rig["settings"], "statics": rig["statics"], "bodies": [b]}, graphs=False)
             for b in rig["bodies"]]
    for n in (33, 20, 33):
        batched.step_substeps(n)
        for w in alone:
            w.step_substeps(n)
    for b, w in enumerate(alone):
        x, y = batched.bodies()[b].nodes(), w.bodies()[0].nodes()
        assert np.array_equal(bits(x["p"]), bits(y["p"])) and np.array_equal(bits(x["v"]), bits(y["v"])), f"vehicle {b}"
        assert np.array_equal(batched.bodies()[b].beams()["stress"].view(np.uint32), w.bodies()[0].beams()["stress"].view(np.uint32))
    assert sum(w.stats()["kernel_launches"] for w in alone) > batched.stats()["kernel_launches"]
    for w in [batched] + alone:
        w.close()
