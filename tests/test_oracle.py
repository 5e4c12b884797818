"""The CPU oracle (the plain-C restatement) pinned against the reference: bitwise equal node and beam states, against
the committed golden fixtures (the reference's outputs) and against the compiled reference live."""
import numpy as np
import pytest

from beamlab_b200 import rigs
from conftest import golden

CASES = {"truss_car_s1": lambda: rigs.truss_car(1), "stress_rig_s7": lambda: rigs.stress_rig(7)}


def bits(a):
    """The float32 bit patterns, every NaN as one (x86 and the GPU give NaNs different payloads)."""
    a = np.ascontiguousarray(a, np.float32).copy()
    a[np.isnan(a)] = np.float32("nan")
    return a.view(np.uint32)


def run_against_golden(world, name):
    g = golden(name)
    rig = CASES[name]()
    frame = int(g["frame_substeps"])
    snaps = set(int(x) for x in g["snap_frames"])
    last = max(snaps)
    for f in range(1, last + 1):
        world.step_substeps(frame)
        if f in snaps:
            for b in range(len(rig["bodies"])):
                nd = world.nodes(b)
                assert np.array_equal(bits(nd["pos"]), bits(g[f"pos_f{f}_b{b}"])), f"{name}: positions differ, frame {f}, body {b}"
                assert np.array_equal(bits(nd["vel"]), bits(g[f"vel_f{f}_b{b}"])), f"{name}: velocities differ, frame {f}, body {b}"
    for b in range(len(rig["bodies"])):
        bm = world.beams(b)
        for k in ("L", "max_pos", "max_neg", "strength", "stress"):
            assert np.array_equal(bits(bm[k]), bits(g[f"beam_{k}_b{b}"])), f"{name}: beam {k} differs, body {b}"
        assert np.array_equal(bm["flags"], g[f"beam_flags_b{b}"])
        st = world.body(b)
        ref = g[f"body_b{b}"]
        assert st["max_speed"] == ref[6] and st["static_contacts"] == ref[8] and st["broken_beams"] == ref[9]
        assert np.array_equal(bits(st["aabb_min"]), bits(ref[0:3])) and np.array_equal(bits(st["aabb_max"]), bits(ref[3:6]))


@pytest.mark.parametrize("name", sorted(CASES))
def test_port_matches_golden(port_lib, name):
    from oracle.oracle import PortWorld, build_world
    run_against_golden(build_world(PortWorld, CASES[name]()), name)


def test_golden_fixtures_exercise_every_branch():
    """The fixtures cover yield, breaks (normal and support beams), and contact on every kind of static."""
    g = golden("stress_rig_s7")
    broken = sum(int((g[f"beam_flags_b{b}"] & 1).sum()) for b in range(3))
    assert broken > 10
    t = golden("truss_car_s1")
    assert float(t["body_b0"][6]) > 0 and int(t["body_b0"][8]) > 0  # moving, on the ground at the end


@pytest.mark.parametrize("make", [lambda: rigs.truss_car(2, speed=30.0), lambda: rigs.stress_rig(11),
                                  lambda: rigs.fleet(6, seed=5, median_nodes=300, min_nodes=60, max_nodes=900,
                                                     terrain_size=300.0, terrain_samples=257, skins=False,
                                                     wheels=False)])
def test_port_matches_reference_live(port_lib, ref_lib, make):
    from oracle.oracle import PortWorld, RefWorld, build_world
    rig = make()
    ref = build_world(RefWorld, rig, multithreaded=False)
    port = build_world(PortWorld, rig)
    for f in range(40):
        n = 20 + (f % 3)  # uneven frames: the static query's margin depends on the frame's length
        ref.step_substeps(n)
        port.step_substeps(n)
    for b in range(len(rig["bodies"])):
        a, c = ref.nodes(b), port.nodes(b)
        assert np.array_equal(bits(a["pos"]), bits(c["pos"])) and np.array_equal(bits(a["vel"]), bits(c["vel"]))
        assert np.array_equal(a["inv_mass"], c["inv_mass"])
        ra, rc = ref.body(b), port.body(b)
        assert ra["max_speed"] == rc["max_speed"] and ra["sleeping"] == rc["sleeping"]
        assert ra["broken_beams"] == rc["broken_beams"] and ra["static_contacts"] == rc["static_contacts"]


def test_port_sleep_matches_reference(port_lib, ref_lib):
    """A body left at rest on the ground falls asleep in the same frame in both."""
    from oracle.oracle import PortWorld, RefWorld, build_world
    rig = rigs.truss_car(3, speed=0.0, dims=(4, 2, 2))
    ref = build_world(RefWorld, rig, multithreaded=False)
    port = build_world(PortWorld, rig)
    asleep_at = [None, None]
    for f in range(150):
        for i, w in enumerate((ref, port)):
            w.step_substeps(33)
            if asleep_at[i] is None and w.body(0)["sleeping"]:
                asleep_at[i] = f
    assert asleep_at[0] is not None and asleep_at[0] == asleep_at[1]
    assert np.array_equal(bits(ref.nodes(0)["pos"]), bits(port.nodes(0)["pos"]))


def test_port_repair_matches_reference(port_lib, ref_lib):
    """A node made non-finite between frames is repaired onto its neighbours' mean (World::repair_nodes)."""
    from oracle.oracle import PortWorld, RefWorld, build_world
    rig = rigs.truss_car(4, speed=5.0, dims=(6, 3, 3))
    ws = [build_world(RefWorld, rig, multithreaded=False), build_world(PortWorld, rig)]
    for w in ws:
        w.step_substeps(20)
        nd = w.nodes(0)
        pos, vel = nd["pos"].copy(), nd["vel"].copy()
        pos[7] = np.nan
        vel[11] = (500.0, 0.0, 0.0)
        w.set_nodes(0, pos, vel)
        w.step_substeps(20)
        w.step_substeps(20)
    a, c = ws[0].nodes(0), ws[1].nodes(0)
    assert np.all(np.isfinite(a["pos"]))
    assert np.array_equal(bits(a["pos"]), bits(c["pos"])) and np.array_equal(bits(a["vel"]), bits(c["vel"]))


def test_portable_exp_pow_within_one_ulp_of_libm(port_lib):
    """The oracle's exp / pow (which the GPU evaluates identically) against libm's expf / powf: at most 1 ulp apart."""
    import ctypes as C
    lib = C.CDLL(port_lib)
    lib.orc_math_exp.argtypes, lib.orc_math_exp.restype = [C.c_float], C.c_float
    lib.orc_math_pow.argtypes, lib.orc_math_pow.restype = [C.c_float, C.c_float], C.c_float
    libm = C.CDLL("libm.so.6")
    libm.expf.argtypes, libm.expf.restype = [C.c_float], C.c_float
    libm.powf.argtypes, libm.powf.restype = [C.c_float, C.c_float], C.c_float
    rng = np.random.default_rng(0)
    xs = np.concatenate([-rng.exponential(3.0, 20000), rng.uniform(-80, 80, 5000), [0.0, -0.0, 1e-30, -87.0, 88.0]])
    worst = 0
    for x in xs.astype(np.float32):
        a, b = np.float32(lib.orc_math_exp(float(x))), np.float32(libm.expf(float(x)))
        worst = max(worst, abs(int(np.int32(a.view(np.int32))) - int(np.int32(b.view(np.int32)))))
    assert worst <= 1
    worst = 0
    for x, y in zip(rng.uniform(0, 20, 20000).astype(np.float32), rng.choice([2.0, 1.5, 0.5, 3.0], 20000).astype(np.float32)):
        a, b = np.float32(lib.orc_math_pow(float(x), float(y))), np.float32(libm.powf(float(x), float(y)))
        worst = max(worst, abs(int(np.int32(a.view(np.int32))) - int(np.int32(b.view(np.int32)))))
    assert worst <= 1
    assert lib.orc_math_pow(0.0, 2.0) == 0.0 and lib.orc_math_pow(3.0, 0.0) == 1.0


def test_port_within_tolerance_of_reference_with_libm(port_lib):
    """Against the reference as it runs (libm's exp / pow): the truss car's nodes within 1e-4 m after 2,000 substeps."""
    from oracle.oracle import PortWorld, RefWorld, build_world, ref_available
    if not ref_available("libm"):
        pytest.skip("the compiled reference (oracle/_ref) is not present")
    rig = rigs.truss_car(1)
    ref = build_world(RefWorld, rig, flavour="libm", multithreaded=False)
    port = build_world(PortWorld, rig)
    for _ in range(100):
        ref.step_substeps(20)
        port.step_substeps(20)
    d = np.abs(ref.nodes(0)["pos"].astype(np.float64) - port.nodes(0)["pos"]).max()
    assert d <= 1e-4, d


@pytest.mark.parametrize("name", ["crash_slow_s1", "crash_hull_s4"])
def test_reference_contact_fixture_reproduces(ref_lib, name):
    """The contact fixtures come from the reference: it gives them again (pairs each frame, node states), and the
    pairs are valid (node, triangle) indices of the two bodies."""
    import importlib.util
    import os
    spec = importlib.util.spec_from_file_location("mgc", os.path.join(os.path.dirname(__file__), "golden", "make_golden_contacts.py"))
    mgc = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mgc)
    d = mgc.generate(name)
    g = golden(name)
    assert set(d) == set(g)
    for k in g:
        assert np.array_equal(d[k], g[k]), k
    rig = mgc.CASES[name]()
    for f in range(len(g["frames"])):
        p = g[f"pairs_f{f}"]
        if len(p):
            assert set(np.unique(p[:, 0])) <= {0, 1} and np.all(p[:, 0] != p[:, 2])
            for row in p:
                assert row[1] < len(rig["bodies"][row[0]]["mass"]) and row[3] < len(rig["bodies"][row[2]]["tris"])
