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


def test_gpu_dense_front_agrees_with_block_columns():
    """The multifrontal factorization, the top chain factored as one dense front, and block column by block column in
    the reference's order: the same system solved in other orders of sums, so the plate's nodes agree far inside the
    tolerance after 60 substeps, and every solution's residual is at rounding level."""
    runs = []
    for dense in (0, 1, 2):
        w = world_from_rig(rigs.shell_plate(20, seed=3), fem_dense_front=dense, fem_check_residual=True)
        for _ in range(3):
            w.step_substeps(20)
        runs.append((np.ascontiguousarray(w.bodies()[0].nodes()["p"]).astype(np.float64), w.fem_stats()["max_residual"]))
        assert w.bodies()[0].state()["fem_failures"] == 0
        w.close()
    for r in runs[1:]:
        assert np.abs(r[0] - runs[0][0]).max() < 1e-9
    assert all(r[1] < 1e-11 for r in runs)


@pytest.mark.parametrize("make", [
    lambda: rigs.frame_ladder(12, joints=[(0, 0), (1, 0), (2, 3), (4, 4), (5, 5), (0, 1)]),
    lambda: rigs.plate_with_rails(12, tris_first=True),
    lambda: rigs.plate_with_rails(12, tris_first=False)])
def test_gpu_frame_members_match_reference(ref_lib, make):
    """Frames with members (elastic tubes, every kind of joint; alone and stiffening a shell plate) stepped 400
    substeps under gravity and a point load on the GPU and by the compiled reference: the nodes within the FEM
    tolerance, no failed factorization, no clamp."""
    from oracle.oracle import RefWorld, build_world
    rig = make()
    w = world_from_rig(rig)
    ref = build_world(RefWorld, rig, multithreaded=False)
    h = w.bodies()[0]
    p0 = np.ascontiguousarray(h.nodes()["p"]).astype(np.float64)
    for f in range(20):
        w.step_substeps(20)
        ref.step_substeps(20)
        if f in (0, 4, 19):
            p = np.ascontiguousarray(h.nodes()["p"]).astype(np.float64)
            r = ref.nodes(0)["pos"].astype(np.float64)
            d = np.abs(p - r).max()
            assert d <= TOL, f"frame {f}: max |dp| {d:.3g} m"
    assert np.abs(p - p0).max() > 1e-3  # (it moves)
    st = h.state()
    assert st["fem_failures"] == 0 and st["fem_clamps"] == 0
    assert ref.fem_info(0)["solve_failures"] == 0
    w.close()


def test_gpu_shell_body_matches_reference(ref_lib):
    """The box-and-pillar shell body (six welded panels of 0.8-2 mm steel, spot welds every other edge node, tube
    pillars; 1,678 nodes, 2,944 triangles, 152 members) under gravity and two point loads, floating: 100 substeps on
    the GPU and by the compiled reference within the FEM tolerance."""
    from oracle.oracle import RefWorld, build_world
    rig = rigs.shell_body(1500)
    w = world_from_rig(rig)
    ref = build_world(RefWorld, rig, multithreaded=False)
    h = w.bodies()[0]
    p0 = np.ascontiguousarray(h.nodes()["p"]).astype(np.float64)
    for f in range(5):
        w.step_substeps(20)
        ref.step_substeps(20)
    p = np.ascontiguousarray(h.nodes()["p"]).astype(np.float64)
    d = np.abs(p - ref.nodes(0)["pos"]).max()
    assert d <= TOL, f"max |dp| {d:.3g} m"
    assert np.abs(p - p0).max() > 1e-3  # (it moves)
    assert h.state()["fem_failures"] == 0 and ref.fem_info(0)["solve_failures"] == 0
    w.close()


def test_gpu_large_shell_body_multifrontal_matches_reference(ref_lib):
    """The shell body at 5,384 nodes (10,024 triangles, 344 members; 4.9 M block updates a factorization by the
    reference's column-by-column Cholesky) factored by the multifrontal path: 60 substeps under gravity and two point
    loads within the FEM tolerance (1e-4 m) of the compiled reference, every solution's relative residual at most 1e-6
    (measured against the assembled system kept aside), no failed factorization on either side."""
    from oracle.oracle import RefWorld, build_world
    rig = rigs.shell_body(5000)
    w = world_from_rig(rig, fem_dense_front=2, fem_check_residual=True)
    ref = build_world(RefWorld, rig, multithreaded=False)
    h = w.bodies()[0]
    p0 = np.ascontiguousarray(h.nodes()["p"]).astype(np.float64)
    for f in range(3):
        w.step_substeps(20)
        ref.step_substeps(20)
    p = np.ascontiguousarray(h.nodes()["p"]).astype(np.float64)
    d = np.abs(p - ref.nodes(0)["pos"]).max()
    fs = w.fem_stats()
    assert fs["fronts"] > 0 and fs["columns"] > 5000
    assert d <= TOL, f"max |dp| {d:.3g} m"
    assert fs["max_residual"] <= 1e-6, fs["max_residual"]
    assert np.abs(p - p0).max() > 1e-4  # (it moves)
    assert h.state()["fem_failures"] == 0 and ref.fem_info(0)["solve_failures"] == 0
    w.close()


def test_gpu_yielding_plate_matches_reference(ref_lib):
    """A plate of a yielding section (250 MPa) under a 3 kN point load, on a body that deforms and does not break:
    its membrane flows (the rest shapes follow the stretch, the elements built again) and its bending yields (the
    corners' rest frames turn) in the reference's eval_tris (frame_fem.cpp:1690-1741); on the GPU the same triangles
    flow, the same triangles flow, the rest shapes and plastic stretches agree. The flow amplifies the kinematics'
    last-bit differences (atan2 / sin / cos, the substitutions' order of sums) smoothly - 1e-6 m after 100 substeps,
    1e-5 m after 120 as the flow spreads - so the nodes are held to the FEM tolerance (1e-4 m) over 140 substeps and to
    1e-4 of the plate's 1.8 m motion (1.8e-4 m) over 200."""
    from oracle.oracle import RefWorld, build_world
    rig = rigs.shell_plate(20, yield_stress=2.5e8, load=3000.0, seed=2)
    w = world_from_rig(rig)
    ref = build_world(RefWorld, rig, multithreaded=False)
    h = w.bodies()[0]
    X0 = h.fem_tris()["X"].copy()
    p0 = np.ascontiguousarray(h.nodes()["p"]).astype(np.float64)
    for f in range(10):
        w.step_substeps(20)
        ref.step_substeps(20)
        p = np.ascontiguousarray(h.nodes()["p"]).astype(np.float64)
        d = np.abs(p - ref.nodes(0)["pos"]).max()
        lim = TOL if f <= 6 else 1e-4 * np.abs(p - p0).max()
        assert d <= lim, f"frame {f}: max |dp| {d:.3g} m"
        g, r = h.fem_tris(), ref.fem_tris(0)
        assert np.array_equal((g["X"] != X0).any(1), (r["X"] != X0).any(1)), f"frame {f}: other triangles flowed"
    assert (r["X"] != X0).any(1).sum() > 100 and np.abs(p - p0).max() > 1.0
    assert np.abs(g["X"] - r["X"]).max() <= 1e-5
    assert np.abs(g["dmg"] - r["dmg"]).max() <= 1e-4 and r["dmg"].max() > 1e-3
    st = h.state()
    assert st["fem_failures"] == 0 and st["fem_clamps"] == 0
    w.close()


def test_gpu_yielding_section_on_a_breaking_body_is_refused():
    """Tears and bisections of a yielding plate are topology events this path does not make: refused at add_body."""
    from beamlab_b200.world import BeamLabError
    rig = rigs.shell_plate(8, yield_stress=2.5e8)
    rig["bodies"][0]["params"]["allow_break"] = 1
    with pytest.raises(BeamLabError, match="unsupported"):
        world_from_rig(rig)


@pytest.mark.parametrize("load,joints", [(1500.0, None), (3000.0, None), (3000.0, [(0, 0), (1, 0), (2, 3), (4, 4), (5, 5), (0, 1)])])
def test_gpu_yielding_frame_matches_reference(ref_lib, load, joints):
    """A ladder of yielding steel tubes (250 MPa: axial yield and Euler buckling, twist, hardening radial-return hinges
    at the ends, the plastic rotations baked into the rest frames - eval_forces, frame_fem.cpp:1915-2054) on a body
    that deforms and does not break, loaded past its plastic moment: the tangent of the parts that flow, and where the
    step unloads one, its elastic tangent and the step again (frame_fem.cpp:2959-2995). 400 substeps on the GPU and by
    the reference: the nodes within the FEM tolerance as the ladder folds metres; re-passes ran on both sides."""
    from oracle.oracle import RefWorld, build_world
    rig = rigs.frame_ladder(12, load=load, joints=joints, section=rigs.tube_section(yield_stress=2.5e8))
    w = world_from_rig(rig)
    ref = build_world(RefWorld, rig, multithreaded=False)
    h = w.bodies()[0]
    p0 = np.ascontiguousarray(h.nodes()["p"]).astype(np.float64)
    for f in range(20):
        w.step_substeps(20)
        ref.step_substeps(20)
        if f in (4, 9, 19):
            p = np.ascontiguousarray(h.nodes()["p"]).astype(np.float64)
            d = np.abs(p - ref.nodes(0)["pos"]).max()
            assert d <= TOL, f"frame {f}: max |dp| {d:.3g} m"
    assert np.abs(p - p0).max() > 1.0
    ref_repasses = ref.fem_info(0)["passes"] - 400
    assert ref_repasses > 0 and w.fem_stats()["repasses"] == ref_repasses
    st = h.state()
    assert st["fem_failures"] == 0 and st["fem_clamps"] == 0
    w.close()


def test_gpu_yielding_frame_graphs_equal_launches():
    """The re-passes under IF nodes of the frame's graph and, launched one by one, always run (solving the same system
    again where no hinge unloaded): the same bits."""
    rig = rigs.frame_ladder(12, load=3000.0, section=rigs.tube_section(yield_stress=2.5e8))
    ws = [world_from_rig(rig), world_from_rig(rig, graphs=False)]
    for _ in range(12):
        for w in ws:
            w.step_substeps(20)
    a, b = (np.ascontiguousarray(w.bodies()[0].nodes()["p"]) for w in ws)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert ws[0].fem_stats()["repasses"] > 0
    for w in ws:
        w.close()


def test_gpu_frame_on_ground_matches_reference(ref_lib):
    """A ladder frame of members dropped onto flat grass: its nodes' static contacts (World::collide_static's
    primitive_collision into the node forces) and the frame step's hold on the pressed nodes (FemFrame::contact_n:
    kappa = 200 m along the normal, and along the ground where a node sticks - gather_part, frame_fem.cpp:1043-1064),
    the landing, the bounce and the settling: the nodes within the FEM tolerance of the reference over 600 substeps."""
    from oracle.oracle import RefWorld, build_world
    rig = rigs.frame_ladder(12, origin=(0.0, 0.3, 0.0), load=300.0, ground=True)
    w = world_from_rig(rig)
    ref = build_world(RefWorld, rig, multithreaded=False)
    h = w.bodies()[0]
    touched = 0
    for f in range(30):
        w.step_substeps(20)
        ref.step_substeps(20)
        touched = max(touched, ref.body(0)["static_contacts"])
        if f in (9, 14, 19, 29):
            p = np.ascontiguousarray(h.nodes()["p"]).astype(np.float64)
            d = np.abs(p - ref.nodes(0)["pos"]).max()
            assert d <= TOL, f"frame {f}: max |dp| {d:.3g} m"
    assert touched > 0 and np.abs(p[:, 1]).max() < 0.2  # (it landed)
    st = h.state()
    assert st["fem_failures"] == 0 and st["fem_clamps"] == 0
    w.close()


def test_gpu_plastic_state_survives_a_recommit():
    """A body added while a yielding ladder folds and a yielding plate flows (the context commits again, pulling the
    members' plastic state and rest frames, the re-passes' budget, the triangles' rest shapes, frames, stiffnesses and
    plastic rotations back from the device): both frames go on bitwise as in a world that never committed again."""
    from beamlab_b200.world import SoftBody
    lad = rigs.frame_ladder(12, load=3000.0, section=rigs.tube_section(yield_stress=2.5e8))
    pl = rigs.shell_plate(12, yield_stress=2.5e8, load=3000.0, seed=2, origin=(0.0, 1.0, 5.0))
    rig = {"settings": lad["settings"], "statics": {}, "bodies": lad["bodies"] + pl["bodies"]}
    ws = [world_from_rig(rig), world_from_rig(rig)]
    for f in range(14):
        if f == 6:
            extra = rigs.truss_car(4, speed=0.0, dims=(4, 2, 2))["bodies"][0]
            extra["pos"][:, 2] += 30.0
            ws[1].add_body(SoftBody.from_arrays(extra, name="extra"))
        for w in ws:
            w.step_substeps(20)
    for b in (0, 1):
        x, y = (np.ascontiguousarray(w.bodies()[b].nodes()["p"]) for w in ws)
        assert np.array_equal(x.view(np.uint32), y.view(np.uint32)), f"body {b}"
    assert ws[1].fem_stats()["repasses"] > 0
    assert (ws[1].bodies()[1].fem_tris()["dmg"] > 0).any()
    for w in ws:
        w.close()
