"""The FEM shell frame's symbolic phase against the reference, bit for bit: the frame node numbering, the exact
minimum-degree elimination order, the factor's column patterns, every block update with its target, the triangles'
rest shapes (bl_fem_pattern, host only); and the plate rig's node arrays against the reference's own ShellMesher."""
import ctypes as C

import numpy as np
import pytest

from beamlab_b200 import SoftBody, _lib, rigs
from beamlab_b200.world import FEM_MEMBER_DTYPE, FEM_TRI_DTYPE, _FemDesc, _FrameSection, _ShellSection
from conftest import golden


def pattern(rig):
    sb = SoftBody.from_arrays(rig["bodies"][0])
    s = rig["bodies"][0]["fem_sections"][0]
    secs = (_ShellSection * 1)(_ShellSection(s["E"], s["nu"], s["rho"], s["t"], 0.0, s["damping"], s["drill"]))
    tris = np.ascontiguousarray(sb.fem_tris, FEM_TRI_DTYPE)
    fd = _FemDesc(1, C.cast(secs, C.c_void_p), len(tris), tris.ctypes.data, 0.5, 0.02)
    L = _lib.lib()
    sizes = (C.c_int32 * 4)()
    assert L.bl_fem_pattern(sb.nodes.ctypes.data, sb.info.ctypes.data, len(sb.nodes), C.byref(fd), sizes, *([None] * 6)) == 0
    nf, nb, nu, nc = list(sizes)
    out = {"perm": np.zeros(nf, np.int32), "col_ptr": np.zeros(nf + 1, np.int32), "row": np.zeros(nb, np.int32),
           "upd": np.zeros(3 * nu, np.int32), "rest": np.zeros((len(tris), 6), np.float32),
           "inertia": np.zeros(nf, np.float32)}
    assert L.bl_fem_pattern(sb.nodes.ctypes.data, sb.info.ctypes.data, len(sb.nodes), C.byref(fd), sizes,
                            *(out[k].ctypes.data for k in ("perm", "col_ptr", "row", "upd", "rest", "inertia"))) == 0
    out["components"] = nc
    return sb, out


@pytest.mark.parametrize("n", [5, 20, 63])
def test_fem_pattern_matches_reference(ref_lib, n):
    from oracle.oracle import RefWorld, build_world
    rig = rigs.shell_plate(n)
    ref = build_world(RefWorld, rig, multithreaded=False)
    rp, rt = ref.fem_pattern(0), ref.fem_tris(0)
    sb, mine = pattern(rig)
    for k in ("perm", "col_ptr", "row", "upd"):
        assert np.array_equal(mine[k], rp[k]), k
    assert np.array_equal(mine["rest"].view(np.uint32), rt["X"].view(np.uint32))
    assert mine["components"] == ref.fem_info(0)["components"] == 1
    rn = ref.nodes(0)
    assert np.array_equal(rn["pos"].view(np.uint32), np.ascontiguousarray(sb.nodes["p"]).view(np.uint32))
    assert np.array_equal(rn["mass"].view(np.uint32), sb.nodes["mass"].view(np.uint32))
    assert np.array_equal(rn["inv_mass"], sb.nodes["inv_mass"])


def test_plate_rig_shape():
    rig = rigs.shell_plate(63)
    b = rig["bodies"][0]
    assert len(b["mass"]) == 4096 and len(b["fem_tris"]) == 7938
    assert np.count_nonzero(b["node_flags"] & 2) == 64  # the clamped edge
    m = float(b["mass"].astype(np.float64).sum())
    assert abs(m - 7850 * 0.0015 * 1.0) < 1e-3 * m  # 11.8 kg of steel
    (node, f), = b["loads"]
    assert abs(np.linalg.norm(f) - 500.0) < 1e-3 and not (b["node_flags"][node] & 2)


def test_plate_golden_fixture_is_sane():
    g = golden("plate20_s1")
    assert int(g["solve_failures"]) == 0 and int(g["clamps"]) == 0
    p0, p1 = g["pos_f1"], g["pos_f20"]
    assert np.all(np.isfinite(p1)) and float(np.abs(p1 - p0).max()) > 1e-4  # the plate moves under its load


def frame_pattern(rig):
    """bl_fem_pattern of a body with members (and triangles): perm, col_ptr, row, upd, inertia."""
    body = rig["bodies"][0]
    sb = SoftBody.from_arrays(body)
    ss = [(_ShellSection(x["E"], x["nu"], x["rho"], x["t"], 0.0, x["damping"], x["drill"])) for x in body.get("fem_sections", [])]
    secs = (_ShellSection * max(len(ss), 1))(*ss)
    keys = ("E", "G", "rho", "A", "Iy", "Iz", "J", "As_y", "As_z", "damping", "axial", "joint_k", "Np", "Mp", "Tp")
    fs = (_FrameSection * len(body["frame_sections"]))(*[_FrameSection(*[float(d.get(k, 0.0)) for k in keys]) for d in body["frame_sections"]])
    tris = np.ascontiguousarray(sb.fem_tris, FEM_TRI_DTYPE)
    mems = np.ascontiguousarray(sb.fem_members, FEM_MEMBER_DTYPE)
    fd = _FemDesc(len(ss), C.cast(secs, C.c_void_p), len(tris), tris.ctypes.data if len(tris) else None, 0.5, 0.02,
                  len(body["frame_sections"]), C.cast(fs, C.c_void_p), len(mems), mems.ctypes.data, int(sb.fem_tris_first))
    L = _lib.lib()
    sizes = (C.c_int32 * 4)()
    assert L.bl_fem_pattern(sb.nodes.ctypes.data, sb.info.ctypes.data, len(sb.nodes), C.byref(fd), sizes, *([None] * 6)) == 0
    nf, nb, nu, nc = list(sizes)
    out = {"perm": np.zeros(nf, np.int32), "col_ptr": np.zeros(nf + 1, np.int32), "row": np.zeros(nb, np.int32),
           "upd": np.zeros(3 * nu, np.int32), "rest": np.zeros((max(len(tris), 1), 6), np.float32), "inertia": np.zeros(nf, np.float32)}
    assert L.bl_fem_pattern(sb.nodes.ctypes.data, sb.info.ctypes.data, len(sb.nodes), C.byref(fd), sizes,
                            *(out[k].ctypes.data for k in ("perm", "col_ptr", "row", "upd", "rest", "inertia"))) == 0
    return out


@pytest.mark.parametrize("make", [
    lambda: rigs.frame_ladder(12, joints=[(0, 0), (1, 0), (2, 3), (4, 4), (5, 5), (0, 1)]),
    lambda: rigs.plate_with_rails(12, tris_first=True),
    lambda: rigs.plate_with_rails(12, tris_first=False),
    lambda: rigs.shell_body(1500)])
def test_frame_members_pattern_matches_reference(ref_lib, make):
    """Frames with members (FemFrame::add_element): the same frame node numbering, ordering, factor pattern and update
    list as the reference's, bit for bit - members alone with every kind of joint, and members with triangles added in
    either order."""
    from oracle.oracle import RefWorld, build_world
    rig = make()
    ref = build_world(RefWorld, rig, multithreaded=False)
    rp = ref.fem_pattern(0)
    mine = frame_pattern(rig)
    for k in ("perm", "col_ptr", "row", "upd"):
        assert np.array_equal(mine[k], rp[k]), k
    rn = ref.fem_nodes(0)
    sb = SoftBody.from_arrays(rig["bodies"][0])
    assert np.array_equal(sb.nodes["p"][rn["node"]].astype(np.float64), rn["xd"])  # (the same frame node numbering)
