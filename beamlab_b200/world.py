"""Python host mirror of BeamLab's physics step API over the C ABI (include/beamlab_gpu.h).

Names, argument meaning and defaults follow the reference's ``bl::phys`` classes, so code written against them reads
the same here:

* ``WorldSettings``   - WorldSettings (src/phys/world.h:24-77), the fields the path reads
* ``StaticWorld``     - StaticWorld (src/phys/static_world.h:182-201): terrain, add_box, build_grid, kill_y
* ``SoftBody``        - a SoftBody under construction: add_node / add_beam / finalize (src/phys/softbody.cpp:8-83)
* ``World``           - World (src/phys/world.h:150-171): add_body, step_substeps, step_frame, stats
* ``BodyHandle``      - what World.add_body returns (the reference's SoftBody* owned by the World): state read-back

Everything is computed by the CUDA library; this module only describes rigs and moves arrays. Without the built
library (or without an sm_100 GPU) World() raises - there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib

# == bl_node / bl_node_info / bl_beam (include/beamlab_gpu.h) == the reference's Node / NodeInfo / Beam
NODE_DTYPE = np.dtype([("p", "<f4", 3), ("inv_mass", "<f4"), ("v", "<f4", 3), ("mass", "<f4")])
NODE_INFO_DTYPE = np.dtype([("flags", "<u2"), ("surface", "u1"), ("pad", "u1"), ("friction", "<f4"), ("radius", "<f4"),
                            ("frame", "<i4"), ("ror_id", "<i4")])
BEAM_DTYPE = np.dtype([("a", "<u4"), ("b", "<u4"), ("L", "<f4"), ("k", "<f4"), ("d", "<f4"), ("max_pos", "<f4"),
                       ("max_neg", "<f4"), ("strength", "<f4"), ("plastic", "<f4"), ("stress", "<f4"), ("L0", "<f4"),
                       ("support_limit", "<f4"), ("type", "u1"), ("flags", "u1"), ("group", "<u2")])
# == bl_tri == the reference's Triangle (softbody.h:138-147)
TRI_DTYPE = np.dtype([("a", "<u4"), ("b", "<u4"), ("c", "<u4"), ("surface", "u1"), ("two_sided", "u1"), ("torn", "u1"),
                      ("pad", "u1"), ("rest_edge2", "<f4")])
assert NODE_DTYPE.itemsize == 32 and NODE_INFO_DTYPE.itemsize == 20 and BEAM_DTYPE.itemsize == 52
assert TRI_DTYPE.itemsize == 20

NF_GROUND, NF_FIXED, NF_CONTACTER = 1, 2, 16
BF_BROKEN, BF_SHOCK = 1, 64


class BeamLabError(RuntimeError):
    """A C-ABI call returned a negative BL_GPU_E* code."""


def _check(rc: int, what: str, ctx=None):
    if rc != 0:
        msg = _lib.lib().bl_gpu_error_string(rc).decode()
        extra = ""
        if ctx is not None and rc == -3:
            extra = f" (cuda error {_lib.lib().bl_gpu_last_cuda_error(ctx)})"
        raise BeamLabError(f"{what}: {msg} [{rc}]{extra}")


@dataclass
class WorldSettings:
    """WorldSettings (world.h:24-77): the fields of the explicit substep."""
    gravity: tuple = (0.0, -9.81, 0.0)
    dt: float = 0.0005
    sleeping: bool = True
    sleep_speed: float = 0.06
    sleep_time: float = 1.0
    collision_hz: float = 120.0
    inter_body_collisions: bool = True
    max_pairs: int = 0                        # the contact pair list's capacity (0: the library's default, 2^21)
    # the FEM frames' implicit step (no counterpart in the reference, which always factors): "cholesky", "pcg",
    # "pcg_learned", "pcg_previous"; a PCG solve that misses pcg_tol within pcg_max_iters falls back to the Cholesky
    fem_solver: str = "cholesky"
    pcg_max_iters: int = 200
    pcg_tol: float = 1e-6
    fem_check_residual: bool = False
    pcg_learned_scale: bool = False
    # True: each frame captured once as a CUDA graph and replayed; False: its kernels launched one by one (plain path)
    graphs: bool = True
    # the beams' kernel: 0 streams the beam arrays by bulk (TMA) copies, 1 plain loads (the same results)
    beam_kernel: int = 0
    # the FEM factorization: 3 by size (1 up to 8 M block updates, else 2), 2 multifrontal (dense fronts, level by level
    # of the front tree), 1 block columns with the top chain as one dense front, 0 block columns in the reference's order
    fem_dense_front: int = 3
    tyre_grip: float = 1.0                    # WorldSettings::tyre_grip: a factor on the tyres' friction
    bulk_wait_s: float = 1.0                  # the beams kernel's bound on a wait for its bulk copies (0: runs out)
    contact_whole_max: int = 6144             # an island's contacts run whole up to this many, else 512 at a time
    # launch shapes (None: the tuned ones of beamlab_b200/tuned.json when present, else the library's defaults);
    # results do not depend on them
    force_block: int | None = None
    integrate_block: int | None = None
    beams_per_sm: int | None = None


@dataclass
class StaticWorld:
    """StaticWorld (static_world.h:182-201): a heightfield, boxes, vertical cylinders. Boxes are candidates for
    contact only after build_grid(), as in the reference."""
    terrain: dict | None = None
    boxes: list = field(default_factory=list)
    cylinders: list = field(default_factory=list)
    grid_built: bool = False
    kill_y: float = -200.0

    def create_terrain(self, nx: int, nz: int, cell: float, origin=(0.0, 0.0), heights=None, surfaces=None):
        """Heightfield::create (static_world.cpp:147-152) + the heights and surfaces (nz rows of nx, x fastest)."""
        h = np.zeros((nz, nx), np.float32) if heights is None else np.asarray(heights, np.float32).reshape(nz, nx)
        s = np.zeros((nz, nx), np.uint8) if surfaces is None else np.asarray(surfaces, np.uint8).reshape(nz, nx)
        self.terrain = {"nx": nx, "nz": nz, "cell": cell, "origin": tuple(origin), "heights": h, "surfaces": s}

    def add_box(self, center, half, rot=(0.0, 0.0, 0.0, 1.0), surface: int = 3, max_force: float = 0.0):
        """StaticWorld::add_box (static_world.cpp:298-306); rot is a quaternion (x, y, z, w)."""
        self.boxes.append({"center": tuple(center), "half": tuple(half), "rot": tuple(rot), "surface": surface,
                           "max_force": max_force})

    def add_cylinder(self, base, radius: float, height: float, surface: int = 3):
        self.cylinders.append({"base": tuple(base), "radius": radius, "height": height, "surface": surface})

    def build_grid(self):
        """StaticWorld::build_grid (static_world.cpp:308-338)."""
        self.grid_built = True


def _dist32(pa: np.ndarray, pb: np.ndarray) -> np.ndarray:
    """distance(a, b) in float32, in math.h's order: sqrt((dx*dx + dy*dy) + dz*dz)."""
    d = (pa - pb).astype(np.float32)
    l2 = (d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1]) + d[..., 2] * d[..., 2]
    return np.sqrt(l2.astype(np.float32))


class SoftBody:
    """A soft body under construction (SoftBody, softbody.h:595-1119): nodes, beams and the explicit path's knobs."""

    def __init__(self, name: str = ""):
        self.name = name
        self._nodes: list = []
        self._info: list = []
        self._beams: list = []
        self.ground_friction = 1.0
        self.bounce = -1.0
        self.contact_push_max = 2.0
        self.contact_slop = 0.0
        self.collision_radius = 0.05
        self.allow_deform = True
        self.allow_break = True
        self.ductile = False
        self.can_sleep = True
        self.sleep_speed = 0.0
        # contacts with other bodies (softbody.h:614-721)
        self.contact_friction = 1.0
        self.hull_depth = 0.3
        self.face_skin = 0.002
        self.faces_only = False
        self.collision_group = 0
        self.self_collision = False
        self.air_drag = 0.0                           # SoftBody::air_drag (RoR's per-node drag, against the part's mean)
        self.aero_cda = 0.0                           # SoftBody::aero_cda (Cd A on the parts' mean velocities)
        self.wheels: list[dict] = []                  # Wheel: axle0, axle1, nodes (even: axle0's ring), radius, width, mass
        self.shocks: list[dict] = []                  # Shock: beam, type, soft_bump and the rates of SHOCK_KEYS
        self._tris: list = []
        self.tris = np.zeros(0, TRI_DTYPE)
        self.nodes = np.zeros(0, NODE_DTYPE)
        self.info = np.zeros(0, NODE_INFO_DTYPE)
        self.beams = np.zeros(0, BEAM_DTYPE)
        # FEM frame of triangle elements (FemFrame: add_shell_section / add_tri)
        self.fem_sections: list[dict] = []
        self.fem_tris = np.zeros(0, FEM_TRI_DTYPE)
        self.frame_sections: list[dict] = []           # FrameSection fields (frame_fem.h:90-112) by name
        self.fem_members = np.zeros(0, FEM_MEMBER_DTYPE)
        self.fem_tris_first = False                   # the add_tri calls before the add_element calls
        self.fem_theta = 0.5
        self.fem_dissipation = 0.02

    def add_node(self, p, mass: float, flags: int = NF_GROUND | NF_CONTACTER, v=(0.0, 0.0, 0.0), friction=1.0,
                 radius=0.0) -> int:
        """SoftBody::add_node (softbody.cpp:8-20): an anchored or massless node has inverse mass 0."""
        m = np.float32(mass)
        inv = np.float32(0.0) if (flags & NF_FIXED) or m <= 0 else np.float32(1.0) / m
        self._nodes.append((tuple(np.float32(x) for x in p), inv, tuple(np.float32(x) for x in v), m))
        self._info.append((flags, 0, 0, np.float32(friction), np.float32(radius), -1, -1))
        return len(self._nodes) - 1

    def add_beam(self, a: int, b: int, k: float, d: float, strength: float = 1e6, deform: float = 4e5,
                 type: int = 0, flags: int = 0) -> int:
        """SoftBody::add_beam (softbody.cpp:22-40)."""
        self._beams.append((a, b, k, d, strength, deform, type, flags))
        return len(self._beams) - 1

    def add_triangle(self, a: int, b: int, c: int, two_sided: bool = True) -> int:
        """SoftBody::add_triangle (softbody.h:958): a collision triangle; two_sided False makes a hull triangle."""
        self._tris.append((a, b, c, bool(two_sided)))
        return len(self._tris) - 1

    @classmethod
    def from_arrays(cls, body: dict, name: str = "") -> "SoftBody":
        """A body from the arrays of beamlab_b200.rigs (the builder calls' arguments), finalized."""
        sb = cls(name)
        n = len(body["mass"])
        nodes = np.zeros(n, NODE_DTYPE)
        nodes["p"] = np.asarray(body["pos"], np.float32)
        nodes["v"] = np.asarray(body["vel"], np.float32)
        m = np.asarray(body["mass"], np.float32)
        nodes["mass"] = m
        fl = np.asarray(body["node_flags"], np.uint16)
        with np.errstate(divide="ignore"):
            inv = np.where(((fl & NF_FIXED) != 0) | (m <= 0), np.float32(0), np.float32(1) / np.where(m > 0, m, 1))
        nodes["inv_mass"] = inv.astype(np.float32)
        info = np.zeros(n, NODE_INFO_DTYPE)
        info["flags"] = fl
        info["friction"] = np.asarray(body["friction"], np.float32)
        info["radius"] = np.asarray(body["radius"], np.float32)
        info["frame"] = -1
        info["ror_id"] = -1
        mb = len(body["k"])
        beams = np.zeros(mb, BEAM_DTYPE)
        ab = np.asarray(body["ab"], np.uint32).reshape(mb, 2)
        beams["a"], beams["b"] = ab[:, 0], ab[:, 1]
        beams["k"] = np.asarray(body["k"], np.float32)
        beams["d"] = np.asarray(body["d"], np.float32)
        beams["strength"] = np.asarray(body["strength"], np.float32)
        dfm = np.asarray(body["deform"], np.float32)
        beams["max_pos"], beams["max_neg"] = dfm, -dfm
        beams["support_limit"] = np.float32(4.0)
        beams["type"] = np.asarray(body["beam_type"], np.uint8)
        beams["flags"] = np.asarray(body["beam_flags"], np.uint8)
        sb.nodes, sb.info, sb.beams = nodes, info, beams
        for k_, v_ in body.get("params", {}).items():
            setattr(sb, k_, v_)
        if "fem_tris" in body:
            sb.fem_sections = list(body["fem_sections"])
            ft = np.zeros(len(body["fem_tris"]), FEM_TRI_DTYPE)
            tri = np.asarray(body["fem_tris"], np.uint32).reshape(-1, 3)
            ft["a"], ft["b"], ft["c"] = tri[:, 0], tri[:, 1], tri[:, 2]
            ft["section"] = np.asarray(body.get("fem_tri_section", np.zeros(len(tri))), np.uint16)
            ft["mass"] = np.asarray(body["fem_tri_mass"], np.float32)
            sb.fem_tris = ft
        if "fem_members" in body:
            sb.frame_sections = list(body["frame_sections"])
            mab = np.asarray(body["fem_members"], np.uint32).reshape(-1, 2)
            fm = np.zeros(len(mab), FEM_MEMBER_DTYPE)
            fm["a"], fm["b"] = mab[:, 0], mab[:, 1]
            fm["section"] = np.asarray(body.get("member_section", np.zeros(len(mab))), np.uint16)
            ends = np.asarray(body.get("member_ends", np.zeros((len(mab), 2))), np.uint8).reshape(-1, 2)
            fm["end_a"], fm["end_b"] = ends[:, 0], ends[:, 1]
            fm["mass"] = np.asarray(body.get("member_mass", np.zeros(len(mab))), np.float32)
            sb.fem_members = fm
            sb.fem_tris_first = bool(body.get("fem_tris_first", False))
        if "wheels" in body:
            sb.wheels = [dict(w) for w in body["wheels"]]
        if "shocks" in body:
            sb.shocks = [dict(x) for x in body["shocks"]]
        if "tris" in body and len(body["tris"]):
            tri = np.asarray(body["tris"], np.uint32).reshape(-1, 3)
            tr = np.zeros(len(tri), TRI_DTYPE)
            tr["a"], tr["b"], tr["c"] = tri[:, 0], tri[:, 1], tri[:, 2]
            tr["two_sided"] = np.asarray(body.get("tri_two_sided", np.ones(len(tri))), np.uint8)
            sb.tris = tr
        sb._finalize_arrays()
        return sb

    def finalize(self):
        """SoftBody::finalize (softbody.cpp:76-83): the node and beam arrays, rest lengths at least 1 mm."""
        n = len(self._nodes)
        nodes = np.zeros(n, NODE_DTYPE)
        info = np.zeros(n, NODE_INFO_DTYPE)
        for i, (p, inv, v, m) in enumerate(self._nodes):
            nodes[i] = (p, inv, v, m)
        for i, t in enumerate(self._info):
            info[i] = t
        beams = np.zeros(len(self._beams), BEAM_DTYPE)
        for j, (a, b, k, d, s, dfm, t, f) in enumerate(self._beams):
            beams[j]["a"], beams[j]["b"] = a, b
            beams[j]["k"], beams[j]["d"], beams[j]["strength"] = k, d, s
            beams[j]["max_pos"], beams[j]["max_neg"] = np.float32(dfm), -np.float32(dfm)
            beams[j]["support_limit"] = 4.0
            beams[j]["type"], beams[j]["flags"] = t, f
        self.nodes, self.info, self.beams = nodes, info, beams
        tr = np.zeros(len(self._tris), TRI_DTYPE)
        for t, (a, b, c, two) in enumerate(self._tris):
            tr[t]["a"], tr[t]["b"], tr[t]["c"], tr[t]["two_sided"] = a, b, c, int(two)
        self.tris = tr
        self._finalize_arrays()

    def _finalize_arrays(self):
        if len(self.beams):
            L = _dist32(self.nodes["p"][self.beams["a"]], self.nodes["p"][self.beams["b"]])
            L = np.where(np.float32(1e-3) < L, L, np.float32(1e-3)).astype(np.float32)  # std::max(1e-3f, len)
            self.beams["L"] = L
            self.beams["L0"] = L
            self.beams["plastic"] = 0
            self.beams["stress"] = 0
        if len(self.tris):  # rest_edge2: max_edge2 of the triangle at finalize (softbody.cpp:80, softbody.h:155)
            p = self.nodes["p"]
            a, b, c = p[self.tris["a"]], p[self.tris["b"]], p[self.tris["c"]]

            def l2(d):
                d = d.astype(np.float32)
                return ((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]).astype(np.float32)
            e0, e1, e2 = l2(b - a), l2(c - b), l2(a - c)
            m12 = np.where(e1 < e2, e2, e1)  # std::max(e1, e2)
            self.tris["rest_edge2"] = np.where(e0 < m12, m12, e0)

    def node_count(self) -> int:
        return len(self.nodes)


class _ShellSection(C.Structure):
    _fields_ = [("E", C.c_float), ("nu", C.c_float), ("rho", C.c_float), ("t", C.c_float), ("yield_", C.c_float),
                ("damping", C.c_float), ("drill", C.c_float)]


FEM_TRI_DTYPE = np.dtype([("a", "<u4"), ("b", "<u4"), ("c", "<u4"), ("section", "<u2"), ("pad", "<u2"), ("mass", "<f4")])


class _FrameSection(C.Structure):
    _fields_ = [(k, C.c_float) for k in ("E", "G", "rho", "A", "Iy", "Iz", "J", "As_y", "As_z", "damping", "axial", "joint_k",
                                         "Np", "Mp", "Tp", "hardening")]


# == bl_fem_member: a member between two body nodes (FemFrame::add_element), its section, the joints at its ends
FEM_MEMBER_DTYPE = np.dtype([("a", "<u4"), ("b", "<u4"), ("section", "<u2"), ("end_a", "u1"), ("end_b", "u1"), ("mass", "<f4")])
FJ_RIGID, FJ_BALL, FJ_HINGE_V, FJ_HINGE_H, FJ_SWIVEL, FJ_ELASTIC = range(6)


class _FemDesc(C.Structure):
    _fields_ = [("n_sections", C.c_int32), ("sections", C.c_void_p), ("n_tris", C.c_int32), ("tris", C.c_void_p),
                ("theta", C.c_float), ("dissipation", C.c_float), ("n_frame_sections", C.c_int32),
                ("frame_sections", C.c_void_p), ("n_members", C.c_int32), ("members", C.c_void_p),
                ("tris_first", C.c_int32)]


class _BodyDesc(C.Structure):
    _fields_ = [("n_nodes", C.c_int32), ("nodes", C.c_void_p), ("info", C.c_void_p), ("n_beams", C.c_int32),
                ("beams", C.c_void_p), ("ground_friction", C.c_float), ("bounce", C.c_float),
                ("contact_push_max", C.c_float), ("contact_slop", C.c_float), ("allow_deform", C.c_int32),
                ("allow_break", C.c_int32), ("ductile", C.c_int32), ("can_sleep", C.c_int32),
                ("sleep_speed", C.c_float), ("max_speed", C.c_float), ("sleeping", C.c_int32),
                ("fem", C.POINTER(_FemDesc)), ("n_tris", C.c_int32), ("tris", C.c_void_p),
                ("collision_radius", C.c_float), ("contact_friction", C.c_float), ("hull_depth", C.c_float),
                ("face_skin", C.c_float), ("faces_only", C.c_int32), ("collision_group", C.c_int32),
                ("self_collision", C.c_int32), ("air_drag", C.c_float), ("aero_cda", C.c_float),
                ("n_wheels", C.c_int32), ("wheels", C.c_void_p), ("n_shocks", C.c_int32), ("shocks", C.c_void_p)]


SHOCK_KEYS = ("spring", "damp", "spring_in", "damp_in", "prog_spring_in", "prog_damp_in", "spring_out", "damp_out",
              "prog_spring_out", "prog_damp_out", "damp_in_slow", "split_in", "damp_in_fast", "damp_out_slow", "split_out",
              "damp_out_fast", "short_bound", "long_bound", "bound_spring", "bound_damp")
SHOCK_DEFAULTS = {"damp_in_slow": 1.0, "split_in": 1.0, "damp_in_fast": 1.0, "damp_out_slow": 1.0, "split_out": 1.0,
                  "damp_out_fast": 1.0, "bound_spring": 9e6, "bound_damp": 12000.0}


class _Shock(C.Structure):
    _fields_ = [("beam", C.c_uint32), ("type", C.c_uint8), ("soft_bump", C.c_uint8), ("pad", C.c_uint16)] + \
               [(k, C.c_float) for k in SHOCK_KEYS]


class _Wheel(C.Structure):
    _fields_ = [("axle0", C.c_uint32), ("axle1", C.c_uint32), ("n_nodes", C.c_int32), ("nodes", C.c_void_p),
                ("radius", C.c_float), ("width", C.c_float), ("mass", C.c_float), ("propulsed", C.c_int32),
                ("arm", C.c_int32), ("near_attach", C.c_int32)]


class _BodyState(C.Structure):
    _fields_ = [("aabb_min", C.c_float * 3), ("aabb_max", C.c_float * 3), ("max_speed", C.c_float),
                ("sleeping", C.c_int32), ("static_contacts", C.c_int32), ("broken_beams", C.c_int32),
                ("sleep_timer", C.c_float), ("repaired_nodes", C.c_int32), ("fem_failures", C.c_int32),
                ("fem_clamps", C.c_int32), ("body_contacts", C.c_int32), ("wake_request", C.c_int32)]


class _WorldStats(C.Structure):
    _fields_ = [("substeps", C.c_int32), ("active_bodies", C.c_int32), ("sleeping_bodies", C.c_int32),
                ("active_nodes", C.c_int32), ("active_beams", C.c_int32), ("total_substeps", C.c_int64),
                ("kernel_launches", C.c_int64), ("device_errors", C.c_uint32), ("contacts", C.c_int64),
                ("pair_searches", C.c_int64), ("pairs", C.c_int32), ("islands", C.c_int32)]


class _FrameProfile(C.Structure):
    _fields_ = [("substeps", C.c_int32), ("frame_ms", C.c_float), ("begin_ms", C.c_float), ("beams_ms", C.c_float),
                ("nodes_ms", C.c_float), ("finish_ms", C.c_float), ("force_ms", C.c_float), ("contacts_ms", C.c_float),
                ("integrate_ms", C.c_float), ("fem_ms", C.c_float), ("search_ms", C.c_float)]


class _Config(C.Structure):
    _fields_ = [("gravity", C.c_float * 3), ("dt", C.c_float), ("sleeping", C.c_int32), ("sleep_speed", C.c_float),
                ("sleep_time", C.c_float), ("device", C.c_int32), ("deterministic", C.c_int32),
                ("collision_hz", C.c_float), ("inter_body_collisions", C.c_int32), ("max_pairs", C.c_int32),
                ("fem_solver", C.c_int32), ("pcg_max_iters", C.c_int32), ("pcg_tol", C.c_float),
                ("fem_check_residual", C.c_int32), ("pcg_learned_scale", C.c_int32), ("graphs", C.c_int32),
                ("beam_kernel", C.c_int32), ("fem_dense_front", C.c_int32), ("force_block", C.c_int32),
                ("integrate_block", C.c_int32), ("beams_per_sm", C.c_int32), ("tyre_grip", C.c_float),
                ("bulk_wait_s", C.c_float), ("contact_whole_max", C.c_int32)]


class _FemStats(C.Structure):
    _fields_ = [("pcg_solves", C.c_int64), ("pcg_fallbacks", C.c_int64), ("pcg_iterations", C.c_int64),
                ("last_iterations", C.c_int32), ("pad", C.c_int32), ("last_pcg_residual", C.c_double),
                ("max_residual", C.c_double), ("last_residual", C.c_double), ("columns", C.c_int64),
                ("blocks", C.c_int64), ("updates", C.c_int64), ("levels", C.c_int64), ("repasses", C.c_int64),
                ("fronts", C.c_int64), ("factor_flops", C.c_double)]


FEM_SOLVERS = {"cholesky": 0, "pcg": 1, "pcg_learned": 2, "pcg_previous": 3}


def _tuned_shapes() -> dict:
    """The launch shapes beamlab_b200/autotune.py chose (beamlab_b200/tuned.json), if any."""
    import json
    import os
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuned.json")
    try:
        with open(path) as f:
            return {k: int(v) for k, v in json.load(f).get("shapes", {}).items()}
    except (OSError, ValueError):
        return {}


class BodyHandle:
    """A body held by a World (the reference's SoftBody* from World::add_body)."""

    def __init__(self, world: "World", index: int, n_nodes: int, n_beams: int, name: str):
        self.world, self.index, self.name = world, index, name
        self.n_nodes, self.n_beams = n_nodes, n_beams

    def nodes(self) -> np.ndarray:
        out = np.zeros(self.n_nodes, NODE_DTYPE)
        _check(self.world._L.bl_gpu_download_nodes(self.world._ctx, self.index, out.ctypes.data), "download_nodes",
               self.world._ctx)
        return out

    def set_nodes(self, nodes: np.ndarray):
        nodes = np.ascontiguousarray(nodes, NODE_DTYPE)
        _check(self.world._L.bl_gpu_upload_nodes(self.world._ctx, self.index, nodes.ctypes.data), "upload_nodes",
               self.world._ctx)

    def beams(self) -> np.ndarray:
        out = np.zeros(self.n_beams, BEAM_DTYPE)
        _check(self.world._L.bl_gpu_download_beams(self.world._ctx, self.index, out.ctypes.data), "download_beams",
               self.world._ctx)
        return out

    def state(self) -> dict:
        s = _BodyState()
        _check(self.world._L.bl_gpu_body_state(self.world._ctx, self.index, C.byref(s)), "body_state",
               self.world._ctx)
        return {"aabb_min": np.array(s.aabb_min, np.float32), "aabb_max": np.array(s.aabb_max, np.float32),
                "max_speed": float(s.max_speed), "sleeping": bool(s.sleeping), "static_contacts": s.static_contacts,
                "broken_beams": s.broken_beams, "sleep_timer": float(s.sleep_timer),
                "repaired_nodes": s.repaired_nodes, "fem_failures": s.fem_failures, "fem_clamps": s.fem_clamps,
                "body_contacts": s.body_contacts, "wake_request": bool(s.wake_request)}

    def fem(self) -> dict | None:
        """The FEM frame's nodes: body node, double positions, orientations (x y z w), angular velocities."""
        L, ctx = self.world._L, self.world._ctx
        n = C.c_int32()
        _check(L.bl_gpu_download_fem(ctx, self.index, C.byref(n), None, None, None, None), "download_fem", ctx)
        if n.value == 0:
            return None
        node = np.zeros(n.value, np.int32)
        xd = np.zeros((n.value, 3), np.float64)
        q = np.zeros((n.value, 4), np.float32)
        w = np.zeros((n.value, 3), np.float32)
        _check(L.bl_gpu_download_fem(ctx, self.index, C.byref(n), node.ctypes.data, xd.ctypes.data, q.ctypes.data,
                                     w.ctypes.data), "download_fem", ctx)
        return {"node": node, "xd": xd, "q": q, "w": w}

    def fem_tris(self) -> dict | None:
        """The FEM triangles' plastic state: rest shapes (6 each), rest frames (x y z w per corner), plastic stretch."""
        L, ctx = self.world._L, self.world._ctx
        n = C.c_int32()
        _check(L.bl_gpu_download_fem_tris(ctx, self.index, C.byref(n), None, None, None), "download_fem_tris", ctx)
        if n.value == 0:
            return None
        X = np.zeros((n.value, 6), np.float32)
        r0 = np.zeros((n.value, 12), np.float32)
        dmg = np.zeros(n.value, np.float32)
        _check(L.bl_gpu_download_fem_tris(ctx, self.index, C.byref(n), X.ctypes.data, r0.ctypes.data, dmg.ctypes.data),
               "download_fem_tris", ctx)
        return {"X": X, "r0": r0, "dmg": dmg}

    def set_wheel_drive(self, wheel: int, torque: float, brake: float = 0.0):
        """A wheel's drive and brake torque (N m), every substep from the next on."""
        _check(self.world._L.bl_gpu_set_wheel_drive(self.world._ctx, self.index, int(wheel), float(torque), float(brake)),
               "set_wheel_drive", self.world._ctx)

    def wheels(self) -> dict:
        """Its wheels' tread speed (Wheel::speed, m/s) and average speed."""
        L, ctx = self.world._L, self.world._ctx
        n = C.c_int32()
        _check(L.bl_gpu_download_wheels(ctx, self.index, C.byref(n), None, None), "download_wheels", ctx)
        sp, av = np.zeros(n.value, np.float32), np.zeros(n.value, np.float32)
        _check(L.bl_gpu_download_wheels(ctx, self.index, C.byref(n), sp.ctypes.data, av.ctypes.data), "download_wheels", ctx)
        return {"speed": sp, "avg_speed": av}

    def wheel_speed(self) -> tuple[float, float]:
        """SoftBody::wheel_speed and wheel_spin: the forward-propelled wheels' mean tread speed and spin."""
        sp, spin = C.c_float(), C.c_float()
        _check(self.world._L.bl_gpu_wheel_speed(self.world._ctx, self.index, C.byref(sp), C.byref(spin)), "wheel_speed",
               self.world._ctx)
        return sp.value, spin.value

    def set_node_force(self, node: int, force):
        """A constant force on one node, every substep after gravity (a SoftBody::pre_substep push)."""
        f = (C.c_float * 3)(*[float(x) for x in force])
        _check(self.world._L.bl_gpu_set_node_force(self.world._ctx, self.index, int(node), f), "set_node_force",
               self.world._ctx)


class World:
    """World (world.h:150-171) on one B200: the statics, the bodies, frames of 2 kHz substeps."""

    def __init__(self, settings: WorldSettings | None = None, device: int = 0):
        self.settings = settings or WorldSettings()
        self.statics = StaticWorld()
        self._L = _lib.lib()
        cfg = _Config()
        self._L.bl_gpu_default_config(C.byref(cfg))
        cfg.gravity[:] = [float(x) for x in self.settings.gravity]
        cfg.dt = self.settings.dt
        cfg.sleeping = int(self.settings.sleeping)
        cfg.sleep_speed = self.settings.sleep_speed
        cfg.sleep_time = self.settings.sleep_time
        cfg.device = device
        cfg.collision_hz = self.settings.collision_hz
        cfg.inter_body_collisions = int(self.settings.inter_body_collisions)
        if self.settings.max_pairs > 0:
            cfg.max_pairs = int(self.settings.max_pairs)
        cfg.fem_solver = FEM_SOLVERS[self.settings.fem_solver]
        cfg.pcg_max_iters = int(self.settings.pcg_max_iters)
        cfg.pcg_tol = float(self.settings.pcg_tol)
        cfg.fem_check_residual = int(self.settings.fem_check_residual)
        cfg.pcg_learned_scale = int(self.settings.pcg_learned_scale)
        cfg.graphs = int(self.settings.graphs)
        cfg.beam_kernel = int(self.settings.beam_kernel)
        cfg.fem_dense_front = int(self.settings.fem_dense_front)
        cfg.tyre_grip = float(self.settings.tyre_grip)
        cfg.bulk_wait_s = float(self.settings.bulk_wait_s)
        cfg.contact_whole_max = int(self.settings.contact_whole_max)
        tuned = _tuned_shapes()
        for k in ("force_block", "integrate_block", "beams_per_sm"):
            v = getattr(self.settings, k)
            setattr(cfg, k, int(v if v is not None else tuned.get(k, 0)))
        self._ctx = C.c_void_p()
        _check(self._L.bl_gpu_create(C.byref(cfg), C.byref(self._ctx)), "create")
        self._bodies: list[BodyHandle] = []
        self._statics_sent = False
        self._keep = []
        self._accum = 0.0

    def close(self):
        if getattr(self, "_ctx", None):
            self._L.bl_gpu_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- statics
    def _send_statics(self):
        if self._statics_sent:
            return
        st, L, ctx = self.statics, self._L, self._ctx
        if st.terrain is not None:
            t = st.terrain
            h = np.ascontiguousarray(t["heights"], np.float32)
            s = np.ascontiguousarray(t["surfaces"], np.uint8) if t.get("surfaces") is not None else None
            _check(L.bl_gpu_set_terrain(ctx, int(t["nx"]), int(t["nz"]), float(t["cell"]), float(t["origin"][0]),
                                        float(t["origin"][1]), h.ctypes.data, s.ctypes.data if s is not None else None),
                   "set_terrain", ctx)
        for b in st.boxes:
            arr = (C.c_float * 3)(*b["center"]), (C.c_float * 3)(*b["half"]), (C.c_float * 4)(*b.get("rot", (0, 0, 0, 1)))
            _check(L.bl_gpu_add_box(ctx, arr[0], arr[1], arr[2], int(b.get("surface", 3)), float(b.get("max_force", 0.0))),
                   "add_box", ctx)
        for c in st.cylinders:
            _check(L.bl_gpu_add_cylinder(ctx, (C.c_float * 3)(*c["base"]), float(c["radius"]), float(c["height"]),
                                         int(c.get("surface", 3))), "add_cylinder", ctx)
        if st.grid_built:
            _check(L.bl_gpu_build_grid(ctx), "build_grid", ctx)
        _check(L.bl_gpu_set_kill_y(ctx, float(st.kill_y)), "set_kill_y", ctx)
        self._statics_sent = True

    # ---- bodies
    def add_body(self, body: SoftBody) -> BodyHandle:
        """World::add_body (world.cpp:283-289): the body is copied to the device."""
        if body.node_count() == 0 and len(body._nodes):
            body.finalize()
        nodes = np.ascontiguousarray(body.nodes, NODE_DTYPE)
        info = np.ascontiguousarray(body.info, NODE_INFO_DTYPE)
        beams = np.ascontiguousarray(body.beams, BEAM_DTYPE)
        fem_ptr = None
        if len(body.fem_tris) or len(body.fem_members):
            secs = (_ShellSection * max(len(body.fem_sections), 1))(*[
                _ShellSection(float(x["E"]), float(x["nu"]), float(x["rho"]), float(x["t"]), float(x.get("yield", 0.0)),
                              float(x.get("damping", 3e-4)), float(x.get("drill", 0.05))) for x in body.fem_sections])
            tris = np.ascontiguousarray(body.fem_tris, FEM_TRI_DTYPE)
            fsecs = (_FrameSection * max(len(body.frame_sections), 1))(*[
                _FrameSection(*(float(x.get(k, d)) for k, d in (("E", 2.1e11), ("G", 8.1e10), ("rho", 7850.0), ("A", 0.0),
                                                                 ("Iy", 0.0), ("Iz", 0.0), ("J", 0.0), ("As_y", 0.0),
                                                                 ("As_z", 0.0), ("damping", 2e-5), ("axial", 1.0),
                                                                 ("joint_k", 2.0e4), ("Np", 0.0), ("Mp", 0.0),
                                                                 ("Tp", 0.0), ("hardening", 0.25)))) for x in body.frame_sections])
            mems = np.ascontiguousarray(body.fem_members, FEM_MEMBER_DTYPE)
            fd = _FemDesc(len(body.fem_sections), C.cast(secs, C.c_void_p), len(tris), tris.ctypes.data if len(tris) else None,
                          float(body.fem_theta), float(body.fem_dissipation), len(body.frame_sections),
                          C.cast(fsecs, C.c_void_p), len(mems), mems.ctypes.data if len(mems) else None,
                          int(body.fem_tris_first))
            self._keep += [secs, tris, fsecs, mems, fd]
            fem_ptr = C.pointer(fd)
        d = _BodyDesc(len(nodes), nodes.ctypes.data, info.ctypes.data, len(beams), beams.ctypes.data,
                      body.ground_friction, body.bounce, body.contact_push_max, body.contact_slop,
                      int(body.allow_deform), int(body.allow_break), int(body.ductile), int(body.can_sleep),
                      body.sleep_speed, 0.0, 0, fem_ptr)
        tris = np.ascontiguousarray(body.tris, TRI_DTYPE)
        self._keep.append(tris)
        d.n_tris, d.tris = len(tris), (tris.ctypes.data if len(tris) else None)
        d.collision_radius, d.contact_friction = float(body.collision_radius), float(body.contact_friction)
        d.hull_depth, d.face_skin, d.faces_only = float(body.hull_depth), float(body.face_skin), int(body.faces_only)
        d.collision_group, d.self_collision = int(body.collision_group), int(body.self_collision)
        d.air_drag, d.aero_cda = float(body.air_drag), float(body.aero_cda)
        if body.wheels:
            wl = []
            for wh in body.wheels:
                wn = np.ascontiguousarray(wh["nodes"], np.uint32)
                self._keep.append(wn)
                wl.append(_Wheel(int(wh["axle0"]), int(wh["axle1"]), len(wn), wn.ctypes.data, float(wh.get("radius", 0.4)),
                                 float(wh.get("width", 0.2)), float(wh.get("mass", 0.0)), int(wh.get("propulsed", 0)),
                                 int(wh.get("arm", -1)), int(wh.get("near_attach", -1))))
            wa = (_Wheel * len(wl))(*wl)
            self._keep.append(wa)
            d.n_wheels, d.wheels = len(wl), C.cast(wa, C.c_void_p)
        if body.shocks:
            sa = (_Shock * len(body.shocks))(*[
                _Shock(int(x["beam"]), int(x.get("type", 1)), int(bool(x.get("soft_bump", False))), 0,
                       *(float(x.get(k, SHOCK_DEFAULTS.get(k, 0.0))) for k in SHOCK_KEYS)) for x in body.shocks])
            self._keep.append(sa)
            d.n_shocks, d.shocks = len(body.shocks), C.cast(sa, C.c_void_p)
        idx = C.c_int32()
        _check(self._L.bl_gpu_add_body(self._ctx, C.byref(d), C.byref(idx)), "add_body", self._ctx)
        h = BodyHandle(self, idx.value, len(nodes), len(beams), body.name)
        self._bodies.append(h)
        return h

    def bodies(self) -> list[BodyHandle]:
        return list(self._bodies)

    # ---- stepping
    def step_substeps(self, n: int, stream=None):
        """World::step_substeps (world.cpp:368-585): one frame of n substeps, enqueued (asynchronous).
        stream: a torch.cuda.Stream, a raw cudaStream_t (int) or None (the world's own)."""
        self._send_statics()
        _check(self._L.bl_gpu_step_substeps(self._ctx, int(n), self._stream(stream)), "step_substeps", self._ctx)

    def step_frame(self, frame_dt: float):
        """World::step_frame (world.cpp:312-346) without the load-dependent substep limits: the substeps the
        accumulated time holds, at most 100."""
        self._accum += frame_dt
        n = int(self._accum / self.settings.dt)
        if n > 100:
            n, self._accum = 100, 0.0
        else:
            self._accum -= n * self.settings.dt
        if n > 0:
            self.step_substeps(n)

    def synchronize(self):
        _check(self._L.bl_gpu_synchronize(self._ctx), "synchronize", self._ctx)

    def stats(self) -> dict:
        s = _WorldStats()
        self._send_statics()
        _check(self._L.bl_gpu_stats(self._ctx, C.byref(s)), "stats", self._ctx)
        return {k: getattr(s, k) for k, _ in _WorldStats._fields_}

    def device_nodes(self):
        """(pointer, total): the device array of every body's nodes back to back, in NODE_DTYPE records."""
        self._send_statics()
        p, n = C.c_void_p(), C.c_int32()
        _check(self._L.bl_gpu_device_nodes(self._ctx, C.byref(p), C.byref(n)), "device_nodes", self._ctx)
        return p.value, n.value

    @staticmethod
    def _stream(stream):
        s = getattr(stream, "cuda_stream", stream) if stream is not None else None
        return C.c_void_p(s) if s else None

    def upload_all_nodes(self, nodes: np.ndarray, stream=None):
        """Every body's nodes (NODE_DTYPE, back to back) to the device, asynchronous on `stream`."""
        self._send_statics()
        _check(self._L.bl_gpu_upload_all_nodes(self._ctx, nodes.ctypes.data, len(nodes), self._stream(stream)),
               "upload_all_nodes", self._ctx)

    def download_all_nodes(self, out: np.ndarray, stream=None):
        """Every body's nodes from the device into `out` (NODE_DTYPE), asynchronous on `stream`."""
        self._send_statics()
        _check(self._L.bl_gpu_download_all_nodes(self._ctx, out.ctypes.data, len(out), self._stream(stream)),
               "download_all_nodes", self._ctx)

    def profile_frame(self, n: int, stream=None) -> dict:
        """One frame of n substeps (it advances the world) with the GPU time of each kind of kernel; synchronous."""
        self._send_statics()
        p = _FrameProfile()
        _check(self._L.bl_gpu_profile_frame(self._ctx, int(n), self._stream(stream), C.byref(p)), "profile_frame",
               self._ctx)
        return {k: getattr(p, k) for k, _ in _FrameProfile._fields_}

    def fem_stats(self) -> dict:
        """The implicit FEM step's solver counters: PCG solves, fallbacks, iterations, residuals."""
        self._send_statics()
        s = _FemStats()
        _check(self._L.bl_gpu_fem_stats(self._ctx, C.byref(s)), "fem_stats", self._ctx)
        return {k: getattr(s, k) for k, _ in _FemStats._fields_ if k != "pad"}

    # ---- the learned warm start's network (include/beamlab_gpu.h: bl_gpu_mlp_*)
    MLP_PARAMS, MLP_INPUTS, MLP_OUTPUTS = 11468, 36, 12

    def mlp_init(self, seed: int = 1):
        _check(self._L.bl_gpu_mlp_init(self._ctx, int(seed)), "mlp_init", self._ctx)

    def mlp_weights(self) -> np.ndarray:
        w = np.zeros(self.MLP_PARAMS, np.float32)
        _check(self._L.bl_gpu_mlp_get_weights(self._ctx, w.ctypes.data, len(w)), "mlp_get_weights", self._ctx)
        return w

    def set_mlp_weights(self, w: np.ndarray):
        w = np.ascontiguousarray(w, np.float32)
        _check(self._L.bl_gpu_mlp_set_weights(self._ctx, w.ctypes.data, len(w)), "mlp_set_weights", self._ctx)

    def mlp_record(self, capacity: int):
        """Record one training sample per frame node and substep into a ring of `capacity` (0: stop recording)."""
        self._send_statics()
        _check(self._L.bl_gpu_mlp_record(self._ctx, int(capacity)), "mlp_record", self._ctx)

    def mlp_samples(self) -> int:
        n = C.c_int32()
        _check(self._L.bl_gpu_mlp_samples(self._ctx, C.byref(n)), "mlp_samples", self._ctx)
        return n.value

    def mlp_train(self, epochs: int, batch: int = 4096, lr: float = 1e-3, seed: int = 1) -> float:
        loss = C.c_float()
        _check(self._L.bl_gpu_mlp_train(self._ctx, int(epochs), int(batch), float(lr), int(seed), C.byref(loss)),
               "mlp_train", self._ctx)
        return loss.value

    def mlp_forward(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float32).reshape(-1, self.MLP_INPUTS)
        y = np.zeros((len(x), self.MLP_OUTPUTS), np.float32)
        _check(self._L.bl_gpu_mlp_forward(self._ctx, x.ctypes.data, len(x), y.ctypes.data), "mlp_forward", self._ctx)
        return y

    def mlp_gradient(self, x: np.ndarray, t: np.ndarray, w: np.ndarray):
        """(gradient, loss) of sum_s sum_o w (y - t)^2 / (2 n) over the n samples."""
        x = np.ascontiguousarray(x, np.float32).reshape(-1, self.MLP_INPUTS)
        t = np.ascontiguousarray(t, np.float32).reshape(-1, self.MLP_OUTPUTS)
        w = np.ascontiguousarray(w, np.float32).reshape(-1, self.MLP_OUTPUTS)
        g = np.zeros(self.MLP_PARAMS, np.float32)
        loss = C.c_float()
        _check(self._L.bl_gpu_mlp_gradient(self._ctx, x.ctypes.data, t.ctypes.data, w.ctypes.data, len(x), g.ctypes.data,
                                           C.byref(loss)), "mlp_gradient", self._ctx)
        return g, loss.value

    def pairs(self) -> np.ndarray:
        """The contact pairs of the last pair search, island after island, each in the reference's order: rows of
        (node's body, node, triangle's body, triangle)."""
        self._send_statics()
        n = C.c_int32()
        _check(self._L.bl_gpu_download_pairs(self._ctx, None, 0, C.byref(n)), "download_pairs", self._ctx)
        out = np.zeros((n.value, 4), np.int32)
        if n.value:
            _check(self._L.bl_gpu_download_pairs(self._ctx, out.ctypes.data, n.value, C.byref(n)), "download_pairs",
                   self._ctx)
        return out

    def body_range(self, body: int):
        a, b, c, d = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32()
        _check(self._L.bl_gpu_body_range(self._ctx, body, C.byref(a), C.byref(b), C.byref(c), C.byref(d)),
               "body_range", self._ctx)
        return a.value, b.value, c.value, d.value


def world_from_rig(rig: dict, device: int = 0, **overrides) -> World:
    """A World holding a rig of beamlab_b200.rigs: its settings, statics and bodies."""
    s = dict(rig.get("settings", {}))
    s.update(overrides)
    w = World(WorldSettings(**{k: v for k, v in s.items() if k in WorldSettings.__dataclass_fields__}), device)
    st = rig.get("statics", {})
    t = st.get("terrain")
    if t is not None:
        w.statics.create_terrain(t["nx"], t["nz"], t["cell"], t["origin"], t["heights"], t.get("surfaces"))
    for b in st.get("boxes", []):
        w.statics.add_box(b["center"], b["half"], b.get("rot", (0, 0, 0, 1)), b.get("surface", 3),
                          b.get("max_force", 0.0))
    for c in st.get("cylinders", []):
        w.statics.add_cylinder(c["base"], c["radius"], c["height"], c.get("surface", 3))
    if st.get("build_grid", True):
        w.statics.build_grid()
    if "kill_y" in st:
        w.statics.kill_y = st["kill_y"]
    for i, b in enumerate(rig["bodies"]):
        h = w.add_body(SoftBody.from_arrays(b, name=f"body{i}"))
        for node, f in b.get("loads", []):
            h.set_node_force(node, f)
    return w


__all__ = ["World", "WorldSettings", "StaticWorld", "SoftBody", "BodyHandle", "BeamLabError", "world_from_rig",
           "NODE_DTYPE", "NODE_INFO_DTYPE", "BEAM_DTYPE"]
