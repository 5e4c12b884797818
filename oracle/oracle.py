"""Test infrastructure only: ctypes front ends for the two CPU oracles of the explicit soft-body substep.

* ``PortWorld``  - the plain-C restatement (oracle/softbody_oracle.c, built into oracle/_build/liboracle.so);
* ``RefWorld``   - the reference itself (BeamLab src/phys + src/core, compiled by oracle/Makefile into
  oracle/_ref/libbeamlab_ref_{parity,timing}.so, driven through oracle/ref_driver.cpp).

Both take the same rig description (a dict of numpy arrays, see beamlab_b200.rigs) and expose the same calls, so a
test can step one rig through either and compare. Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
leg import this module; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_LIB = os.path.join(HERE, "_build", "liboracle.so")
REF_LIBS = {
    "parity": os.path.join(HERE, "_ref", "libbeamlab_ref_parity.so"),
    "libm": os.path.join(HERE, "_ref", "libbeamlab_ref_libm.so"),
    "timing": os.path.join(HERE, "_ref", "libbeamlab_ref_timing.so"),
}


class BodyParams(C.Structure):
    """SoftBody knobs of the explicit path (softbody.h:650-700); the layout of RefBodyParams / OrcBodyParams."""
    _fields_ = [
        ("ground_friction", C.c_float), ("bounce", C.c_float), ("contact_push_max", C.c_float),
        ("contact_slop", C.c_float), ("collision_radius", C.c_float), ("allow_deform", C.c_int32),
        ("allow_break", C.c_int32), ("ductile", C.c_int32), ("can_sleep", C.c_int32), ("sleep_speed", C.c_float),
        # contacts with other bodies (RefBodyParams only; the restatement reads the fields above)
        ("contact_friction", C.c_float), ("hull_depth", C.c_float), ("face_skin", C.c_float), ("faces_only", C.c_int32),
        ("collision_group", C.c_int32),
    ]


def body_params(body: dict) -> BodyParams:
    p = body.get("params", {})
    return BodyParams(
        float(p.get("ground_friction", 1.0)), float(p.get("bounce", -1.0)), float(p.get("contact_push_max", 2.0)),
        float(p.get("contact_slop", 0.0)), float(p.get("collision_radius", 0.05)), int(p.get("allow_deform", 1)),
        int(p.get("allow_break", 1)), int(p.get("ductile", 0)), int(p.get("can_sleep", 1)),
        float(p.get("sleep_speed", 0.0)), float(p.get("contact_friction", 1.0)), float(p.get("hull_depth", 0.3)),
        float(p.get("face_skin", 0.002)), int(p.get("faces_only", 0)), int(p.get("collision_group", 0)),
    )


def _ptr(a, ctype):
    return a.ctypes.data_as(C.POINTER(ctype)) if a is not None else None


_loaded: dict[str, C.CDLL] = {}


def _load(path: str, prefix: str) -> C.CDLL:
    if path in _loaded:
        return _loaded[path]
    if not os.path.exists(path):
        raise FileNotFoundError(f"oracle library missing: {path} (run `make -C oracle`)")
    lib = C.CDLL(path)
    vp, f, i = C.c_void_p, C.c_float, C.c_int
    fp, u8p, u16p, u32p = C.POINTER(C.c_float), C.POINTER(C.c_uint8), C.POINTER(C.c_uint16), C.POINTER(C.c_uint32)
    sig = {
        "world_new": ([], vp),
        "world_free": ([vp], None),
        "world_settings": ([vp, f, f, f, f, i, i, i, f, f], None),
        "set_terrain": ([vp, i, i, f, f, f, fp, u8p], None),
        "add_box": ([vp, f, f, f, f, f, f, f, f, f, f, i, f], None),
        "add_cylinder": ([vp, f, f, f, f, f, i], None),
        "build_grid": ([vp], None),
        "set_kill_y": ([vp, f], None),
        "add_body": ([vp, i, fp, fp, fp, u16p, fp, fp, i, u32p, fp, fp, fp, fp, u8p, u8p, i, u32p, C.POINTER(BodyParams)], i),
        "step_substeps": ([vp, i], None),
        "body_nodes": ([vp, i], i),
        "body_beams": ([vp, i], i),
        "get_nodes": ([vp, i, fp, fp, fp, fp], None),
        "set_nodes": ([vp, i, fp, fp], None),
        "get_beams": ([vp, i, fp, fp, fp, fp, fp, u8p], None),
        "get_body": ([vp, i, fp], None),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, f"{prefix}_{name}")
        fn.argtypes = args
        fn.restype = res
    if prefix == "ref":
        lib.ref_jobs_init.argtypes = [i]
        lib.ref_jobs_threads.restype = i
        lib.ref_add_plate.argtypes = [vp, i] + [f] * 9 + [f] * 7 + [i, i]
        lib.ref_add_plate.restype = i
        lib.ref_set_point_load.argtypes = [vp, i, i, f, f, f]
        lib.ref_set_drag.argtypes = [vp, i, f, f]
        lib.ref_add_wheel.argtypes = [vp, i, C.c_uint32, C.c_uint32, u32p, i, f, f, f, i, i, i]
        lib.ref_set_wheel_drive.argtypes = [vp, i, i, f, f]
        lib.ref_wheel_state.argtypes = [vp, i, vp, vp]
        lib.ref_body_wheel_speed.argtypes = [vp, i, vp]
        lib.ref_set_tyre_grip.argtypes = [vp, f]
        lib.ref_set_body_flags.argtypes = [vp, i, i, i]
        lib.ref_fem_tri_dmg.argtypes = [vp, i, vp]
        lib.ref_add_shock.argtypes = [vp, i, C.c_uint32, i, i, fp]
        lib.ref_add_fem_body.argtypes = [vp, i, fp, fp, fp, u16p, i, fp, i, u32p, u16p, fp, i, fp, i, u32p, u16p, u8p, fp, i]
        lib.ref_add_fem_body.restype = i
        lib.ref_fem_info.argtypes = [vp, i, C.POINTER(C.c_longlong)]
        lib.ref_fem_pattern.argtypes = [vp, i, vp, vp, vp, vp]
        lib.ref_fem_nodes.argtypes = [vp, i, vp, vp, vp, vp]
        lib.ref_fem_tris.argtypes = [vp, i, vp, vp, vp, vp, vp]
        lib.ref_set_tri_sides.argtypes = [vp, i, vp]
        lib.ref_get_pairs.argtypes = [vp, vp, i]
        lib.ref_get_pairs.restype = i
    _loaded[path] = lib
    return lib


# Shock's rates in ref_add_shock's order, and Shock's defaults where they are not 0 (softbody.h:88-101)
_SHOCK_KEYS = ("spring", "damp", "spring_in", "damp_in", "prog_spring_in", "prog_damp_in", "spring_out", "damp_out",
               "prog_spring_out", "prog_damp_out", "damp_in_slow", "split_in", "damp_in_fast", "damp_out_slow", "split_out",
               "damp_out_fast", "short_bound", "long_bound", "bound_spring", "bound_damp")
_SHOCK_DEFAULTS = {"damp_in_slow": 1.0, "split_in": 1.0, "damp_in_fast": 1.0, "damp_out_slow": 1.0, "split_out": 1.0,
                   "damp_out_fast": 1.0, "bound_spring": 9e6, "bound_damp": 12000.0}


class _OracleWorld:
    """One world of the oracle: statics, bodies, frames of substeps (World::step_substeps)."""

    prefix = ""

    def __init__(self, lib: C.CDLL):
        self._lib = lib
        self._fn = lambda name: getattr(lib, f"{self.prefix}_{name}")
        self._w = self._fn("world_new")()
        self._keep = []

    def close(self):
        if self._w:
            self._fn("world_free")(self._w)
            self._w = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def settings(self, gravity=(0.0, -9.81, 0.0), dt=0.0005, sleeping=True, multithreaded=True, inter_body=True,
                 sleep_speed=0.06, sleep_time=1.0, tyre_grip=1.0):
        self._fn("world_settings")(self._w, *map(float, gravity), float(dt), int(sleeping), int(multithreaded),
                                   int(inter_body), float(sleep_speed), float(sleep_time))
        if self.prefix == "ref":
            self._lib.ref_set_tyre_grip(self._w, float(tyre_grip))
        elif float(tyre_grip) != 1.0:
            raise ValueError("tyre grip other than 1 steps in the reference only (RefWorld)")

    def load_statics(self, statics: dict):
        t = statics.get("terrain")
        if t is not None:
            h = np.ascontiguousarray(t["heights"], dtype=np.float32)
            s = t.get("surfaces")
            s = np.ascontiguousarray(s, dtype=np.uint8) if s is not None else None
            self._keep += [h, s]
            self._fn("set_terrain")(self._w, int(t["nx"]), int(t["nz"]), float(t["cell"]), float(t["origin"][0]),
                                    float(t["origin"][1]), _ptr(h, C.c_float), _ptr(s, C.c_uint8))
        for b in statics.get("boxes", []):
            q = b.get("rot", (0.0, 0.0, 0.0, 1.0))
            self._fn("add_box")(self._w, *map(float, b["center"]), *map(float, b["half"]), *map(float, q),
                                int(b.get("surface", 3)), float(b.get("max_force", 0.0)))
        for c in statics.get("cylinders", []):
            self._fn("add_cylinder")(self._w, *map(float, c["base"]), float(c["radius"]), float(c["height"]),
                                     int(c.get("surface", 3)))
        if statics.get("build_grid", True):
            self._fn("build_grid")(self._w)
        if "kill_y" in statics:
            self._fn("set_kill_y")(self._w, float(statics["kill_y"]))

    def add_body(self, body: dict) -> int:
        a = {k: np.ascontiguousarray(body[k], dtype=dt) for k, dt in (
            ("pos", np.float32), ("vel", np.float32), ("mass", np.float32), ("node_flags", np.uint16),
            ("friction", np.float32), ("radius", np.float32), ("ab", np.uint32), ("k", np.float32),
            ("d", np.float32), ("strength", np.float32), ("deform", np.float32), ("beam_type", np.uint8),
            ("beam_flags", np.uint8))}
        tris = np.ascontiguousarray(body.get("tris", np.zeros((0, 3), np.uint32)), dtype=np.uint32)
        prm = body_params(body)
        self._keep += list(a.values()) + [tris, prm]
        idx = self._fn("add_body")(
            self._w, len(a["mass"]), _ptr(a["pos"], C.c_float), _ptr(a["vel"], C.c_float), _ptr(a["mass"], C.c_float),
            _ptr(a["node_flags"], C.c_uint16), _ptr(a["friction"], C.c_float), _ptr(a["radius"], C.c_float),
            len(a["k"]), _ptr(a["ab"], C.c_uint32), _ptr(a["k"], C.c_float), _ptr(a["d"], C.c_float),
            _ptr(a["strength"], C.c_float), _ptr(a["deform"], C.c_float), _ptr(a["beam_type"], C.c_uint8),
            _ptr(a["beam_flags"], C.c_uint8), len(tris), _ptr(tris, C.c_uint32), C.byref(prm))
        p = body.get("params", {})
        if float(p.get("air_drag", 0.0)) > 0 or float(p.get("aero_cda", 0.0)) > 0:
            if self.prefix != "ref":
                raise ValueError("air drag steps in the reference only (RefWorld)")
            self._lib.ref_set_drag(self._w, idx, float(p.get("air_drag", 0.0)), float(p.get("aero_cda", 0.0)))
        for sh in body.get("shocks", ()):
            if self.prefix != "ref":
                raise ValueError("shocks step in the reference only (RefWorld)")
            prm = np.asarray([float(sh.get(k, _SHOCK_DEFAULTS.get(k, 0.0))) for k in _SHOCK_KEYS], np.float32)
            self._keep.append(prm)
            self._lib.ref_add_shock(self._w, idx, int(sh["beam"]), int(sh.get("type", 1)), int(bool(sh.get("soft_bump", False))),
                                    _ptr(prm, C.c_float))
        for wh in body.get("wheels", ()):
            if self.prefix != "ref":
                raise ValueError("wheels step in the reference only (RefWorld)")
            wn = np.ascontiguousarray(wh["nodes"], dtype=np.uint32)
            self._keep.append(wn)
            self._lib.ref_add_wheel(self._w, idx, int(wh["axle0"]), int(wh["axle1"]), _ptr(wn, C.c_uint32), len(wn),
                                    float(wh.get("radius", 0.4)), float(wh.get("width", 0.2)), float(wh.get("mass", 0.0)),
                                    int(wh.get("propulsed", 0)), int(wh.get("arm", -1)), int(wh.get("near_attach", -1)))
        if self.prefix == "ref" and len(tris) and "tri_two_sided" in body:
            sides = np.ascontiguousarray(body["tri_two_sided"], dtype=np.uint8)
            self._keep.append(sides)
            self._lib.ref_set_tri_sides(self._w, idx, sides.ctypes.data)
        return idx

    def step_substeps(self, n: int):
        self._fn("step_substeps")(self._w, int(n))

    def set_wheel_drive(self, body: int, wheel: int, torque: float, brake: float):
        """A wheel's drive and brake torque (N m), set every substep from now on (RefWorld only)."""
        self._lib.ref_set_wheel_drive(self._w, body, wheel, float(torque), float(brake))

    def wheels(self, body: int, n: int) -> dict:
        """The first n wheels' speed and average speed (RefWorld only)."""
        sp, av = np.zeros(n, np.float32), np.zeros(n, np.float32)
        self._lib.ref_wheel_state(self._w, body, sp.ctypes.data, av.ctypes.data)
        ws = np.zeros(2, np.float32)
        self._lib.ref_body_wheel_speed(self._w, body, ws.ctypes.data)
        return {"speed": sp, "avg_speed": av, "wheel_speed": ws[0], "wheel_spin": ws[1]}

    def nodes(self, body: int):
        n = self._fn("body_nodes")(self._w, body)
        pos = np.zeros((n, 3), np.float32)
        vel = np.zeros((n, 3), np.float32)
        im = np.zeros(n, np.float32)
        m = np.zeros(n, np.float32)
        self._fn("get_nodes")(self._w, body, _ptr(pos, C.c_float), _ptr(vel, C.c_float), _ptr(im, C.c_float),
                              _ptr(m, C.c_float))
        return {"pos": pos, "vel": vel, "inv_mass": im, "mass": m}

    def set_nodes(self, body: int, pos, vel):
        pos = np.ascontiguousarray(pos, np.float32)
        vel = np.ascontiguousarray(vel, np.float32)
        self._fn("set_nodes")(self._w, body, _ptr(pos, C.c_float), _ptr(vel, C.c_float))

    def beams(self, body: int):
        m = self._fn("body_beams")(self._w, body)
        out = {k: np.zeros(m, np.float32) for k in ("L", "max_pos", "max_neg", "strength", "stress")}
        fl = np.zeros(m, np.uint8)
        self._fn("get_beams")(self._w, body, *(_ptr(out[k], C.c_float) for k in ("L", "max_pos", "max_neg",
                                                                                "strength", "stress")),
                              _ptr(fl, C.c_uint8))
        out["flags"] = fl
        return out

    def body(self, body: int):
        o = np.zeros(11, np.float32)
        self._fn("get_body")(self._w, body, _ptr(o, C.c_float))
        return {"aabb_min": o[0:3].copy(), "aabb_max": o[3:6].copy(), "max_speed": float(o[6]),
                "sleeping": bool(o[7]), "static_contacts": int(o[8]), "broken_beams": int(o[9]),
                "sleep_timer": float(o[10])}


class _FemMixin:
    """The reference's FEM frames (RefWorld only): shell plates built by its own ShellMesher, their pattern and state."""

    def add_plate(self, body: dict) -> int:
        pl = body["plate"]
        sec = body["fem_sections"][0]
        n, size = int(pl["n"]), float(pl["size"])
        o = pl["origin"]
        du = float(np.float32(size / n))
        b = self._lib.ref_add_plate(self._w, n, *map(float, o), du, 0.0, 0.0, 0.0, 0.0, du, float(sec["E"]), float(sec["nu"]),
                                    float(sec["rho"]), float(sec["t"]), float(sec.get("yield", 0.0)), float(sec.get("damping", 3e-4)),
                                    float(sec.get("drill", 0.05)), 1 if (body["node_flags"][0] & 2) else 0, int(body["node_flags"][-1]))
        self._body_flags(b, body)
        for node, fv in body.get("loads", []):
            self._lib.ref_set_point_load(self._w, b, int(node), *map(float, fv))
        return b

    def _body_flags(self, b: int, body: dict):
        p = body.get("params", {})
        self._lib.ref_set_body_flags(self._w, b, int(p.get("allow_deform", 1)), int(p.get("allow_break", 1)))

    def add_fem_body(self, body: dict) -> int:
        """A body with a FEM frame of members and triangles from its arrays (FemFrame::add_section /
        add_shell_section / add_element / add_tri in the body's order), its point loads."""
        n = len(body["mass"])
        a = {k: np.ascontiguousarray(body[k], dtype=dt) for k, dt in (("pos", np.float32), ("vel", np.float32),
                                                                      ("mass", np.float32), ("node_flags", np.uint16))}
        ss = np.asarray([[float(x["E"]), float(x["nu"]), float(x["rho"]), float(x["t"]), float(x.get("yield", 0.0)),
                          float(x.get("damping", 3e-4)), float(x.get("drill", 0.05))] for x in body.get("fem_sections", [])],
                        np.float32).reshape(-1, 7)
        tri = np.ascontiguousarray(body.get("fem_tris", np.zeros((0, 3))), dtype=np.uint32).reshape(-1, 3)
        nt = len(tri)
        tsec = np.ascontiguousarray(body.get("fem_tri_section", np.zeros(nt)), dtype=np.uint16)
        tmass = np.ascontiguousarray(body.get("fem_tri_mass", np.zeros(nt)), dtype=np.float32)
        keys = ("E", "G", "rho", "A", "Iy", "Iz", "J", "As_y", "As_z", "damping", "axial", "joint_k", "Np", "Mp", "Tp",
                "hardening")
        dflt = {"E": 2.1e11, "G": 8.1e10, "rho": 7850.0, "damping": 2e-5, "axial": 1.0, "joint_k": 2.0e4, "hardening": 0.25}
        fs = np.asarray([[float(sd.get(k, dflt.get(k, 0.0))) for k in keys] for sd in body.get("frame_sections", [])],
                        np.float32).reshape(-1, 16)
        ab = np.ascontiguousarray(body.get("fem_members", np.zeros((0, 2))), dtype=np.uint32).reshape(-1, 2)
        m = len(ab)
        msec = np.ascontiguousarray(body.get("member_section", np.zeros(m)), dtype=np.uint16)
        ends = np.ascontiguousarray(body.get("member_ends", np.zeros((m, 2))), dtype=np.uint8)
        mm = np.ascontiguousarray(body.get("member_mass", np.zeros(m)), dtype=np.float32)
        self._keep += list(a.values()) + [ss, tri, tsec, tmass, fs, ab, msec, ends, mm]
        b = self._lib.ref_add_fem_body(self._w, n, _ptr(a["pos"], C.c_float), _ptr(a["vel"], C.c_float),
                                       _ptr(a["mass"], C.c_float), _ptr(a["node_flags"], C.c_uint16), len(ss),
                                       _ptr(ss, C.c_float), nt, _ptr(tri, C.c_uint32), _ptr(tsec, C.c_uint16),
                                       _ptr(tmass, C.c_float), len(fs), _ptr(fs, C.c_float), m, _ptr(ab, C.c_uint32),
                                       _ptr(msec, C.c_uint16), _ptr(ends, C.c_uint8), _ptr(mm, C.c_float),
                                       int(body.get("fem_tris_first", False)))
        self._body_flags(b, body)
        for node, fv in body.get("loads", []):
            self._lib.ref_set_point_load(self._w, b, int(node), *map(float, fv))
        return b

    def fem_info(self, body: int) -> dict:
        o = (C.c_longlong * 8)()
        self._lib.ref_fem_info(self._w, body, o)
        return dict(zip(("frame_nodes", "tris", "components", "blocks", "updates", "solve_failures", "clamps", "passes"),
                        list(o)))

    def fem_pattern(self, body: int) -> dict:
        info = self.fem_info(body)
        n, nb, nu = info["frame_nodes"], info["blocks"], info["updates"]
        out = {"perm": np.zeros(n, np.int32), "col_ptr": np.zeros(n + 1, np.int32), "row": np.zeros(nb, np.int32),
               "upd": np.zeros(3 * nu, np.int32)}
        self._lib.ref_fem_pattern(self._w, body, *(out[k].ctypes.data for k in ("perm", "col_ptr", "row", "upd")))
        return out

    def fem_nodes(self, body: int) -> dict:
        n = self.fem_info(body)["frame_nodes"]
        out = {"node": np.zeros(n, np.int32), "xd": np.zeros((n, 3), np.float64), "q": np.zeros((n, 4), np.float32),
               "w": np.zeros((n, 3), np.float32)}
        self._lib.ref_fem_nodes(self._w, body, *(out[k].ctypes.data for k in ("node", "xd", "q", "w")))
        return out

    def fem_tris(self, body: int) -> dict:
        t = self.fem_info(body)["tris"]
        out = {"n": np.zeros((t, 3), np.int32), "X": np.zeros((t, 6), np.float32), "r0": np.zeros((t, 12), np.float32),
               "mass": np.zeros(t, np.float32), "area0": np.zeros(t, np.float32)}
        self._lib.ref_fem_tris(self._w, body, *(out[k].ctypes.data for k in ("n", "X", "r0", "mass", "area0")))
        out["dmg"] = np.zeros(t, np.float32)
        self._lib.ref_fem_tri_dmg(self._w, body, out["dmg"].ctypes.data)
        return out


class PortWorld(_OracleWorld):
    """The plain-C restatement (single-threaded)."""

    prefix = "orc"

    def __init__(self):
        super().__init__(_load(PORT_LIB, "orc"))


class RefWorld(_FemMixin, _OracleWorld):
    """The reference's own World, compiled from its sources (flavour "parity", "libm" or "timing")."""

    prefix = "ref"

    def __init__(self, flavour: str = "parity"):
        super().__init__(_load(REF_LIBS[flavour], "ref"))

    def pairs(self) -> np.ndarray:
        """Island::nt of the islands that searched for pairs in the last frame (world.cpp:3466-3475): rows of
        (node's body, node, triangle's body, triangle)."""
        n = self._lib.ref_get_pairs(self._w, None, 0)
        out = np.zeros((n, 4), np.int32)
        if n:
            self._lib.ref_get_pairs(self._w, out.ctypes.data, n)
        return out


def ref_available(flavour: str = "parity") -> bool:
    return os.path.exists(REF_LIBS[flavour])


def port_available() -> bool:
    return os.path.exists(PORT_LIB)


def ref_jobs_init(workers: int, flavour: str = "timing") -> int:
    """JobSystem::get().init(workers) of the reference library (src/core/jobs.h:22); returns its thread count. The
    workers are shut down at interpreter exit (a process with them running does not end)."""
    import atexit
    lib = _load(REF_LIBS[flavour], "ref")
    lib.ref_jobs_init(int(workers))
    atexit.register(lib.ref_jobs_shutdown)
    return lib.ref_jobs_threads()


def ref_jobs_shutdown(flavour: str = "timing"):
    """JobSystem::get().shutdown() (src/core/jobs.h:23)."""
    _load(REF_LIBS[flavour], "ref").ref_jobs_shutdown()


def build_world(cls, rig: dict, **settings):
    """A world of `cls` holding the rig's statics and bodies (in order)."""
    w = cls() if cls is PortWorld else cls(settings.pop("flavour", "parity"))
    s = dict(rig.get("settings", {}))
    s.update(settings)
    w.settings(**s)
    w.load_statics(rig.get("statics", {}))
    for b in rig["bodies"]:
        if "plate" in b and "fem_members" not in b:
            if not hasattr(w, "add_plate"):
                raise ValueError("FEM plates step in the reference only (RefWorld)")
            w.add_plate(b)
        elif "fem_members" in b:
            if not hasattr(w, "add_fem_body"):
                raise ValueError("FEM frames step in the reference only (RefWorld)")
            w.add_fem_body(b)
        else:
            w.add_body(b)
    return w
