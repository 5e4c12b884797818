"""The drop-in shim a BeamLab maintainer would add (tests/shim/gpu_world.h), compiled against the reference's own
headers: the compiler checks that Node, NodeInfo, Beam and Triangle have every field at the same offset and size as
bl_node, bl_node_info, bl_beam and bl_tri, and that the flag values agree (static_asserts). On the GPU, one body built
by the reference's own builder API is stepped by World::step_substeps and, a copy of it, through GpuWorld: the node and
beam states must be bitwise equal."""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

from beamlab_b200 import BEAM_DTYPE, NODE_DTYPE, rigs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHIM = os.path.join(ROOT, "tests", "shim")
LIB = os.path.join(SHIM, "_build", "libshim.so")
REFERENCE = "/root/reference"


def have_reference():
    return os.path.isdir(os.path.join(REFERENCE, "src", "phys")) and shutil.which("g++") is not None


@pytest.mark.skipif(not have_reference(), reason="the reference's headers are not on this machine")
def test_shim_layout_compiles_against_reference_headers():
    r = subprocess.run(["make", "-s", "-C", SHIM, "layout", f"REF={REFERENCE}"], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr


def test_shim_layout_check_fails_on_a_wrong_offset(tmp_path):
    """The check itself bites: a record whose field moved fails to compile (a planted mistake, on the host)."""
    if not shutil.which("g++"):
        pytest.skip("no host compiler")
    src = tmp_path / "moved.cpp"
    src.write_text('#include <cstddef>\n#include "beamlab_gpu.h"\n'
                   "struct Node { float inv_mass; float p[3]; float v[3]; float mass; };\n"
                   "static_assert(offsetof(Node, p) == offsetof(bl_node, p), \"p\");\n")
    r = subprocess.run(["g++", "-std=c++20", "-fsyntax-only", f"-I{ROOT}/include", str(src)], capture_output=True, text=True)
    assert r.returncode != 0 and "static assertion failed" in r.stderr


@pytest.mark.gpu
def test_shim_steps_a_reference_body_bitwise():
    if not os.path.exists(LIB):
        pytest.skip("the shim is built where the reference's headers are (make -C tests/shim)")
    lib = C.CDLL(LIB)
    rig = rigs.truss_car(2, speed=30.0)
    b = rig["bodies"][0]
    n, m = len(b["mass"]), len(b["k"])
    pos = np.ascontiguousarray(b["pos"], np.float32)
    vel = np.ascontiguousarray(b["vel"], np.float32) + np.random.default_rng(4).uniform(-2, 2, (n, 3)).astype(np.float32)
    mass = np.ascontiguousarray(b["mass"], np.float32)
    ab = np.ascontiguousarray(b["ab"], np.uint32).reshape(m, 2)
    k = np.ascontiguousarray(b["k"], np.float32)
    d = np.ascontiguousarray(b["d"], np.float32)
    strength = np.ascontiguousarray(b["strength"], np.float32) * np.float32(0.01)  # (weakened: beams yield and break)
    deform = np.ascontiguousarray(b["deform"], np.float32) * np.float32(0.01)
    out = {key: np.zeros(cnt, dt) for key, cnt, dt in (("rn", n, NODE_DTYPE), ("gn", n, NODE_DTYPE), ("rb", m, BEAM_DTYPE), ("gb", m, BEAM_DTYPE))}
    f = lib.shim_step_compare
    f.restype = C.c_int
    f.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                  C.c_float, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    rc = f(n, pos.ctypes.data, vel.ctypes.data, mass.ctypes.data, m, ab.ctypes.data, k.ctypes.data, d.ctypes.data,
           strength.ctypes.data, deform.ctypes.data, float(pos[:, 1].min()) - 0.05, 20, 33, *(out[key].ctypes.data for key in ("rn", "gn", "rb", "gb")))
    assert rc == 0
    for field in ("p", "v"):
        a, g = out["rn"][field].copy(), out["gn"][field].copy()
        a[np.isnan(a)] = 0
        g[np.isnan(g)] = 0
        assert np.array_equal(a.view(np.uint32), g.view(np.uint32)), field
    for field in ("L", "stress", "strength", "flags"):
        assert np.array_equal(np.ascontiguousarray(out["rb"][field]).view(np.uint8), np.ascontiguousarray(out["gb"][field]).view(np.uint8)), field
    assert (out["rb"]["flags"] & 1).any() or (out["rb"]["L"] != out["rb"]["L0"]).any()  # beams yielded or broke
