"""bl_gpu_substep_noalloc, the entry point for callers that cannot let the library allocate GPU memory (their memory
belongs to another allocator, or they step where allocation is forbidden): it must give what the context API gives.

The test allocates the body's device buffers itself (as such a caller does, here through torch), calls the entry
point twice in a row through the C ABI, and after each call compares the nodes and beams with the context API's
(bl_gpu_step_substeps, one-substep frames) on the same rig - bitwise, the tolerance of every parity test here. The
file sorts last, so it runs after the other tests; test_noalloc_in_a_fresh_process runs the comparison again in a
python process of its own, where the entry point's first call is the process's first use of the GPU."""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest

from beamlab_b200 import BEAM_DTYPE, NODE_DTYPE, SoftBody, World, WorldSettings, _lib, rigs

pytestmark = pytest.mark.gpu


def incidence(beams, n_nodes):
    """Each node's beams in beam order; bit 31 marks the node as the beam's b end."""
    a, b = beams["a"].astype(np.int64), beams["b"].astype(np.int64)
    ptr = np.zeros(n_nodes + 1, np.int64)
    np.add.at(ptr, a + 1, 1)
    np.add.at(ptr, b + 1, 1)
    ptr = np.cumsum(ptr)
    fill = ptr[:-1].copy()
    inc = np.zeros(2 * len(beams), np.int64)
    for j in range(len(beams)):
        inc[fill[a[j]]] = j
        fill[a[j]] += 1
        inc[fill[b[j]]] = j | 0x80000000
        fill[b[j]] += 1
    return ptr.astype(np.int32), inc.astype(np.uint32).view(np.int32)


def bits(a):
    a = np.ascontiguousarray(a, np.float32).copy()
    a[np.isnan(a)] = np.float32("nan")
    return a.view(np.uint32)


def test_noalloc_substep_matches_the_context_api():
    import torch
    rig = rigs.truss_car(1, speed=30.0)
    body = SoftBody.from_arrays(rig["bodies"][0])
    # nodes shaken apart at a few m/s, some beams weak: beams yield and break within the two substeps
    body.nodes["v"] += np.random.default_rng(1).uniform(-3.0, 3.0, body.nodes["v"].shape).astype(np.float32)
    body.beams["strength"][::7] = 1e3
    body.beams["max_pos"][::5], body.beams["max_neg"][::5] = 1e2, -1e2
    g = (0.0, -9.81, 0.0)
    dt = 0.0005

    # the context API: no statics, frames of one substep
    w = World(WorldSettings(gravity=g, dt=dt))
    h = w.add_body(body)

    # the caller's own device buffers
    dev = torch.device("cuda", 0)
    nodes = torch.from_numpy(body.nodes.copy().view(np.uint8)).to(dev)
    beams = torch.from_numpy(body.beams.copy().view(np.uint8)).to(dev)
    ptr, inc = incidence(body.beams, len(body.nodes))
    ptr_d = torch.from_numpy(ptr).to(dev)
    inc_d = torch.from_numpy(inc).to(dev)
    grav = (C.c_float * 3)(*g)
    L = _lib.lib()
    for call in range(2):
        w.step_substeps(1)
        rc = L.bl_gpu_substep_noalloc(nodes.data_ptr(), len(body.nodes), beams.data_ptr(), len(body.beams), ptr_d.data_ptr(),
                                      inc_d.data_ptr(), grav, dt, 1, 1, 0, None)
        assert rc == 0, L.bl_gpu_error_string(rc)
        torch.cuda.synchronize()
        got_n = nodes.cpu().numpy().view(NODE_DTYPE)
        got_b = beams.cpu().numpy().view(BEAM_DTYPE)
        ref_n, ref_b = h.nodes(), h.beams()
        assert np.array_equal(bits(got_n["p"]), bits(ref_n["p"])), f"call {call}: positions differ"
        assert np.array_equal(bits(got_n["v"]), bits(ref_n["v"])), f"call {call}: velocities differ"
        for k in ("L", "max_pos", "max_neg", "strength", "stress"):
            assert np.array_equal(bits(got_b[k]), bits(ref_b[k])), f"call {call}: beam {k} differs"
        assert np.array_equal(got_b["flags"], ref_b["flags"])
    assert (ref_b["flags"] & 1).any() and (ref_b["L"] != body.beams["L"]).any()  # breaks and yields were exercised
    w.close()


def test_noalloc_rejects_too_many_beams():
    L = _lib.lib()
    n = L.bl_gpu_substep_noalloc(C.c_void_p(16), 1, C.c_void_p(16), (1 << 20) + 1, C.c_void_p(16), C.c_void_p(16),
                                 (C.c_float * 3)(0, -9.81, 0), 0.0005, 1, 1, 0, None)
    assert n == -5 and L.bl_gpu_error_string(n).decode() == "capacity exceeded"


def test_noalloc_in_a_fresh_process():
    here = os.path.dirname(os.path.abspath(__file__))
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-p", "no:cacheprovider", "-m", "gpu",
                        f"{os.path.join(here, 'test_zz_no_alloc.py')}::test_noalloc_substep_matches_the_context_api"],
                       cwd=os.path.dirname(here), capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    assert "1 passed" in r.stdout
