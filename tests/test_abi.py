"""The C ABI without a GPU: the library loads, exports every function include/beamlab_gpu.h declares, its records
have the reference's layouts, and the host mirror builds bodies as the reference's builder does."""
import ctypes as C
import os
import subprocess
import tempfile

import numpy as np
import pytest

from beamlab_b200 import _lib, rigs
from beamlab_b200.world import BEAM_DTYPE, NODE_DTYPE, NODE_INFO_DTYPE, SoftBody, _BodyDesc, _BodyState, _Config, _Shock, _Wheel, _WorldStats
from conftest import ROOT


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    names = _lib.header_symbols()
    assert len(names) >= 20
    for n in names:
        assert hasattr(L, n), n
    assert L.bl_gpu_abi_version() == 7
    assert L.bl_gpu_error_string(-4).decode() == "unsupported feature"


def _c_layout():
    """sizeof / offsetof of the header's records, from a C compiler."""
    tmp = tempfile.mkdtemp(prefix="bl_abi_")
    src = os.path.join(tmp, "abi_layout.c")
    exe = src[:-2]
    with open(src, "w") as f:
        f.write('#include <stdio.h>\n#include <stddef.h>\n#include "beamlab_gpu.h"\n'
                'int main(){printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\\n", sizeof(bl_node), sizeof(bl_node_info),'
                ' sizeof(bl_beam), sizeof(bl_body_desc), sizeof(bl_body_state), sizeof(bl_world_stats),'
                ' sizeof(bl_gpu_config), offsetof(bl_beam, type), offsetof(bl_body_desc, ground_friction),'
                ' sizeof(bl_wheel), offsetof(bl_body_desc, wheels), sizeof(bl_shock));return 0;}\n')
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), src, "-o", exe], check=True)
    return [int(x) for x in subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()]


def test_record_layouts_match_the_header():
    node, info, beam, desc, state, stats, cfg, off_type, off_gf, wheel, off_wheels, shock = _c_layout()
    assert (node, info, beam) == (32, 20, 52)  # the reference's Node, NodeInfo, Beam
    assert NODE_DTYPE.itemsize == node and NODE_INFO_DTYPE.itemsize == info and BEAM_DTYPE.itemsize == beam
    assert C.sizeof(_BodyDesc) == desc and C.sizeof(_BodyState) == state and C.sizeof(_WorldStats) == stats
    assert C.sizeof(_Config) == cfg and BEAM_DTYPE.fields["type"][1] == off_type
    assert _BodyDesc.ground_friction.offset == off_gf
    assert C.sizeof(_Wheel) == wheel and _BodyDesc.wheels.offset == off_wheels and C.sizeof(_Shock) == shock


def test_world_needs_a_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from beamlab_b200 import BeamLabError, World
    with pytest.raises(BeamLabError, match="no sm_100"):
        World()


def test_softbody_finalize_matches_the_reference_builder(port_lib):
    """Rest lengths, inverse masses and yield limits as SoftBody::add_node/add_beam/finalize make them."""
    from oracle.oracle import PortWorld, build_world
    rig = rigs.stress_rig(7)
    w = build_world(PortWorld, rig)
    for b, body in enumerate(rig["bodies"]):
        sb = SoftBody.from_arrays(body)
        ref_b, ref_n = w.beams(b), w.nodes(b)
        assert np.array_equal(sb.beams["L"].view(np.uint32), ref_b["L"].view(np.uint32))
        assert np.array_equal(sb.nodes["inv_mass"].view(np.uint32), ref_n["inv_mass"].view(np.uint32))
        assert np.array_equal(sb.beams["max_neg"], ref_b["max_neg"])


def test_softbody_builder_calls():
    sb = SoftBody("t")
    a = sb.add_node((0, 0, 0), 2.0)
    b = sb.add_node((0.0003, 0, 0), 0.0)
    c = sb.add_node((1, 2, 2), 5.0, flags=2)
    sb.add_beam(a, b, 1e5, 10)
    sb.add_beam(a, c, 1e5, 10, strength=7.0, deform=3.0, type=1)
    sb.finalize()
    assert sb.nodes["inv_mass"].tolist() == [0.5, 0.0, 0.0]
    assert sb.beams["L"][0] == np.float32(1e-3) and sb.beams["L"][1] == np.float32(3.0)
    assert sb.beams["max_neg"][1] == -3.0 and sb.beams["type"][1] == 1 and sb.beams["strength"][1] == 7.0


def test_config_defaults_and_refusals_without_a_gpu():
    """bl_gpu_default_config's contact_whole_max is the most an island runs whole (6,144); bl_gpu_create refuses a
    value outside 0..6,144 (and other out-of-range settings) before it touches a device."""
    L = _lib.lib()
    cfg = _Config()
    L.bl_gpu_default_config(C.byref(cfg))
    assert cfg.contact_whole_max == 6144 and cfg.max_pairs == 1 << 21 and cfg.bulk_wait_s == 1.0
    ctx = C.c_void_p()
    for field, bad in (("contact_whole_max", 6145), ("contact_whole_max", -1), ("max_pairs", 0), ("bulk_wait_s", 11.0)):
        c = _Config()
        L.bl_gpu_default_config(C.byref(c))
        setattr(c, field, bad)
        assert L.bl_gpu_create(C.byref(c), C.byref(ctx)) == -1, field  # (BL_GPU_EINVAL)
        assert not ctx.value
