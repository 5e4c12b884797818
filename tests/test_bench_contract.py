"""bench.py's host-side arithmetic without a GPU: the pair search's algorithmic bytes (the broadphase formula: 120 B a
contacter node, 48 B a collision triangle, 12 B a pair written) and the searches a substep."""
import importlib.util
import os

import numpy as np

from beamlab_b200 import rigs
from conftest import ROOT


def _bench():
    spec = importlib.util.spec_from_file_location("bench_module", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_broadphase_bytes_of_a_crash_pair():
    bench = _bench()
    rig = rigs.crash_pair(1, speed_a=3.0, speed_b=0.0, gap=0.1)
    contacters = sum(int(np.count_nonzero(np.asarray(b["node_flags"]) & rigs.NF_CONTACTER)) for b in rig["bodies"])
    tris = sum(len(b["tris"]) for b in rig["bodies"])
    bp = bench.broadphase_bytes(rig, 1000)
    assert bp["contacter_nodes"] == contacters > 0 and bp["triangles"] == tris > 0
    assert bp["bytes_per_search"] == 120 * contacters + 48 * tris + 12 * 1000
    # 120 Hz at 0.5 ms: a search every 17 substeps, on substeps 0 and 17 of a 33-substep frame
    assert bp["searches_per_substep"] == 2 / 33


def test_broadphase_searches_follow_the_collision_rate():
    bench = _bench()
    rig = rigs.crash_pair(1)
    rig = {**rig, "settings": {**rig["settings"], "collision_hz": 2000.0}}
    assert bench.broadphase_bytes(rig, 0)["searches_per_substep"] == 1.0
