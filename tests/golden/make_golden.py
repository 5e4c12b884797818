"""Writes the golden fixtures of the explicit substep from the reference itself.

The reference's physics (BeamLab src/phys + src/core, compiled from its sources by oracle/Makefile, parity flavour:
no FMA contraction) steps the seeded rigs of beamlab_b200.rigs through World::step_substeps in frames of 20
substeps; the node states at a few frames and the beams' state at the end are saved as .npz. The reference has no
golden data files of its own (its tests are analytic or live), so these fixtures are its outputs on this path.

    python tests/golden/make_golden.py        (needs oracle/_ref/libbeamlab_ref_parity.so)
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", ".."))

from beamlab_b200 import rigs  # noqa: E402
from oracle.oracle import RefWorld, build_world  # noqa: E402

FRAME = 20
CASES = {
    "truss_car_s1": (lambda: rigs.truss_car(1), 100, (1, 10, 50, 100)),
    "stress_rig_s7": (lambda: rigs.stress_rig(7), 100, (1, 10, 50, 100)),
}


def generate(name: str) -> dict:
    make, frames, snaps = CASES[name]
    rig = make()
    w = build_world(RefWorld, rig, multithreaded=False)
    out = {"frame_substeps": np.int32(FRAME), "snap_frames": np.asarray(snaps, np.int32)}
    for f in range(1, frames + 1):
        w.step_substeps(FRAME)
        if f in snaps:
            for b in range(len(rig["bodies"])):
                nd = w.nodes(b)
                out[f"pos_f{f}_b{b}"] = nd["pos"]
                out[f"vel_f{f}_b{b}"] = nd["vel"]
    for b in range(len(rig["bodies"])):
        bm = w.beams(b)
        for k in ("L", "max_pos", "max_neg", "strength", "stress", "flags"):
            out[f"beam_{k}_b{b}"] = bm[k]
        st = w.body(b)
        out[f"body_b{b}"] = np.asarray([*st["aabb_min"], *st["aabb_max"], st["max_speed"], st["sleeping"],
                                        st["static_contacts"], st["broken_beams"]], np.float32)
    return out


if __name__ == "__main__":
    for name in CASES:
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **generate(name))
        print(path, os.path.getsize(path))
