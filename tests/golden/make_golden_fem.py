"""Writes the golden fixtures of the FEM shell plate from the reference itself.

The reference's physics (compiled from its sources by oracle/Makefile, parity flavour, one thread) builds the plate
with its own ShellMesher (fem_shell.cpp) and steps it with World::step_substeps in frames of 20 substeps; the body's
node positions and its frame's double positions and orientations at a few frames are saved as .npz.

    python tests/golden/make_golden_fem.py [name ...]      (needs oracle/_ref/libbeamlab_ref_parity.so)
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", ".."))

from beamlab_b200 import rigs  # noqa: E402
from oracle.oracle import RefWorld, build_world  # noqa: E402

FRAME = 20
CASES = {
    "plate20_s1": (lambda: rigs.shell_plate(20, seed=1), 20, (1, 5, 20)),
    "plate63_s1": (lambda: rigs.shell_plate(63, seed=1), 50, (1, 10, 50)),
}


def generate(name: str) -> dict:
    make, frames, snaps = CASES[name]
    w = build_world(RefWorld, make(), multithreaded=False)
    out = {"frame_substeps": np.int32(FRAME), "snap_frames": np.asarray(snaps, np.int32)}
    for f in range(1, frames + 1):
        w.step_substeps(FRAME)
        if f in snaps:
            nd = w.nodes(0)
            fn = w.fem_nodes(0)
            out[f"pos_f{f}"] = nd["pos"]
            out[f"vel_f{f}"] = nd["vel"]
            out[f"xd_f{f}"] = fn["xd"]
            out[f"q_f{f}"] = fn["q"]
    info = w.fem_info(0)
    out["solve_failures"] = np.int32(info["solve_failures"])
    out["clamps"] = np.int32(info["clamps"])
    return out


if __name__ == "__main__":
    for name in sys.argv[1:] or list(CASES):
        t0 = time.time()
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **generate(name))
        print(path, os.path.getsize(path), f"{time.time() - t0:.1f} s")
