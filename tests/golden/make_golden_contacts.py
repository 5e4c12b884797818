"""Writes the golden fixtures of contacts between bodies from the reference itself.

The reference's physics (compiled from its sources by oracle/Makefile, parity flavour, one thread) steps two lattice
trusses with collision skins into each other (beamlab_b200.rigs.crash_pair) with World::step_substeps: a first frame
of one substep, then frames of 33. After each frame the islands' contact pairs of the last pair search
(World::Island::nt after rebuild_pairs + near_pairs) are saved, and the node states at a few frames.

    python tests/golden/make_golden_contacts.py [name ...]      (needs oracle/_ref/libbeamlab_ref_parity.so)
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", ".."))

from beamlab_b200 import rigs  # noqa: E402
from oracle.oracle import RefWorld, build_world  # noqa: E402

FRAMES = [1] + [33] * 12
SNAPS = (1, 4, 12)
CASES = {
    # both slow (the spatial hash of nodes), both fast (each one's dense grid), fast into slow, hull skins
    "crash_slow_s1": lambda: rigs.crash_pair(1, speed_a=3.0, speed_b=0.0, gap=0.1),
    "crash_fast_s2": lambda: rigs.crash_pair(2, speed_a=12.0, speed_b=12.0, gap=0.5),
    "crash_mixed_s3": lambda: rigs.crash_pair(3, speed_a=25.0, speed_b=3.0, gap=0.6),
    "crash_hull_s4": lambda: rigs.crash_pair(4, speed_a=10.0, speed_b=4.0, gap=0.2, hull=True),
}


def generate(name: str) -> dict:
    w = build_world(RefWorld, CASES[name](), multithreaded=False)
    out = {"frames": np.asarray(FRAMES, np.int32), "snap_frames": np.asarray(SNAPS, np.int32)}
    for f, n in enumerate(FRAMES):
        w.step_substeps(n)
        out[f"pairs_f{f}"] = w.pairs()
        if f in SNAPS:
            for b in range(2):
                nd = w.nodes(b)
                out[f"pos{b}_f{f}"] = nd["pos"]
                out[f"vel{b}_f{f}"] = nd["vel"]
    return out


if __name__ == "__main__":
    for name in sys.argv[1:] or list(CASES):
        d = generate(name)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **d)
        print(name, "pairs per frame", [len(d[f"pairs_f{f}"]) for f in range(len(FRAMES))])
