"""Launch-shape autotuner for the explicit substep: times each candidate launch shape of the beams' persistent kernel
(blocks an SM) and of the two node kernels (block size) on a workload, with CUDA events around each kernel of
profiled frames (bl_gpu_profile_frame), and writes the fastest to beamlab_b200/tuned.json, which World() reads for
settings left unset. Results do not depend on the shapes (each beam and node is computed alone); only the time does.

    python -m beamlab_b200.autotune [--workload fleet256|truss_car] [--frames 3] [--out PATH]
"""
from __future__ import annotations

import argparse
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
FRAME = 33
CANDIDATES = {"beams_per_sm": (1, 2, 3, 4), "force_block": (64, 128, 256), "integrate_block": (64, 128, 256)}
KERNEL_MS = {"beams_per_sm": "beams_ms", "force_block": "force_ms", "integrate_block": "integrate_ms"}


def _rig(name: str):
    from . import rigs
    if name == "fleet256":
        return rigs.fleet(256, seed=3)
    if name == "truss_car":
        return rigs.truss_car(1)
    raise SystemExit(f"unknown workload {name}")


def tune(workload: str = "fleet256", frames: int = 3, device: int = 0) -> dict:
    """{setting: {candidate: ms a substep of its kernel}} and the chosen shapes (each setting tuned with the others at
    their defaults)."""
    from .world import world_from_rig
    rig = _rig(workload)
    times = {k: {} for k in CANDIDATES}
    for key, cands in CANDIDATES.items():
        for v in cands:
            w = world_from_rig(rig, device=device, **{key: v})
            w.step_substeps(FRAME)  # (warm-up: commits, captures the graphs)
            w.profile_frame(FRAME)
            times[key][v] = min(w.profile_frame(FRAME)[KERNEL_MS[key]] for _ in range(frames)) / FRAME
            w.close()
    shapes = {k: min(t, key=t.get) for k, t in times.items()}
    return {"workload": workload, "ms_per_substep": {k: {str(c): t for c, t in d.items()} for k, d in times.items()},
            "shapes": shapes}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="fleet256")
    ap.add_argument("--frames", type=int, default=3)
    ap.add_argument("--out", default=os.path.join(HERE, "tuned.json"))
    a = ap.parse_args()
    res = tune(a.workload, a.frames)
    try:
        import torch
        res["device"] = torch.cuda.get_device_name(0)
    except Exception:
        pass
    with open(a.out, "w") as f:
        json.dump(res, f, indent=1)
    json.dump(res, sys.stdout)
    print()


if __name__ == "__main__":
    main()
