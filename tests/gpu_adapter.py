"""The GPU World seen through the oracle's interface (nodes / beams / body as dicts), for side-by-side tests."""
import numpy as np

from beamlab_b200 import world_from_rig


class GpuWorld:
    def __init__(self, rig, **overrides):
        self.w = world_from_rig(rig, **overrides)
        self.h = self.w.bodies()

    def step_substeps(self, n, stream=None):
        self.w.step_substeps(n, stream)

    def nodes(self, b):
        nd = self.h[b].nodes()
        return {"pos": np.ascontiguousarray(nd["p"]), "vel": np.ascontiguousarray(nd["v"]),
                "inv_mass": nd["inv_mass"].copy(), "mass": nd["mass"].copy()}

    def set_nodes(self, b, pos, vel):
        nd = self.h[b].nodes()
        nd["p"], nd["v"] = pos, vel
        self.h[b].set_nodes(nd)

    def beams(self, b):
        bm = self.h[b].beams()
        return {k: bm[k].copy() for k in ("L", "max_pos", "max_neg", "strength", "stress", "flags")}

    def body(self, b):
        s = self.h[b].state()
        return {k: s[k] for k in ("aabb_min", "aabb_max", "max_speed", "sleeping", "static_contacts", "broken_beams",
                                  "sleep_timer")}
