"""beamlab_b200: BeamLab's 2 kHz soft-body substep on one B200 (sm_100a), behind the C ABI of include/beamlab_gpu.h.

``World`` / ``SoftBody`` / ``StaticWorld`` / ``WorldSettings`` mirror the reference's ``bl::phys`` step API;
``rigs`` builds the seeded synthetic rigs of the benchmarks.
"""
from .world import (BEAM_DTYPE, NODE_DTYPE, NODE_INFO_DTYPE, BeamLabError, BodyHandle, SoftBody, StaticWorld, World,
                    WorldSettings, world_from_rig)

__all__ = ["World", "WorldSettings", "StaticWorld", "SoftBody", "BodyHandle", "BeamLabError", "world_from_rig",
           "NODE_DTYPE", "NODE_INFO_DTYPE", "BEAM_DTYPE"]
