"""Free-rolling node wheels on the GPU against the reference compiled from its sources (oracle/_ref, parity build):
the wheel's turn (SoftBody::compute_wheel_forces with no torque, softbody.cpp:691-744), the tyre contact
(tyre_contact, static_world.cpp:53-83) and each wheel's patch sharing its grip (World::collide_static,
world.cpp:871-898) - node and beam states bitwise equal after 1,485 substeps of a wheeled car landing sideways, rolling
and hitting a wall, and after three frames of a small wheeled fleet with collision skins."""
import numpy as np
import pytest

from beamlab_b200 import rigs, world_from_rig
from beamlab_b200.world import BeamLabError
from gpu_adapter import GpuWorld
from test_gpu_parity import assert_same

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("variant", ["plain", "drag", "grip", "launches"])
def test_gpu_wheeled_car_matches_reference(ref_lib, variant):
    """plain: the car as built; drag: with air drag (RoR's per-node drag skips the tyre nodes); grip: the world's
    tyre grip at 0.6; launches: the frames' kernels launched one by one instead of as CUDA graphs."""
    from oracle.oracle import RefWorld, build_world
    rig = rigs.wheeled_car()
    if variant == "drag":
        rig["bodies"][0]["params"].update({"air_drag": 0.05, "aero_cda": 0.8})
    if variant == "grip":
        rig["settings"]["tyre_grip"] = 0.6
    gw = GpuWorld(rig, graphs=False) if variant == "launches" else GpuWorld(rig)
    rw = build_world(RefWorld, rig, multithreaded=False)
    for f in range(45):
        gw.step_substeps(33)
        rw.step_substeps(33)
        if f in (5, 13, 22, 30, 44):
            assert_same(gw, rw, 1, f"frame {f}")
    b = rig["bodies"][0]
    tn = np.concatenate([w["nodes"] for w in b["wheels"]])
    assert rw.body(0)["static_contacts"] > 0 or rw.nodes(0)["pos"][tn, 1].min() < 0.05  # (the tyres reached the ground)


def test_gpu_wheeled_fleet_matches_reference(ref_lib):
    """Six wheeled lattice vehicles with collision skins on the heightfield, batched in one World: bitwise the
    reference's after three uneven frames."""
    from oracle.oracle import RefWorld, build_world
    rig = rigs.fleet(6, seed=9, median_nodes=600, min_nodes=200, max_nodes=1500, terrain_size=300.0, terrain_samples=257)
    for b in rig["bodies"]:
        b["pos"][:, 1] -= 0.28  # (the tyres start a few cm over the ground: they land within the frames)
    gw = GpuWorld(rig)
    rw = build_world(RefWorld, rig, multithreaded=False)
    for n in (33, 20, 33, 33, 33):
        gw.step_substeps(n)
        rw.step_substeps(n)
    assert_same(gw, rw, len(rig["bodies"]), "fleet")
    assert sum(rw.body(b)["static_contacts"] for b in range(len(rig["bodies"]))) > 0


def test_gpu_wheel_rejections():
    """A node on two wheels, or a wheel's node out of the body, is refused at add_body."""
    rig = rigs.wheeled_car()
    w = rig["bodies"][0]["wheels"]
    w[1]["nodes"] = np.concatenate([w[1]["nodes"], w[0]["nodes"][:1]])
    with pytest.raises(BeamLabError, match="unsupported"):
        world_from_rig(rig)
    rig = rigs.wheeled_car()
    rig["bodies"][0]["wheels"][0]["axle0"] = len(rig["bodies"][0]["mass"])
    with pytest.raises(BeamLabError, match="invalid"):
        world_from_rig(rig)


@pytest.mark.parametrize("shock_type,soft_bump", [(1, False), (2, False), (2, True), (3, False)])
def test_gpu_shocks_match_reference(ref_lib, shock_type, soft_bump):
    """The wheeled car hung on shocks (three a wheel from its inner hub; SoftBody::compute_shock_forces,
    softbody.cpp:472-566: bounded, progressive with and without soft bump stops, split damping), landing, rolling
    and hitting the wall: node and beam states bitwise the reference's after 1,485 substeps."""
    from oracle.oracle import RefWorld, build_world
    rig = rigs.wheeled_car(shocks=dict(rigs.SHOCK_TYPES[shock_type], soft_bump=soft_bump))
    gw = GpuWorld(rig)
    rw = build_world(RefWorld, rig, multithreaded=False)
    for f in range(45):
        gw.step_substeps(33)
        rw.step_substeps(33)
        if f in (13, 22, 44):
            assert_same(gw, rw, 1, f"frame {f}")
    js = [x["beam"] for x in rig["bodies"][0]["shocks"]]
    assert np.all(rw.beams(0)["stress"][js] != 0)  # (the shocks carry the car)


def test_gpu_shock_rejections():
    """A BF_SHOCK beam without its shock, or a shock on a plain beam, is refused at add_body."""
    rig = rigs.wheeled_car(shocks=rigs.SHOCK_TYPES[1])
    rig["bodies"][0]["shocks"] = rig["bodies"][0]["shocks"][1:]
    with pytest.raises(BeamLabError, match="invalid"):
        world_from_rig(rig)
    rig = rigs.wheeled_car(shocks=rigs.SHOCK_TYPES[1])
    rig["bodies"][0]["shocks"][0]["beam"] = 0
    with pytest.raises(BeamLabError, match="invalid"):
        world_from_rig(rig)


@pytest.mark.parametrize("torque,brake", [(400.0, 1500.0), (-300.0, 600.0)])
def test_gpu_driven_wheels_match_reference(ref_lib, torque, brake):
    """The wheeled car (no wall) driven: its rear wheels' torque spread over their tyre nodes along their tangents with
    the reaction on their arms, then every wheel braked (the stop torque against the average speed and the last
    reaction) - SoftBody::compute_wheel_forces, softbody.cpp:691-767, with the controller setting torque and brake every
    substep. Node and beam states and the wheels' speeds bitwise the reference's."""
    from oracle.oracle import RefWorld, build_world
    rig = rigs.wheeled_car(speed=4.0, yaw=0.0, wall=False)
    gw = GpuWorld(rig)
    rw = build_world(RefWorld, rig, multithreaded=False)
    h = gw.h[0]
    wheels = rig["bodies"][0]["wheels"]
    top = 0.0
    for f in range(50):
        if f in (0, 30):
            for k, w in enumerate(wheels):
                t, b = (torque if w["propulsed"] else 0.0, 0.0) if f == 0 else (0.0, brake)
                h.set_wheel_drive(k, t, b)
                rw.set_wheel_drive(0, k, t, b)
        gw.step_substeps(33)
        rw.step_substeps(33)
        if f in (12, 29, 49):
            assert_same(gw, rw, 1, f"frame {f}")
            gs, rs = h.wheels(), rw.wheels(0, len(wheels))
            assert np.array_equal(gs["speed"].view(np.uint32), rs["speed"].view(np.uint32)), f"frame {f}: wheel speeds"
            assert np.array_equal(gs["avg_speed"].view(np.uint32), rs["avg_speed"].view(np.uint32))
            gsp, gspin = h.wheel_speed()
            assert np.float32(gsp) == rs["wheel_speed"] and np.float32(gspin) == rs["wheel_spin"]
            top = max(top, float(np.abs(rs["speed"]).max()))
    assert top > 5.0  # (the driven wheels spun up before the brakes held them)


def test_gpu_wheel_state_survives_a_recommit(ref_lib):
    """A body added while a driven, braked wheeled car rolls (the context commits its bodies again, pulling every
    state back from the device - the wheels' speeds, last torques and reactions with them): both bodies and the wheels'
    speeds stay bitwise the reference's, which takes the new body into its running world the same way."""
    from beamlab_b200.world import SoftBody
    from oracle.oracle import RefWorld, build_world
    rig = rigs.wheeled_car(speed=4.0, yaw=0.0, wall=False)
    gw = GpuWorld(rig)
    rw = build_world(RefWorld, rig, multithreaded=False)
    h = gw.h[0]
    wheels = rig["bodies"][0]["wheels"]
    for k, w in enumerate(wheels):
        t, b = (300.0 if w["propulsed"] else 0.0), (0.0 if w["propulsed"] else 200.0)
        h.set_wheel_drive(k, t, b)
        rw.set_wheel_drive(0, k, t, b)
    for _ in range(10):
        gw.step_substeps(33)
        rw.step_substeps(33)
    extra = rigs.truss_car(4, speed=3.0, dims=(6, 3, 3))["bodies"][0]
    extra["pos"][:, 2] += 20.0
    gw.w.add_body(SoftBody.from_arrays(extra, name="extra"))
    gw.h = gw.w.bodies()
    rw.add_body(extra)
    for _ in range(10):
        gw.step_substeps(33)
        rw.step_substeps(33)
    assert_same(gw, rw, 2, "after the recommit")
    gs, rs = gw.h[0].wheels(), rw.wheels(0, len(wheels))
    assert np.array_equal(gs["speed"].view(np.uint32), rs["speed"].view(np.uint32))
    assert np.array_equal(gs["avg_speed"].view(np.uint32), rs["avg_speed"].view(np.uint32))
