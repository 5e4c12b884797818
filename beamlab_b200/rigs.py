"""Seeded synthetic rigs of the benchmark shapes, as plain numpy arrays.

A rig is a dict ``{"settings": {...}, "statics": {...}, "bodies": [body, ...]}``; a body holds its nodes
(``pos``, ``vel``, ``mass``, ``node_flags``, ``friction``, ``radius``), its beams (``ab``, ``k``, ``d``, ``strength``,
``deform``, ``beam_type``, ``beam_flags``) and its knobs (``params``) - the arguments of the reference's builder calls
``SoftBody::add_node`` / ``add_beam`` (softbody.cpp:8-40) before ``finalize``. The same arrays feed the GPU world
(beamlab_b200.World) and the CPU oracles, so both step the very same rig.

Random numbers come from a xorshift32 generator seeded like the reference test suite's ``TRng``
(tests/test_physics.cpp:44-54: state = seed * 2654435761 + 1; uniform = the low 24 bits / 2^24).
"""
from __future__ import annotations

import math

import numpy as np

# node flags (softbody.h:29-39) and beam types (softbody.h:60)
NF_GROUND, NF_FIXED, NF_TYRE, NF_RIM, NF_CONTACTER = 1, 2, 4, 8, 16
BT_NORMAL, BT_ROPE, BT_SUPPORT = 0, 1, 2
BF_SHOCK = 1 << 6  # beam flags (softbody.h:62-69): a shock's beam
SURF_GRASS, SURF_CONCRETE = 0, 3
GRASS_STATIC_FRICTION = 0.80  # ground model "grass", ms (static_world.cpp:97)


class TRng:
    """xorshift32 with the reference test suite's seeding (tests/test_physics.cpp:44-54)."""

    def __init__(self, seed: int):
        self.s = (seed * 2654435761 + 1) & 0xFFFFFFFF

    def next(self) -> int:
        s = self.s
        s ^= (s << 13) & 0xFFFFFFFF
        s ^= s >> 17
        s ^= (s << 5) & 0xFFFFFFFF
        self.s = s
        return s

    def uni(self) -> np.float32:
        return np.float32(self.next() & 0xFFFFFF) / np.float32(0x1000000)

    def range(self, a: float, b: float) -> np.float32:
        a32, b32 = np.float32(a), np.float32(b)
        return np.float32(a32 + (b32 - a32) * self.uni())

    def gauss(self) -> float:
        """A standard normal draw (Box-Muller over two uniforms, in double precision)."""
        u1 = 1.0 - float(self.uni())
        u2 = float(self.uni())
        return math.sqrt(-2.0 * math.log(u1)) * math.cos(2.0 * math.pi * u2)


def flat_terrain(nx=81, nz=41, cell=1.0, origin=(-40.0, -20.0), height=0.0, surface=SURF_GRASS) -> dict:
    """A flat heightfield (Heightfield::create, static_world.cpp:147-152) of nz rows of nx samples."""
    return {"nx": nx, "nz": nz, "cell": cell, "origin": origin,
            "heights": np.full((nz, nx), height, np.float32),
            "surfaces": np.full((nz, nx), surface, np.uint8)}


def lattice_body(rng: TRng, dims=(20, 4, 5), spacing=0.25, origin=(0.0, 0.0, 0.0), jitter=0.002,
                 mass_range=(4.0, 6.0), k_median=2e6, k_sigma=0.3, damping=500.0, deform=5e4, strength=1.5e5,
                 velocity=(0.0, 0.0, 0.0), ground_friction=1.0) -> dict:
    """A jittered lattice truss: nodes on an nx x ny x nz grid (x fastest-varying last: index = (ix*ny + iy)*nz + iz),
    beams between every pair of lattice neighbours (|di|,|dj|,|dk| <= 1) whose jittered distance is within
    sqrt(3) * spacing, stiffness log-normal about k_median."""
    nx, ny, nz = dims
    n = nx * ny * nz
    pos = np.zeros((n, 3), np.float32)
    mass = np.zeros(n, np.float32)
    sp = np.float32(spacing)
    for ix in range(nx):
        for iy in range(ny):
            for iz in range(nz):
                i = (ix * ny + iy) * nz + iz
                jx, jy, jz = rng.range(-jitter, jitter), rng.range(-jitter, jitter), rng.range(-jitter, jitter)
                pos[i] = (np.float32(origin[0]) + np.float32(ix) * sp + jx,
                          np.float32(origin[1]) + np.float32(iy) * sp + jy,
                          np.float32(origin[2]) + np.float32(iz) * sp + jz)
                mass[i] = rng.range(*mass_range)
    thr = np.float32(math.sqrt(3.0) * spacing)
    offsets = [(dx, dy, dz) for dx in (-1, 0, 1) for dy in (-1, 0, 1) for dz in (-1, 0, 1) if (dx, dy, dz) > (0, 0, 0)]
    ab, ks = [], []
    for ix in range(nx):
        for iy in range(ny):
            for iz in range(nz):
                a = (ix * ny + iy) * nz + iz
                for dx, dy, dz in offsets:
                    jx, jy, jz = ix + dx, iy + dy, iz + dz
                    if not (0 <= jx < nx and 0 <= jy < ny and 0 <= jz < nz):
                        continue
                    b = (jx * ny + jy) * nz + jz
                    d = pos[a] - pos[b]
                    dist = np.sqrt(np.float32(d[0] * d[0] + d[1] * d[1]) + np.float32(d[2] * d[2]))
                    if dist > thr:
                        continue
                    ab.append((a, b))
                    ks.append(np.float32(k_median * math.exp(k_sigma * rng.gauss())))
    m = len(ab)
    vel = np.tile(np.asarray(velocity, np.float32), (n, 1))
    return {
        "pos": pos, "vel": vel, "mass": mass,
        "node_flags": np.full(n, NF_GROUND | NF_CONTACTER, np.uint16),
        "friction": np.ones(n, np.float32), "radius": np.zeros(n, np.float32),
        "ab": np.asarray(ab, np.uint32).reshape(m, 2), "k": np.asarray(ks, np.float32),
        "d": np.full(m, damping, np.float32), "strength": np.full(m, strength, np.float32),
        "deform": np.full(m, deform, np.float32), "beam_type": np.zeros(m, np.uint8),
        "beam_flags": np.zeros(m, np.uint8),
        "params": {"ground_friction": ground_friction, "bounce": -1.0, "contact_push_max": 2.0, "contact_slop": 0.0,
                   "collision_radius": 0.05, "allow_deform": 1, "allow_break": 1, "ductile": 0, "can_sleep": 1,
                   "sleep_speed": 0.0},
    }


def lattice_body_fast(gen: np.random.Generator, dims=(20, 4, 5), spacing=0.25, origin=(0.0, 0.0, 0.0), jitter=0.002,
                      mass_range=(4.0, 6.0), k_median=2e6, k_sigma=0.3, damping=500.0, deform=5e4, strength=1.5e5,
                      velocity=(0.0, 0.0, 0.0), ground_friction=1.0) -> dict:
    """lattice_body's structure (node order, beam rule and order: node a ascending, then its forward neighbour
    offsets) with numpy's generator for the random draws, vectorized - for rigs of millions of beams."""
    nx, ny, nz = dims
    n = nx * ny * nz
    ix, iy, iz = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    sp = np.float32(spacing)
    jit = gen.uniform(-jitter, jitter, size=(n, 3)).astype(np.float32)
    pos = np.stack([np.float32(origin[0]) + ix.ravel().astype(np.float32) * sp,
                    np.float32(origin[1]) + iy.ravel().astype(np.float32) * sp,
                    np.float32(origin[2]) + iz.ravel().astype(np.float32) * sp], 1).astype(np.float32) + jit
    mass = gen.uniform(mass_range[0], mass_range[1], size=n).astype(np.float32)
    thr = np.float32(math.sqrt(3.0) * spacing)
    offsets = [(dx, dy, dz) for dx in (-1, 0, 1) for dy in (-1, 0, 1) for dz in (-1, 0, 1) if (dx, dy, dz) > (0, 0, 0)]
    A, Bn, O = [], [], []
    idx = np.arange(n).reshape(nx, ny, nz)
    for o, (dx, dy, dz) in enumerate(offsets):
        sx = slice(max(0, -dx), nx - max(0, dx)); sy = slice(max(0, -dy), ny - max(0, dy)); sz = slice(max(0, -dz), nz - max(0, dz))
        a = idx[sx, sy, sz].ravel()
        b = idx[slice(sx.start + dx, sx.stop + dx), slice(sy.start + dy, sy.stop + dy), slice(sz.start + dz, sz.stop + dz)].ravel()
        d = pos[a] - pos[b]
        dist = np.sqrt((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2])
        keep = dist <= thr
        A.append(a[keep]), Bn.append(b[keep]), O.append(np.full(int(keep.sum()), o))
    A, Bn, O = np.concatenate(A), np.concatenate(Bn), np.concatenate(O)
    order = np.lexsort((O, A))
    ab = np.stack([A[order], Bn[order]], 1).astype(np.uint32)
    m = len(ab)
    k = (k_median * np.exp(k_sigma * gen.standard_normal(m))).astype(np.float32)
    return {
        "pos": pos, "vel": np.tile(np.asarray(velocity, np.float32), (n, 1)), "mass": mass,
        "node_flags": np.full(n, NF_GROUND | NF_CONTACTER, np.uint16),
        "friction": np.ones(n, np.float32), "radius": np.zeros(n, np.float32),
        "ab": ab, "k": k, "d": np.full(m, damping, np.float32), "strength": np.full(m, strength, np.float32),
        "deform": np.full(m, deform, np.float32), "beam_type": np.zeros(m, np.uint8), "beam_flags": np.zeros(m, np.uint8),
        "params": {"ground_friction": ground_friction, "bounce": -1.0, "contact_push_max": 2.0, "contact_slop": 0.0,
                   "collision_radius": 0.05, "allow_deform": 1, "allow_break": 1, "ductile": 0, "can_sleep": 1,
                   "sleep_speed": 0.0},
    }


def lattice_tris(dims) -> np.ndarray:
    """Collision triangles over the outer faces of an nx x ny x nz lattice (node index (ix*ny + iy)*nz + iz): each face
    quad as two triangles wound so that cross(b - a, c - a) points out of the body - the SoftBody::add_triangle calls
    (softbody.h:958) that give a lattice truss a skin other bodies' nodes collide with (hull triangles when one-sided)."""
    nx, ny, nz = dims
    idx = lambda ix, iy, iz: (ix * ny + iy) * nz + iz
    tris = []

    def face(corner, nu, nv, outward):
        # corner(i, j) -> node; (u, v) spans the face; outward: cross(u, v) points out of the body
        for i in range(nu - 1):
            for j in range(nv - 1):
                p00, p10, p01, p11 = corner(i, j), corner(i + 1, j), corner(i, j + 1), corner(i + 1, j + 1)
                if outward:
                    tris.append((p00, p10, p11)), tris.append((p00, p11, p01))
                else:
                    tris.append((p00, p11, p10)), tris.append((p00, p01, p11))
    face(lambda i, j: idx(0, i, j), ny, nz, False)            # -x: cross(y, z) = +x points in
    face(lambda i, j: idx(nx - 1, i, j), ny, nz, True)        # +x
    face(lambda i, j: idx(i, 0, j), nx, nz, True)             # -y: cross(x, z) = -y points out
    face(lambda i, j: idx(i, ny - 1, j), nx, nz, False)       # +y
    face(lambda i, j: idx(i, j, 0), nx, ny, False)            # -z: cross(x, y) = +z points in
    face(lambda i, j: idx(i, j, nz - 1), nx, ny, True)        # +z
    return np.asarray(tris, np.uint32).reshape(-1, 3)


def crash_pair(seed: int = 1, speed_a: float = 12.0, speed_b: float = 12.0, gap: float = 0.3, hull: bool = False,
               dims=(12, 4, 5), sleeping: bool = False) -> dict:
    """Two lattice trusses with collision skins (lattice_tris) head on along x over flat ground: body 0 at speed_a
    towards +x, body 1 at speed_b towards -x, their fronts `gap` apart; hull: one-sided (hull) skins."""
    rng = TRng(seed)
    length = (dims[0] - 1) * 0.25
    a = lattice_body(rng, dims=dims, origin=(-gap / 2 - length, 0.05, -0.5), velocity=(speed_a, 0.0, 0.0),
                     ground_friction=0.8 / GRASS_STATIC_FRICTION)
    b = lattice_body(rng, dims=dims, origin=(gap / 2, 0.05, -0.45), velocity=(-speed_b, 0.0, 0.0),
                     ground_friction=0.8 / GRASS_STATIC_FRICTION)
    for body in (a, b):
        body["tris"] = lattice_tris(dims)
        body["tri_two_sided"] = np.full(len(body["tris"]), 0 if hull else 1, np.uint8)
    return {
        "settings": {"gravity": (0.0, -9.81, 0.0), "dt": 0.0005, "sleeping": sleeping},
        "statics": {"terrain": flat_terrain(), "boxes": [], "build_grid": True},
        "bodies": [a, b],
        "name": f"crash_pair(seed={seed}, {speed_a}, {speed_b}, hull={hull})",
    }


def drop_pair(seed: int = 1, height: float = 7.0, dims=(8, 3, 4), hull: bool = False) -> dict:
    """A lattice truss at rest on flat ground and another dropped onto it from `height` m above (both with collision
    skins; sleeping on): the one below falls asleep before the other lands, and is woken by it."""
    rng = TRng(seed)
    b = lattice_body(rng, dims=dims, origin=(-1.0, 0.02, -0.4), ground_friction=0.8 / GRASS_STATIC_FRICTION)
    a = lattice_body(rng, dims=dims, origin=(-0.9, 0.02 + height, -0.35), ground_friction=0.8 / GRASS_STATIC_FRICTION)
    for body in (b, a):
        body["tris"] = lattice_tris(dims)
        body["tri_two_sided"] = np.full(len(body["tris"]), 0 if hull else 1, np.uint8)
    return {
        "settings": {"gravity": (0.0, -9.81, 0.0), "dt": 0.0005, "sleeping": True},
        "statics": {"terrain": flat_terrain(), "boxes": [], "build_grid": True},
        "bodies": [b, a],
        "name": f"drop_pair(seed={seed}, height={height}, hull={hull})",
    }


def truss_car(seed: int = 1, speed: float = 15.0, dims=(20, 4, 5)) -> dict:
    """The plain explicit mass-spring truss car: a 20 x 4 x 5 node lattice (4.75 m long, 0.75 m high, 1 m wide) at
    0.25 m with +-2 mm jitter, node mass uniform in [4, 6] kg, beams to every neighbour within sqrt(3) * 0.25 m
    (about 3,100), k log-normal (median 2e6 N/m, sigma 0.3), d = 500 N s/m, plastic-deform threshold 5e4 N, break
    threshold 1.5e5 N; gravity 9.81 m/s^2 over flat grass ground at y = 0 (friction 0.8: the grass model's static
    coefficient, so the body's ground friction factor is 1); driving at `speed` m/s along +x into a rigid concrete
    wall 2 m ahead; dt = 0.5 ms."""
    rng = TRng(seed)
    body = lattice_body(rng, dims=dims, origin=(-6.0, 0.05, -0.5), velocity=(speed, 0.0, 0.0),
                        ground_friction=0.8 / GRASS_STATIC_FRICTION)
    front = -6.0 + (dims[0] - 1) * 0.25
    wall = {"center": (front + 2.0 + 0.25, 1.0, 0.0), "half": (0.25, 1.0, 2.0), "rot": (0.0, 0.0, 0.0, 1.0),
            "surface": SURF_CONCRETE}
    return {
        "settings": {"gravity": (0.0, -9.81, 0.0), "dt": 0.0005},
        "statics": {"terrain": flat_terrain(), "boxes": [wall], "build_grid": True},
        "bodies": [body],
        "name": f"truss_car(seed={seed})",
    }


def add_wheels(body: dict, dims, radius: float = 0.3, rays: int = 12, width: float = 0.2, gap: float = 0.1,
               tyre_mass: float = 0.8, hub_mass: float = 5.0, k_tyre: float = 3e5, d_tyre: float = 300.0,
               k_hub: float = 2e6, d_hub: float = 500.0, strength: float = 1e7, shocks: dict | None = None) -> dict:
    """Four free-rolling wheel rings on a lattice body (lattice_body / lattice_body_fast node order): each wheel two hub
    nodes on an axle along z beside the lattice's bottom layer, a quarter of the length in from each end, `gap` m out
    from the side, `width` m apart (axle0 the one of the lesser z, as the reference's vehicle builder spawns them), and
    `rays` spokes of two tyre nodes (even: axle0's ring, odd: axle1's) at `radius` round the hubs - 24 tyre nodes a
    wheel with the 12 rays. Beams: each tyre node to both hubs, each ray's pair, the two rings, one diagonal a ray;
    each hub to the lattice's bottom nodes about its axle and the two hubs to each other. Tyre nodes: NF_GROUND |
    NF_TYRE | NF_CONTACTER; they and the hubs move at the body's starting velocity. The rear wheels (the lesser x) are
    the propelled ones; each wheel's reaction arm is the lattice node over its axle, its near axle node the inner hub.
    shocks: a Shock's type and rates
    (softbody.h:88-101) - the beams from each inner hub to the lattice's second layer become shocks of them (BF_SHOCK).
    Appends the nodes and beams in place, sets body["wheels"] (and body["shocks"]), returns the body."""
    nx, ny, nz = dims
    pos = body["pos"]
    n0, m0 = len(pos), len(body["k"])
    v0 = np.asarray(body["vel"][0], np.float32)
    new_pos, new_mass, new_flags, ab, ks, ds = [], [], [], [], [], []

    def node(p, m, flags):
        new_pos.append(p), new_mass.append(m), new_flags.append(flags)
        return n0 + len(new_pos) - 1

    shock_beams = []

    def beam(a, b, k, d, shock=False):
        if shock:
            shock_beams.append(len(ab))
        ab.append((a, b)), ks.append(k), ds.append(d)

    wheels, blocks = [], []
    xs = sorted({max(0, (nx - 1) // 4), min(nx - 1, nx - 1 - (nx - 1) // 4)})
    for ix in xs:
        for side in (0, 1):
            iz = 0 if side == 0 else nz - 1
            base = pos[(ix * ny) * nz + iz]
            zi = float(base[2]) + (-gap if side == 0 else gap)
            zo = zi + (-width if side == 0 else width)
            y = float(base[1])
            x = float(base[0])
            b_start, v_start, ln_max = len(ab), len(new_pos), 0
            inner = node((x, y, zi), hub_mass, NF_GROUND | NF_CONTACTER)
            outer = node((x, y, zo), hub_mass, NF_GROUND | NF_CONTACTER)
            a0, a1 = (outer, inner) if side == 0 else (inner, outer)
            beam(a0, a1, k_hub, d_hub)
            for jx in range(max(0, ix - 1), min(nx, ix + 2)):
                for jy in range(min(2, ny)):
                    ln = (jx * ny + jy) * nz + iz
                    ln_max = max(ln_max, ln)
                    beam(ln, inner, k_hub, d_hub, shock=shocks is not None and jy == 1)
                    beam(ln, outer, k_hub, d_hub)
            tyre = []
            for r in range(rays):
                ang = 2.0 * math.pi * r / rays
                dx, dy = radius * math.cos(ang), radius * math.sin(ang)
                e = node((x + dx, y + dy, float(new_pos[a0 - n0][2])), tyre_mass, NF_GROUND | NF_TYRE | NF_CONTACTER)
                o = node((x + dx, y + dy, float(new_pos[a1 - n0][2])), tyre_mass, NF_GROUND | NF_TYRE | NF_CONTACTER)
                tyre += [e, o]
            for r in range(rays):
                e, o = tyre[2 * r], tyre[2 * r + 1]
                e2, o2 = tyre[(2 * r + 2) % (2 * rays)], tyre[(2 * r + 3) % (2 * rays)]
                for t in (e, o):
                    beam(t, a0, k_tyre, d_tyre)
                    beam(t, a1, k_tyre, d_tyre)
                beam(e, o, k_tyre, d_tyre)
                beam(e, e2, k_tyre, d_tyre)
                beam(o, o2, k_tyre, d_tyre)
                beam(e, o2, k_tyre, d_tyre)
            arm = (ix * ny + min(1, ny - 1)) * nz + iz  # (the lattice node over the axle: the drive's reaction arm)
            wheels.append({"axle0": a0, "axle1": a1, "nodes": np.asarray(tyre, np.uint32), "radius": radius,
                           "width": width, "mass": float(np.float32(tyre_mass) * np.float32(len(tyre))),
                           "propulsed": 1 if ix == xs[0] else 0, "arm": arm, "near_attach": inner})
            blocks.append((ln_max, v_start, len(new_pos), b_start, len(ab)))
    k = len(new_pos)
    body["pos"] = np.concatenate([pos, np.asarray(new_pos, np.float32)]).astype(np.float32)
    body["vel"] = np.concatenate([body["vel"], np.tile(v0, (k, 1))]).astype(np.float32)
    body["mass"] = np.concatenate([body["mass"], np.asarray(new_mass, np.float32)])
    body["node_flags"] = np.concatenate([body["node_flags"], np.asarray(new_flags, np.uint16)])
    body["friction"] = np.concatenate([body["friction"], np.ones(k, np.float32)])
    body["radius"] = np.concatenate([body["radius"], np.zeros(k, np.float32)])
    m = len(ab)
    body["ab"] = np.concatenate([body["ab"], np.asarray(ab, np.uint32).reshape(m, 2)])
    body["k"] = np.concatenate([body["k"], np.asarray(ks, np.float32)])
    body["d"] = np.concatenate([body["d"], np.asarray(ds, np.float32)])
    body["strength"] = np.concatenate([body["strength"], np.full(m, strength, np.float32)])
    body["deform"] = np.concatenate([body["deform"], np.full(m, strength, np.float32)])
    body["beam_type"] = np.concatenate([body["beam_type"], np.zeros(m, np.uint8)])
    body["beam_flags"] = np.concatenate([body["beam_flags"], np.zeros(m, np.uint8)])
    body["wheels"] = wheels
    sb = [m0 + q for q in shock_beams]
    body["beam_flags"][sb] |= BF_SHOCK
    assert len(body["k"]) == m0 + m
    if np.all(np.diff(body["ab"][:m0, 0].astype(np.int64)) >= 0):
        # each wheel's nodes right after the last lattice node its hubs hold, its beams right after that node's beams:
        # every 32 consecutive nodes' beams and neighbours then lie within a few lattice slices of each other (the
        # kernels' 4-byte incidences), as a builder numbering the wheels with the axles they hang on would
        order, border = [], []
        lat_ab = body["ab"][:m0, 0].astype(np.int64)
        nxt, bnxt = 0, 0
        for ln_max, v0_, v1_, b0_, b1_ in sorted(blocks, key=lambda t: t[0]):
            order += list(range(nxt, ln_max + 1)) + list(range(n0 + v0_, n0 + v1_))
            nxt = ln_max + 1
            cut = int(np.searchsorted(lat_ab, ln_max, side="right"))
            border += list(range(bnxt, cut)) + list(range(m0 + b0_, m0 + b1_))
            bnxt = cut
        order += list(range(nxt, n0))
        border += list(range(bnxt, m0))
        order, border = np.asarray(order), np.asarray(border)
        assert len(order) == n0 + k and len(border) == m0 + m
        perm = np.empty_like(order)
        perm[order] = np.arange(len(order))
        for key in ("pos", "vel", "mass", "node_flags", "friction", "radius"):
            body[key] = np.ascontiguousarray(body[key][order])
        for key in ("ab", "k", "d", "strength", "deform", "beam_type", "beam_flags"):
            body[key] = np.ascontiguousarray(body[key][border])
        body["ab"] = perm[body["ab"]].astype(np.uint32)
        if "tris" in body:
            body["tris"] = perm[np.asarray(body["tris"], np.int64)].astype(np.uint32)
        for w in wheels:
            w["axle0"], w["axle1"] = int(perm[w["axle0"]]), int(perm[w["axle1"]])
            w["arm"], w["near_attach"] = int(perm[w["arm"]]), int(perm[w["near_attach"]])
            w["nodes"] = perm[w["nodes"].astype(np.int64)].astype(np.uint32)
        bperm = np.empty_like(border)
        bperm[border] = np.arange(len(border))
        sb = [int(bperm[j]) for j in sb]
    if shocks is not None:
        body["shocks"] = [dict(shocks, beam=j) for j in sorted(sb)]
        assert np.count_nonzero(body["beam_flags"] & BF_SHOCK) == len(sb)
    return body


SHOCK_TYPES = {
    1: {"type": 1, "spring": 1.5e5, "damp": 3000.0, "short_bound": 0.1, "long_bound": 0.1, "bound_spring": 2e6},
    2: {"type": 2, "spring_in": 1.5e5, "damp_in": 3000.0, "prog_spring_in": 0.5, "prog_damp_in": 0.5, "spring_out": 1.5e5,
        "damp_out": 2500.0, "prog_spring_out": 0.5, "prog_damp_out": 0.5, "short_bound": 0.1, "long_bound": 0.1,
        "bound_spring": 2e6},
    3: {"type": 3, "spring_in": 1.5e5, "damp_in": 3000.0, "spring_out": 1.5e5, "damp_out": 3000.0, "damp_in_slow": 1.0,
        "split_in": 0.5, "damp_in_fast": 0.5, "damp_out_slow": 1.2, "split_out": 0.5, "damp_out_fast": 0.6,
        "short_bound": 0.1, "long_bound": 0.1, "bound_spring": 2e6},
}


def wheeled_car(seed: int = 1, speed: float = 12.0, yaw: float = 0.3, dims=(14, 3, 5), wall: bool = True,
                height: float = 0.45, shocks: dict | None = None) -> dict:
    """A lattice truss on four wheel rings (add_wheels), `height` m up over flat grass, rolling at `speed` m/s at
    `yaw` rad off +x (so its tyres slip sideways as they land) towards a concrete wall; dt = 0.5 ms."""
    rng = TRng(seed)
    vel = (speed * math.cos(yaw), 0.0, speed * math.sin(yaw))
    body = lattice_body(rng, dims=dims, origin=(-6.0, height, -0.5), velocity=vel, ground_friction=0.8 / GRASS_STATIC_FRICTION)
    add_wheels(body, dims, shocks=shocks)
    front = -6.0 + (dims[0] - 1) * 0.25
    boxes = []
    if wall:
        boxes.append({"center": (front + 4.0 + 0.25, 1.0, 0.0), "half": (0.25, 1.0, 3.0), "rot": (0.0, 0.0, 0.0, 1.0),
                      "surface": SURF_CONCRETE})
    return {
        "settings": {"gravity": (0.0, -9.81, 0.0), "dt": 0.0005},
        "statics": {"terrain": flat_terrain(), "boxes": boxes, "build_grid": True},
        "bodies": [body],
        "name": f"wheeled_car(seed={seed}, speed={speed}, yaw={yaw})",
    }


def rig_counts(rig: dict) -> tuple[int, int]:
    """(nodes, beams) over the rig's bodies."""
    return (sum(len(b["mass"]) for b in rig["bodies"]), sum(len(b["k"]) for b in rig["bodies"]))


def bumpy_terrain(rng: TRng, nx=129, nz=129, cell=0.5, origin=(-32.0, -32.0), amplitude=0.3, surfaces=(0,)) -> dict:
    """A seeded heightfield: a sum of a few random sine waves (amplitude in m), each sample's surface drawn from
    `surfaces`."""
    xs = np.arange(nx, dtype=np.float64) * cell + origin[0]
    zs = np.arange(nz, dtype=np.float64) * cell + origin[1]
    X, Z = np.meshgrid(xs, zs)
    h = np.zeros_like(X)
    for _ in range(4):
        kx, kz = float(rng.range(-0.6, 0.6)), float(rng.range(-0.6, 0.6))
        ph = float(rng.range(0.0, 6.283))
        h += np.sin(kx * X + kz * Z + ph)
    h *= amplitude / 4.0
    surf = np.zeros((nz, nx), np.uint8)
    for iz in range(nz):
        for ix in range(nx):
            surf[iz, ix] = surfaces[rng.next() % len(surfaces)]
    return {"nx": nx, "nz": nz, "cell": cell, "origin": origin, "heights": h.astype(np.float32), "surfaces": surf}


def stress_rig(seed: int = 7) -> dict:
    """A small rig that takes every branch of the explicit path: rope and support beams, weak beams that yield and
    break, a ductile body, anchored nodes, node friction and radii, bumpy ground of grass, mud and sand, a rotated box,
    a yielding box (max force) and a cylinder in the way."""
    rng = TRng(seed)
    bodies = []
    for bi, (dims, origin, vel, ductile) in enumerate((
            ((8, 3, 3), (-8.0, 0.4, -0.4), (25.0, -2.0, 0.5), 0),
            ((6, 3, 2), (-8.0, 0.5, 3.0), (18.0, 0.0, -1.0), 1),
            ((5, 2, 2), (4.0, 0.6, -4.0), (-3.0, 0.0, 9.0), 0))):
        b = lattice_body(rng, dims=dims, origin=origin, velocity=vel, strength=2.5e4, deform=8e3,
                         k_median=6e5, damping=300.0)
        m = len(b["k"])
        for j in range(m):
            r = rng.next() % 10
            if r == 0:
                b["beam_type"][j] = BT_ROPE
            elif r == 1:
                b["beam_type"][j] = BT_SUPPORT
            elif r == 2:
                b["beam_flags"][j] = 4  # BF_NO_DEFORM
            elif r == 3:
                b["beam_flags"][j] = 8  # BF_NO_BREAK
        n = len(b["mass"])
        b["friction"] = np.asarray([rng.range(0.5, 1.5) for _ in range(n)], np.float32)
        b["radius"] = np.asarray([rng.range(0.0, 0.03) for _ in range(n)], np.float32)
        if bi == 2:
            b["node_flags"][0] |= NF_FIXED  # an anchor (and a zero-mass node, inverse mass 0 too)
            b["mass"][1] = 0.0
        b["params"].update({"ductile": ductile, "contact_slop": 0.001 * bi, "contact_push_max": 2.0 - 0.5 * bi,
                            "bounce": 0.3 if bi == 1 else -1.0})
        bodies.append(b)
    half_sin = math.sin(0.3)
    statics = {
        "terrain": bumpy_terrain(rng, surfaces=(0, 0, 2, 5, 6)),
        "boxes": [
            {"center": (0.0, 0.5, 0.0), "half": (0.3, 0.5, 1.5), "rot": (0.0, half_sin, 0.0, math.cos(0.3)), "surface": 3},
            {"center": (1.5, 0.4, 3.3), "half": (0.4, 0.4, 0.6), "rot": (0.1, 0.0, 0.0, math.sqrt(1 - 0.01)),
             "surface": 8, "max_force": 4000.0},
            {"center": (0.0, -0.5, 0.0), "half": (40.0, 0.2, 40.0), "rot": (0.0, 0.0, 0.0, 1.0), "surface": 4},
        ],
        "cylinders": [{"base": (2.0, -0.5, -1.0), "radius": 0.25, "height": 2.0, "surface": 9}],
        "build_grid": True,
    }
    return {"settings": {"gravity": (0.0, -9.81, 0.0), "dt": 0.0005}, "statics": statics, "bodies": bodies,
            "name": f"stress_rig(seed={seed})"}


def fleet(n_vehicles: int = 256, seed: int = 3, median_nodes: float = 3000.0, sigma: float = 0.6,
          min_nodes: int = 500, max_nodes: int = 20000, terrain_size: float = 1000.0, terrain_samples: int = 2048,
          amplitude: float = 2.0, skins: bool = True, wheels: bool = True, layout: str = "grid") -> dict:
    """A batched fleet of lattice trusses with log-normal node counts (median `median_nodes`, clipped to
    [min_nodes, max_nodes]), each driving at a speed uniform in [5, 30] m/s with a random yaw over a square heightfield
    of terrain_samples^2 samples spanning terrain_size metres, `amplitude` m of seeded smooth noise (two octaves of
    bilinear value noise). layout "grid": vehicles start on a grid 40 m apart, each on its own heading (few meet);
    "pairs": vehicles two by two on a grid 40 m apart, each pair head-on along a random axis, each vehicle its reach,
    0.15 m and its speed times the pair's meeting time (uniform in [0.02, 0.12] s) from the pair's centre - every pair
    crashes within its first few frames and stays in contact. With skins (lattice_tris) vehicles that meet collide; with wheels each stands on
    four wheel rings of 24 tyre nodes (add_wheels). Random draws: numpy's PCG64 seeded with `seed` (the skins and
    wheels draw none)."""
    gen = np.random.default_rng(seed)
    cell = terrain_size / (terrain_samples - 1)
    half = terrain_size / 2

    def octave(m, amp):  # bilinear value noise over an m x m lattice of random heights
        g = gen.uniform(-1.0, 1.0, size=(m, m))
        t = np.linspace(0, m - 1, terrain_samples)
        i0 = np.minimum(np.floor(t).astype(int), m - 2)
        f = t - i0
        rows = g[i0] * (1 - f)[:, None] + g[i0 + 1] * f[:, None]
        return amp * (rows[:, i0] * (1 - f)[None, :] + rows[:, i0 + 1] * f[None, :])
    h = (octave(33, amplitude) + octave(129, amplitude * 0.25)).astype(np.float32)
    terrain = {"nx": terrain_samples, "nz": terrain_samples, "cell": cell, "origin": (-half, -half), "heights": h,
               "surfaces": np.zeros((terrain_samples, terrain_samples), np.uint8)}
    if layout not in ("grid", "pairs"):
        raise ValueError(f"unknown layout {layout}")
    slots = n_vehicles if layout == "grid" else (n_vehicles + 1) // 2
    side = int(math.ceil(math.sqrt(slots)))
    sp = 0.25  # (lattice_body_fast's spacing)

    def dims_of(nn):  # lattice dims in a car's proportions: length 4, width 1.25, height 1
        unit = (nn / 5.0) ** (1.0 / 3.0)
        nx = max(2, int(round(4 * unit / 1.7)))
        nz = max(2, int(round(1.25 * unit / 1.7 * 1.2)))
        ny = max(2, int(round(nn / (nx * nz))))
        return nx, ny, nz

    bodies = []
    pair = None  # (the pair's centre, axis, the first vehicle's reach and speed) while its second is drawn
    for v in range(n_vehicles):
        nn = int(np.clip(median_nodes * math.exp(sigma * gen.standard_normal()), min_nodes, max_nodes))
        nx, ny, nz = dims_of(nn)
        reach = 0.5 * sp * math.hypot(nx - 1, nz - 1)  # (the lattice's horizontal half-diagonal)
        speed = float(gen.uniform(5.0, 30.0))
        yaw = float(gen.uniform(0.0, 2 * math.pi))
        if layout == "grid":
            gx, gz = v % side, v // side
            x0, z0 = -half + 60 + gx * 40.0, -half + 60 + gz * 40.0
            vel = (speed * math.cos(yaw), 0.0, speed * math.sin(yaw))
        else:
            if v % 2 == 0:
                gx, gz = (v // 2) % side, (v // 2) // side
                pair = ((-half + 60 + gx * 40.0, -half + 60 + gz * 40.0), (math.cos(yaw), math.sin(yaw)), reach, speed,
                        float(gen.uniform(0.02, 0.12)))
            (cx, cz), (ux, uz), _, _, t_meet = pair
            away = reach + 0.15 + speed * t_meet  # (its reach and its run to the meeting point)
            sgn = -1.0 if v % 2 == 0 else 1.0  # (the first on the axis' near side driving along it, the second facing it)
            ccx, ccz = cx + sgn * away * ux, cz + sgn * away * uz
            x0, z0 = ccx - 0.5 * sp * (nx - 1), ccz - 0.5 * sp * (nz - 1)
            vel = (-sgn * speed * ux, 0.0, -sgn * speed * uz)
        ix, iz = int((x0 + half) / cell), int((z0 + half) / cell)
        ground = float(h[min(max(iz, 0), terrain_samples - 1), min(max(ix, 0), terrain_samples - 1)])
        body = lattice_body_fast(gen, dims=(nx, ny, nz), origin=(x0, ground + 0.6, z0), velocity=vel)
        if skins:
            body["tris"] = lattice_tris((nx, ny, nz))
        if wheels:
            add_wheels(body, (nx, ny, nz))
        bodies.append(body)
    return {"settings": {"gravity": (0.0, -9.81, 0.0), "dt": 0.0005},
            "statics": {"terrain": terrain, "boxes": [], "build_grid": True}, "bodies": bodies,
            "name": f"fleet(n={n_vehicles}, seed={seed}, layout={layout})"}


def shell_plate(n: int = 63, size: float = 1.0, origin=(0.0, 1.0, 0.0), thickness: float = 0.0015, E: float = 210e9,
                nu: float = 0.3, rho: float = 7850.0, damping: float = 3e-4, drill: float = 0.05, clamp_edge: bool = True,
                load: float = 500.0, seed: int = 1, node_flags: int = 0, yield_stress: float = 0.0) -> dict:
    """The co-rotational FEM shell plate: (n + 1)^2 nodes on a size x size square in the horizontal plane at `origin`,
    2 n^2 CST/DKT triangles (two a cell, diagonals alternating: ShellMesher::grid, fem_shell.cpp:34-50), an elastic
    steel section (E, nu, rho, thickness), each triangle's mass a third on each corner; the edge z = origin.z clamped
    (anchored nodes); a seeded random point load of `load` N on a uniformly drawn free node; gravity. The default is
    the 64 x 64-node, 7,938-triangle plate of 1.5 mm steel. yield_stress > 0: a yielding section (the plate flows and
    folds; it does not tear: allow_break off)."""
    ox, oy, oz = (np.float32(v) for v in origin)
    du = np.float32(size / n)
    pos = np.zeros(((n + 1) * (n + 1), 3), np.float32)
    for j in range(n + 1):
        for i in range(n + 1):
            k = j * (n + 1) + i
            # origin + du * i + dv * j, in float (du along x, dv along z)
            x = np.float32(ox + np.float32(du * np.float32(i))) + np.float32(0.0)
            z = np.float32(oz + np.float32(0.0)) + np.float32(du * np.float32(j))
            pos[k] = (x, np.float32(np.float32(oy + np.float32(0.0)) + np.float32(0.0)), z)
    nn = len(pos)
    mass = np.zeros(nn, np.float32)
    tris = []
    tmass = []
    mpm2 = np.float32(np.float32(rho) * np.float32(thickness))

    def tri(a, b, c):
        pa, pb, pc = pos[a], pos[b], pos[c]
        e1, e2 = pb - pa, pc - pa
        cr = np.array([e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]], np.float32)
        area = np.float32(0.5) * np.sqrt(np.float32(cr[0] * cr[0] + cr[1] * cr[1]) + np.float32(cr[2] * cr[2]))
        m = np.float32(mpm2 * area)
        for v in (a, b, c):
            mass[v] = np.float32(mass[v] + np.float32(m / np.float32(3.0)))
        tris.append((a, b, c))
        tmass.append(m)

    for j in range(n):
        for i in range(n):
            n00, n10 = j * (n + 1) + i, j * (n + 1) + i + 1
            n01, n11 = (j + 1) * (n + 1) + i, (j + 1) * (n + 1) + i + 1
            if (i + j) & 1:
                tri(n00, n10, n11), tri(n00, n11, n01)
            else:
                tri(n00, n10, n01), tri(n10, n11, n01)
    flags = np.full(nn, node_flags, np.uint16)
    if clamp_edge:
        flags[: n + 1] |= NF_FIXED
    rng = np.random.default_rng(seed)
    free = np.nonzero((flags & NF_FIXED) == 0)[0]
    node = int(free[rng.integers(len(free))])
    d = rng.normal(size=3)
    f = (load * d / np.linalg.norm(d)).astype(np.float32)
    body = {
        "pos": pos, "vel": np.zeros((nn, 3), np.float32), "mass": mass, "node_flags": flags,
        "friction": np.ones(nn, np.float32), "radius": np.zeros(nn, np.float32),
        "ab": np.zeros((0, 2), np.uint32), "k": np.zeros(0, np.float32), "d": np.zeros(0, np.float32),
        "strength": np.zeros(0, np.float32), "deform": np.zeros(0, np.float32), "beam_type": np.zeros(0, np.uint8),
        "beam_flags": np.zeros(0, np.uint8),
        "params": {"ground_friction": 1.0, "bounce": -1.0, "contact_push_max": 2.0, "contact_slop": 0.0,
                   "collision_radius": 0.05, "allow_deform": 1, "allow_break": 0 if yield_stress > 0 else 1, "ductile": 0,
                   "can_sleep": 0, "sleep_speed": 0.0},
        "fem_sections": [{"E": E, "nu": nu, "rho": rho, "t": thickness, "yield": float(yield_stress), "damping": damping,
                          "drill": drill}],
        "fem_tris": np.asarray(tris, np.uint32), "fem_tri_mass": np.asarray(tmass, np.float32),
        "loads": [(node, tuple(float(x) for x in f))],
        "plate": {"n": n, "size": size, "origin": tuple(float(v) for v in origin)},
    }
    return {"settings": {"gravity": (0.0, -9.81, 0.0), "dt": 0.0005}, "statics": {}, "bodies": [body],
            "name": f"shell_plate(n={n}, seed={seed})"}


def tube_section(outer: float = 0.04, wall: float = 0.003, E: float = 2.1e11, G: float = 8.1e10, rho: float = 7850.0,
                 damping: float = 2e-5, yield_stress: float = 0.0, hardening: float = 0.25) -> dict:
    """A round steel tube's FrameSection fields (frame_fem.h:90-112): area, second moments, torsion constant,
    Timoshenko shear areas (half the area each way); yield_stress > 0: its plastic limits from the textbook formulas
    for a thin tube - Np = fy A, Mp = fy Zp with the plastic modulus Zp = (D^3 - d^3) / 6, Tp = (2 pi / 3) (fy /
    sqrt 3) (R^3 - r^3) - and the hinges' hardening."""
    ro, ri = outer / 2, outer / 2 - wall
    A = math.pi * (ro * ro - ri * ri)
    I = math.pi / 4 * (ro ** 4 - ri ** 4)
    s = {"E": E, "G": G, "rho": rho, "A": A, "Iy": I, "Iz": I, "J": 2 * I, "As_y": A / 2, "As_z": A / 2,
         "damping": damping, "axial": 1.0, "joint_k": 2.0e4}
    if yield_stress > 0:
        D, d = 2 * ro, 2 * ri
        s.update({"Np": yield_stress * A, "Mp": yield_stress * (D ** 3 - d ** 3) / 6,
                  "Tp": 2 * math.pi / 3 * (yield_stress / math.sqrt(3)) * (ro ** 3 - ri ** 3), "hardening": hardening})
    return s


def frame_ladder(rails: int = 12, spacing: float = 0.25, width: float = 0.6, origin=(0.0, 1.0, 0.0), load: float = 300.0,
                 joints=None, section: dict | None = None, ground: bool = False) -> dict:
    """A ladder frame of members (FemFrame::add_element): two rails of `rails` nodes along x, `spacing` apart, `width`
    apart in z, rungs between them at every node and a diagonal in each bay; the rails' first nodes clamped (anchored);
    a constant `load` N down (and a tenth of it across) at the far end of one rail, gravity. Each member's mass is its
    section's rho A L, half on each end node. joints: per rung, the joints at its ends (FJ_*; default rigid) - a few
    balls, hinges, swivels and elastic joints exercise the joints' end stiffnesses and the twist's weighting. ground:
    no anchors, every node NF_GROUND over flat grass (the ladder dropped onto the ground from `origin`)."""
    s = section or tube_section()
    ox, oy, oz = (np.float32(v) for v in origin)
    n = 2 * rails
    pos = np.zeros((n, 3), np.float32)
    for i in range(rails):
        for r in range(2):
            pos[2 * i + r] = (ox + np.float32(spacing * i), oy, oz + np.float32(width * r))
    members, ends = [], []
    for i in range(rails - 1):  # rails
        for r in range(2):
            members.append((2 * i + r, 2 * (i + 1) + r)), ends.append((0, 0))
    for i in range(rails):  # rungs
        members.append((2 * i, 2 * i + 1))
        ends.append(joints[i % len(joints)] if joints else (0, 0))
    for i in range(rails - 1):  # diagonals
        members.append((2 * i, 2 * (i + 1) + 1)), ends.append((0, 0))
    mpm = np.float32(np.float32(s["rho"]) * np.float32(s["A"]))
    mass = np.zeros(n, np.float32)
    for a, b in members:
        d = pos[b] - pos[a]
        m = np.float32(mpm * np.sqrt(np.float32(d[0] * d[0] + d[1] * d[1]) + np.float32(d[2] * d[2])))
        mass[a] += np.float32(m * np.float32(0.5))
        mass[b] += np.float32(m * np.float32(0.5))
    flags = np.zeros(n, np.uint16)
    if ground:
        flags |= NF_GROUND
    else:
        flags[0] |= NF_FIXED
        flags[1] |= NF_FIXED
    body = {
        "pos": pos, "vel": np.zeros((n, 3), np.float32), "mass": mass, "node_flags": flags,
        "friction": np.ones(n, np.float32), "radius": np.zeros(n, np.float32),
        "ab": np.zeros((0, 2), np.uint32), "k": np.zeros(0, np.float32), "d": np.zeros(0, np.float32),
        "strength": np.zeros(0, np.float32), "deform": np.zeros(0, np.float32), "beam_type": np.zeros(0, np.uint8),
        "beam_flags": np.zeros(0, np.uint8),
        "params": {"ground_friction": 1.0, "bounce": -1.0, "contact_push_max": 2.0, "contact_slop": 0.0,
                   "collision_radius": 0.05, "allow_deform": 1, "allow_break": 0 if s.get("Np", 0.0) > 0 else 1,
                   "ductile": 0, "can_sleep": 0, "sleep_speed": 0.0},
        "frame_sections": [s], "fem_members": np.asarray(members, np.uint32),
        "member_section": np.zeros(len(members), np.uint16), "member_ends": np.asarray(ends, np.uint8),
        "member_mass": np.zeros(len(members), np.float32),
        "loads": [(n - 2, (0.0, -float(load), 0.1 * float(load)))],
    }
    statics = {"terrain": flat_terrain(), "boxes": [], "build_grid": True} if ground else {}
    return {"settings": {"gravity": (0.0, -9.81, 0.0), "dt": 0.0005}, "statics": statics, "bodies": [body],
            "name": f"frame_ladder(rails={rails})"}


def plate_with_rails(n: int = 20, seed: int = 1, section: dict | None = None, tris_first: bool = True) -> dict:
    """shell_plate(n) stiffened by members: a rail of tubes along each of the two edges that run away from the clamped
    one, on the plate's own edge nodes (a frame of members and triangles; tris_first: the plate's add_tri calls before
    the rails' add_element calls). The rails' masses are added to their nodes."""
    rig = shell_plate(n, seed=seed)
    b = rig["bodies"][0]
    s = section or tube_section(0.02, 0.002)
    members = []
    for j in range(n):  # (nodes j * (n + 1) + i: the edges i = 0 and i = n, along z)
        members.append((j * (n + 1), (j + 1) * (n + 1)))
        members.append((j * (n + 1) + n, (j + 1) * (n + 1) + n))
    mpm = np.float32(np.float32(s["rho"]) * np.float32(s["A"]))
    pos, mass = b["pos"], b["mass"]
    for a, c in members:
        d = pos[c] - pos[a]
        m = np.float32(mpm * np.sqrt(np.float32(d[0] * d[0] + d[1] * d[1]) + np.float32(d[2] * d[2])))
        mass[a] += np.float32(m * np.float32(0.5))
        mass[c] += np.float32(m * np.float32(0.5))
    b.update({"frame_sections": [s], "fem_members": np.asarray(members, np.uint32),
              "member_section": np.zeros(len(members), np.uint16), "member_ends": np.zeros((len(members), 2), np.uint8),
              "member_mass": np.zeros(len(members), np.float32), "fem_tris_first": tris_first})
    rig["name"] = f"plate_with_rails(n={n}, seed={seed}, tris_first={tris_first})"
    return rig


def rod_section(d: float = 0.006, E: float = 2.1e11, G: float = 8.1e10, rho: float = 7850.0, damping: float = 2e-5) -> dict:
    """A solid round steel rod's FrameSection fields (a spot weld's nugget)."""
    r = d / 2
    A = math.pi * r * r
    I = math.pi * r ** 4 / 4
    return {"E": E, "G": G, "rho": rho, "A": A, "Iy": I, "Iz": I, "J": 2 * I, "As_y": 0.9 * A, "As_z": 0.9 * A,
            "damping": damping, "axial": 1.0, "joint_k": 2.0e4}


def shell_body(target_nodes: int = 50000, size=(4.0, 1.4, 1.8), seed: int = 1, t_range=(0.0008, 0.002), inset: float = 0.01,
               weld_every: int = 2, pillars: int = 2, load: float = 2000.0) -> dict:
    """A procedural box-and-pillar shell car body: the six faces of a size = (x, y, z) box, each a separate panel of
    CST/DKT triangles (a node grid split into two triangles a cell, diagonals alternating) of a seeded thickness in
    t_range, inset `inset` from the box's edges; spot welds - members of a 6 mm rod section - joining the facing edge
    nodes of adjacent panels every `weld_every` nodes (every 5 cm at the default spacing); tube pillars (members on the
    side panels' node columns) at `pillars` stations a side. Node spacing chosen for about target_nodes nodes; steel;
    floating (no ground, no clamp), gravity, a constant `load` N down on the roof's middle node and its seeded random
    push on a side panel node. Members are added first (their add_element calls), then the triangles."""
    Lx, Ly, Lz = size
    area = 2 * (Lx * Ly + Lx * Lz + Ly * Lz)
    du = math.sqrt(area / target_nodes)
    nx, ny, nz = (max(3, int(round((L - 2 * inset) / du)) + 1) for L in (Lx, Ly, Lz))
    gen = np.random.default_rng(seed)
    pos, panels = [], []

    def panel(origin, ua, va, nu, nv):
        # nodes origin + ua * i / (nu - 1) + va * j / (nv - 1): index base + j * nu + i
        base = len(pos)
        o, ua, va = np.asarray(origin, np.float64), np.asarray(ua, np.float64), np.asarray(va, np.float64)
        for j in range(nv):
            for i in range(nu):
                pos.append(o + ua * (i / (nu - 1)) + va * (j / (nv - 1)))
        panels.append((base, nu, nv))
        return base
    e, X, Y, Z = inset, Lx - 2 * inset, Ly - 2 * inset, Lz - 2 * inset
    # floor (y = 0) and roof (y = Ly): x by z; sides (z = 0, z = Lz): x by y; front and back (x = 0, x = Lx): z by y
    panel((e, 0.0, e), (X, 0, 0), (0, 0, Z), nx, nz)
    panel((e, Ly, e), (X, 0, 0), (0, 0, Z), nx, nz)
    panel((e, e, 0.0), (X, 0, 0), (0, Y, 0), nx, ny)
    panel((e, e, Lz), (X, 0, 0), (0, Y, 0), nx, ny)
    panel((0.0, e, e), (0, 0, Z), (0, Y, 0), nz, ny)
    panel((Lx, e, e), (0, 0, Z), (0, Y, 0), nz, ny)
    pos = np.asarray(pos, np.float32)
    n = len(pos)
    tris, tsec, sections = [], [], []
    for pi, (base, nu, nv) in enumerate(panels):
        t = float(gen.uniform(*t_range))
        sections.append({"E": 2.1e11, "nu": 0.3, "rho": 7850.0, "t": t, "yield": 0.0, "damping": 3e-4, "drill": 0.05})
        for j in range(nv - 1):
            for i in range(nu - 1):
                a, b, c, d = base + j * nu + i, base + j * nu + i + 1, base + (j + 1) * nu + i, base + (j + 1) * nu + i + 1
                if (i + j) & 1:
                    tris += [(a, b, d), (a, d, c)]
                else:
                    tris += [(a, b, c), (b, d, c)]
                tsec += [pi, pi]

    def edge(pnl, which):
        base, nu, nv = pnl
        if which == "j0":
            return [base + i for i in range(nu)]
        if which == "j1":
            return [base + (nv - 1) * nu + i for i in range(nu)]
        if which == "i0":
            return [base + j * nu for j in range(nv)]
        return [base + j * nu + nu - 1 for j in range(nv)]
    P = {k: panels[i] for i, k in enumerate(("fl", "rf", "s0", "s1", "f0", "f1"))}
    # spot welds along the twelve seams: (panel A's edge nodes, panel B's), every weld_every-th pair
    seams = [(("fl", "j0"), ("s0", "j0")), (("fl", "j1"), ("s1", "j0")), (("rf", "j0"), ("s0", "j1")), (("rf", "j1"), ("s1", "j1")),
             (("fl", "i0"), ("f0", "j0")), (("fl", "i1"), ("f1", "j0")), (("rf", "i0"), ("f0", "j1")), (("rf", "i1"), ("f1", "j1")),
             (("s0", "i0"), ("f0", "i0")), (("s0", "i1"), ("f1", "i0")), (("s1", "i0"), ("f0", "i1")), (("s1", "i1"), ("f1", "i1"))]
    members, msec = [], []
    for (pa, ea), (pb, eb) in seams:
        A, B = edge(P[pa], ea), edge(P[pb], eb)
        for q in range(0, min(len(A), len(B)), weld_every):
            members.append((A[q], B[q]))
            msec.append(1)
    # pillars: tube members up node columns of the side panels
    for side in ("s0", "s1"):
        base, nu, nv = P[side]
        for k in range(pillars):
            i = int(round((k + 1) * (nu - 1) / (pillars + 1)))
            for j in range(nv - 1):
                members.append((base + j * nu + i, base + (j + 1) * nu + i))
                msec.append(0)
    fsec = [tube_section(0.05, 0.002), rod_section(0.006)]
    # masses: each triangle a third of rho t area on each corner, each member half of rho A L on each end
    mass = np.zeros(n, np.float64)
    tri_a = np.asarray(tris, np.int64)
    pa_, pb_, pc_ = (pos[tri_a[:, c]].astype(np.float64) for c in range(3))
    ar = 0.5 * np.linalg.norm(np.cross(pb_ - pa_, pc_ - pa_), axis=1)
    tth = np.asarray([sections[s]["t"] for s in tsec])
    tm = (7850.0 * tth * ar).astype(np.float32)
    for c in range(3):
        np.add.at(mass, tri_a[:, c], tm.astype(np.float64) / 3)
    mab = np.asarray(members, np.int64)
    ml = np.linalg.norm(pos[mab[:, 1]].astype(np.float64) - pos[mab[:, 0]], axis=1)
    mm = np.asarray([fsec[s]["rho"] * fsec[s]["A"] for s in msec]) * ml
    np.add.at(mass, mab[:, 0], mm / 2)
    np.add.at(mass, mab[:, 1], mm / 2)
    body = {
        "pos": pos, "vel": np.zeros((n, 3), np.float32), "mass": mass.astype(np.float32), "node_flags": np.zeros(n, np.uint16),
        "friction": np.ones(n, np.float32), "radius": np.zeros(n, np.float32),
        "ab": np.zeros((0, 2), np.uint32), "k": np.zeros(0, np.float32), "d": np.zeros(0, np.float32),
        "strength": np.zeros(0, np.float32), "deform": np.zeros(0, np.float32), "beam_type": np.zeros(0, np.uint8),
        "beam_flags": np.zeros(0, np.uint8),
        "params": {"ground_friction": 1.0, "bounce": -1.0, "contact_push_max": 2.0, "contact_slop": 0.0,
                   "collision_radius": 0.05, "allow_deform": 1, "allow_break": 1, "ductile": 0, "can_sleep": 0,
                   "sleep_speed": 0.0},
        "fem_sections": sections, "fem_tris": np.asarray(tris, np.uint32), "fem_tri_section": np.asarray(tsec, np.uint16),
        "fem_tri_mass": tm, "frame_sections": fsec, "fem_members": np.asarray(members, np.uint32),
        "member_section": np.asarray(msec, np.uint16), "member_ends": np.zeros((len(members), 2), np.uint8),
        "member_mass": np.zeros(len(members), np.float32),
        "loads": [(P["rf"][0] + (nz // 2) * nx + nx // 2, (0.0, -float(load), 0.0)),
                  (P["s0"][0] + int(gen.integers(nx * ny)), tuple(float(v) for v in gen.normal(0.0, 0.5 * load, 3)))],
    }
    return {"settings": {"gravity": (0.0, -9.81, 0.0), "dt": 0.0005}, "statics": {}, "bodies": [body],
            "name": f"shell_body(target={target_nodes}, seed={seed})"}
