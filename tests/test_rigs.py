"""The seeded rig generators (beamlab_b200.rigs): shapes, determinism, the truss car's beam count."""
import numpy as np

from beamlab_b200 import rigs


def test_trng_is_xorshift32():
    r = rigs.TRng(1)
    s = (1 * 2654435761 + 1) & 0xFFFFFFFF
    s ^= (s << 13) & 0xFFFFFFFF
    s ^= s >> 17
    s ^= (s << 5) & 0xFFFFFFFF
    assert r.next() == s
    u = [float(r.uni()) for _ in range(2000)]
    assert 0.0 <= min(u) and max(u) < 1.0 and abs(np.mean(u) - 0.5) < 0.03


def test_truss_car_shape():
    rig = rigs.truss_car(1)
    n, m = rigs.rig_counts(rig)
    assert n == 400
    assert 3000 <= m <= 3300  # pairs within sqrt(3) * 0.25 m of the jittered lattice
    b = rig["bodies"][0]
    assert b["mass"].min() >= 4.0 and b["mass"].max() <= 6.0
    k = b["k"].astype(np.float64)
    assert 1.7e6 < np.median(k) < 2.3e6 and 0.25 < np.std(np.log(k)) < 0.35
    d = b["pos"][b["ab"][:, 0]] - b["pos"][b["ab"][:, 1]]
    assert np.sqrt((d.astype(np.float64) ** 2).sum(1)).max() <= np.sqrt(3) * 0.25 + 1e-6


def test_rigs_are_deterministic():
    a, b = rigs.truss_car(5), rigs.truss_car(5)
    for k in ("pos", "mass", "k", "ab"):
        assert np.array_equal(a["bodies"][0][k], b["bodies"][0][k])
    c = rigs.truss_car(6)
    assert not np.array_equal(a["bodies"][0]["pos"], c["bodies"][0]["pos"])


def test_fleet_sizes():
    rig = rigs.fleet(32, seed=3, terrain_samples=257, terrain_size=400.0)
    sizes = np.asarray([len(b["mass"]) for b in rig["bodies"]])
    assert len(sizes) == 32
    assert sizes.min() >= 200 and sizes.max() <= 26000
    assert 1000 < np.median(sizes) < 8000
    t = rig["statics"]["terrain"]
    assert t["heights"].shape == (257, 257) and np.abs(t["heights"]).max() <= 2.6


def test_lattice_skin_faces_outward():
    """lattice_tris: 2 triangles per face quad, every normal pointing away from the lattice's centre."""
    dims = (5, 3, 4)
    tris = rigs.lattice_tris(dims)
    nx, ny, nz = dims
    assert len(tris) == 4 * ((nx - 1) * (ny - 1) + (nx - 1) * (nz - 1) + (ny - 1) * (nz - 1))
    rig = rigs.crash_pair(1, dims=dims)
    p = rig["bodies"][0]["pos"].astype(np.float64)
    c = p.mean(0)
    a, b, d = p[tris[:, 0]], p[tris[:, 1]], p[tris[:, 2]]
    n = np.cross(b - a, d - a)
    assert np.all(np.einsum("ij,ij->i", n, (a + b + d) / 3 - c) > 0)


def test_wheel_rings():
    """add_wheels: four wheels of 24 tyre nodes (even on axle0's side, odd on axle1's, at the radius round the hubs),
    axle0 of the lesser z, every tyre node NF_GROUND | NF_TYRE and beamed to both hubs."""
    rig = rigs.wheeled_car()
    b = rig["bodies"][0]
    p = b["pos"].astype(np.float64)
    pairs = {tuple(sorted(e)) for e in b["ab"].tolist()}
    assert len(b["wheels"]) == 4
    for w in b["wheels"]:
        a0, a1, nodes = w["axle0"], w["axle1"], w["nodes"]
        assert len(nodes) == 24 and p[a0, 2] < p[a1, 2]
        ev, od = nodes[0::2], nodes[1::2]
        assert np.allclose(p[ev, 2], p[a0, 2]) and np.allclose(p[od, 2], p[a1, 2])
        assert np.allclose(np.linalg.norm(p[ev, :2] - p[a0, :2], axis=1), 0.3, atol=1e-5)
        assert np.all(b["node_flags"][nodes] & (rigs.NF_GROUND | rigs.NF_TYRE) == rigs.NF_GROUND | rigs.NF_TYRE)
        for t in nodes.tolist():
            assert tuple(sorted((t, a0))) in pairs and tuple(sorted((t, a1))) in pairs
    every = np.concatenate([w["nodes"] for w in b["wheels"]])
    assert len(np.unique(every)) == len(every)
