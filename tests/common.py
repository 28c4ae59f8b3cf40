"""Shared helpers of the test suite: golden fixtures and comparisons."""
from __future__ import annotations

import gzip
import os
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
CASES = ["square_drop_skip", "bridge", "moving_walls", "droplet_2d", "dam_break_small", "two_fluid_small"]
# 3-D cases over 1000 steps from inputs inside the developed flow; their
# neighbour lists are kept as SHA-256 digests (nptr_sha256, nind_sha256)
LONG_CASES = ["dam_break_1000", "two_fluid_1000"]
STATE_KEYS = ["particle_index", "type", "xyz", "vel", "force", "neighbor_count", "density_a", "vol_strain_p",
              "virial_pressure"]
FIELD_KEYS = ["divergence_p", "pressure_p", "pressure_a", "gravity_center"]
CELL_KEYS = ["cell_index", "fluid_begin", "fluid_end", "wall_begin", "wall_end"]


def has_cuda() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


class GoldenCase:
    """A *.data/*.grid pair and the reference's arrays after `steps` steps."""

    def __init__(self, name: str):
        self.name = name
        self.dir = os.path.join(GOLDEN, name)
        self.data = os.path.join(self.dir, "case.data")
        self._tmp = tempfile.TemporaryDirectory()
        self.grid = os.path.join(self._tmp.name, "case.grid")
        with gzip.open(os.path.join(self.dir, "case.grid.gz"), "rb") as g, open(self.grid, "wb") as f:
            f.write(g.read())
        z = np.load(os.path.join(self.dir, "reference.npz"))
        self.ref = {k: z[k] for k in z.files}
        meta = self.ref["meta"]
        self.dim, self.steps, self.rebuilds = int(meta[0]), int(meta[1]), int(meta[2])
        self.neighbor_ind_count, self.total_cell_count = int(meta[3]), int(meta[4])
        self.cell_count = [int(v) for v in meta[5:8]]

    def reference_bytes(self, what: str) -> bytes | None:
        p = os.path.join(self.dir, "reference.%s.gz" % what)
        if not os.path.exists(p):
            return None
        with gzip.open(p, "rb") as g:
            return g.read()


def csr_digests(ptr, ind) -> tuple[str, str]:
    """SHA-256 of NeighborPtr (int64) and NeighborInd (int32) as the reference
    stores them."""
    import hashlib
    return (hashlib.sha256(np.ascontiguousarray(ptr, np.int64).tobytes()).hexdigest(),
            hashlib.sha256(np.ascontiguousarray(ind, np.int32).tobytes()).hexdigest())


def assert_same(a, b, what=""):
    a = np.asarray(a)
    b = np.asarray(b)
    assert a.shape == b.shape, f"{what}: shape {a.shape} vs {b.shape}"
    if a.dtype.kind == "f":
        same = np.array_equal(a.view(np.int64), b.view(np.int64)) or np.array_equal(a, b)
        if not same:
            d = np.abs(a - b)
            raise AssertionError(f"{what}: not bit-identical, max |diff| {np.nanmax(d):.3e} at {np.nanargmax(d)}")
    else:
        if not np.array_equal(a, b):
            bad = np.flatnonzero(a.ravel() != b.ravel())
            raise AssertionError(f"{what}: {len(bad)} entries differ, first at {bad[:5]}")


def by_original_id(state: dict, key: str) -> np.ndarray:
    """Reorder a sorted-order array by ParticleIndex (file order)."""
    order = np.argsort(state["particle_index"], kind="stable")
    return np.asarray(state[key])[order]


def rel_l2(a, b) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / den) if den > 0 else float(np.linalg.norm(a - b))


def micro_cases():
    """Small hand-built scenes that single out one behaviour each (the
    reference has no tests; these follow its code paths): pairs at every
    kernel radius, a lone particle, a wall with no fluid in reach
    (main.cpp:1416), interaction and motion across every periodic face, and a
    2-D grid with a nonzero z extent.  Yields (name, scene, steps)."""
    from mphexplicit_b200 import make_header, scenes
    from mphexplicit_b200.scenes import Scene

    def params(dim, sigma=0.05, gravity=(0.0, 0.0, 0.0)):
        return scenes.make_params(dt=1e-5, density=1000.0, bulk_modulus=1.0e5, bulk_viscosity=0.2,
                                  shear_viscosity=0.1, surface_tension=sigma, gravity=gravity)

    l0 = 0.01

    def scene(name, dim, typ, xyz, vel, box, sigma=0.05, gravity=(0.0, 0.0, 0.0), lo=None):
        xyz = np.asarray(xyz, float) * l0
        vel = np.asarray(vel, float)
        lo = lo if lo is not None else [0.0, 0.0, -0.5 * l0 if dim == 2 else 0.0]
        hi = [lo[0] + box[0] * l0, lo[1] + box[1] * l0, (lo[2] + box[2] * l0) if dim == 3 or len(box) > 2
              else 0.5 * l0]
        h = make_header(len(xyz), l0, lo, hi)
        return Scene(name, dim, params(dim, sigma, gravity), h, np.asarray(typ, np.int32), xyz, vel, 40)

    # pairs of fluid particles at r inside RP (1.7), between RP and RA (3.5), and
    # beyond RA but inside the list radius (3.6): every kernel shape and both cut-off tests
    for dim in (2, 3):
        z = 0.0 if dim == 2 else 10.0
        xyz = [[10.0, 10.0, z], [11.0, 10.0, z], [10.0, 12.5, z], [13.55, 10.0, z]]
        vel = [[0.01, 0.0, 0.0], [-0.02, 0.01, 0.0], [0.0, -0.01, 0.0], [0.0, 0.0, 0.0]]
        yield ("pairs_%dd" % dim, scene("pairs_%dd" % dim, dim, [0, 0, 0, 0], xyz, vel,
                                        (20.0, 20.0, 20.0) if dim == 3 else (20.0, 20.0))), 40
    # one particle, no neighbour, under gravity
    yield ("lone_3d", scene("lone_3d", 3, [0], [[5.0, 5.0, 5.0]], [[0.1, -0.05, 0.02]], (12.0, 12.0, 12.0),
                            gravity=(0.0, 0.0, -9.81))), 40
    # fluid pair plus a wall particle out of every fluid particle's reach, and
    # one wall within reach
    xyz = [[5.0, 5.0, 5.0], [6.0, 5.0, 5.0], [15.0, 15.0, 15.0], [5.5, 7.0, 5.0]]
    yield ("isolated_wall_3d", scene("isolated_wall_3d", 3, [0, 1, 2, 3], xyz, [[0.0] * 3] * 4,
                                     (20.0, 20.0, 20.0))), 40
    # a cluster around the domain corner (its pairs interact across all three
    # periodic faces) and three lone particles that cross the x, y and z faces
    pts, vs = [], []
    for dx in (-0.6, 0.6):
        for dy in (-0.6, 0.6):
            for dz in (-0.6, 0.6):
                pts.append([(dx % 11.0), (dy % 11.0), (dz % 11.0)])
                vs.append([0.3 * np.sign(dx), -0.2 * np.sign(dy), 0.25 * np.sign(dz)])
    pts += [[0.15, 5.0, 5.0], [5.0, 10.85, 5.5], [5.5, 5.5, 0.1]]
    vs += [[-5.0, 0.0, 0.0], [0.0, 5.0, 0.0], [0.0, 0.0, -5.0]]
    yield ("wrap_faces_3d", scene("wrap_faces_3d", 3, [0] * 11, pts, vs, (11.0, 11.0, 11.0), sigma=0.0)), 60
    # 2-D with a z extent of several l0 and particles off z = 0
    xyz = [[4.0, 4.0, 0.7], [5.0, 4.2, 0.7], [4.6, 5.1, 0.7], [7.2, 4.0, 0.7]]
    yield ("thin_2d", scene("thin_2d", 2, [0, 0, 1, 0], xyz, [[0.01, 0.0, 0.0]] * 4, (12.0, 12.0, 5.0),
                            lo=[0.0, 0.0, -2.0 * l0])), 40
