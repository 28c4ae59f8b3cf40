"""Shared helpers of the test suite: golden fixtures and comparisons."""
from __future__ import annotations

import gzip
import os
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
CASES = ["square_drop_skip", "bridge", "moving_walls", "droplet_2d", "dam_break_small", "two_fluid_small"]
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
