"""Seeded synthetic scenes in the reference's formats (*.data + *.grid).

The reference ships only two 2-D sample inputs and a cuboid generator
(generator/generator.cpp:170-217); the benchmark scenes are generated here
from a seed:

* ``droplet_2d``        40x40 square droplet, periodic, surface tension
* ``dam_break_3d``      fluid block in the corner of a closed box of type-2
                        walls, gravity in -z (2.0 M fluid at full size)
* ``two_fluid_column``  two fluid types (rho 500 / 1000) with a perturbed
                        interface inside type-2/3 walls
* ``droplet_batch_2d``  many uneven 2-D rectangles with random mu / sigma
* ``cuboid_grid``       the reference generator's cuboid lattice

Positions of fluid particles carry a uniform jitter of +-0.01 l0.  The domain is
periodic in every direction (the reference applies Mod on every axis), so
each scene pads the domain so that no pair interacts across it.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import _native as N
from .solver import make_header, write_grid_file


@dataclass
class Scene:
    name: str
    dim: int
    params: N.Params
    header: N.GridHeader
    type: np.ndarray
    xyz: np.ndarray
    vel: np.ndarray
    steps: int
    meta: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return int(self.header.particle_count)

    @property
    def n_fluid(self) -> int:
        return int(np.count_nonzero(self.type < 2))

    def write(self, data_path: str, grid_path: str) -> None:
        write_data_file(data_path, self.params)
        write_grid_file(grid_path, self.header, self.type, self.xyz, self.vel)


def make_params(*, dt, density, bulk_modulus, bulk_viscosity, shear_viscosity, surface_tension,
                gravity=(0.0, 0.0, 0.0), ra=3.5, rp=1.7, rv=3.5, end_time=None, steps=1000,
                output_interval=None, vtk_output_interval=None) -> N.Params:
    p = N.Params()
    p.dt = dt
    p.end_time = end_time if end_time is not None else dt * (steps - 0.5)
    big = 1.0e30
    p.output_interval = output_interval if output_interval is not None else big
    p.vtk_output_interval = vtk_output_interval if vtk_output_interval is not None else big
    p.radius_ratio_a, p.radius_ratio_p, p.radius_ratio_v = ra, rp, rv

    def four(v):
        return list(v) if hasattr(v, "__len__") else [v] * 4

    for name, val in (("density", density), ("bulk_modulus", bulk_modulus), ("bulk_viscosity", bulk_viscosity),
                      ("shear_viscosity", shear_viscosity), ("surface_tension", surface_tension)):
        arr = getattr(p, name)
        for t, x in enumerate(four(val)):
            arr[t] = float(x)
    for a in range(4):
        for b in range(4):
            p.interaction_ratio[a][b] = 1.0
    for d in range(3):
        p.gravity[d] = float(gravity[d])
    return p


def write_data_file(path: str, p: N.Params) -> None:
    """A *.data file the reference's readDataFile (main.cpp:502-521) parses."""
    g = lambda x: "%.17g" % x  # noqa: E731  (round-trips every double)
    four = lambda a: "  ".join(g(a[t]) for t in range(4))  # noqa: E731
    lines = [
        "#######",
        "Dt                      " + g(p.dt),
        "OutputInterval          " + g(p.output_interval),
        "VtkOutputInterval       " + g(p.vtk_output_interval),
        "EndTime                 " + g(p.end_time),
        "RadiusRatioA            " + g(p.radius_ratio_a),
        "RadiusRatioP            " + g(p.radius_ratio_p),
        "RadiusRatioV            " + g(p.radius_ratio_v),
        "Density                 " + four(p.density),
        "BulkModulus             " + four(p.bulk_modulus),
        "BulkViscosity           " + four(p.bulk_viscosity),
        "ShearViscosity          " + four(p.shear_viscosity),
        "SurfaceTension          " + four(p.surface_tension),
    ]
    for t in range(4):
        lines.append("InteractionRatio(Type%d) " % t + four(p.interaction_ratio[t]))
    lines.append("Gravity                 " + " ".join(g(p.gravity[d]) for d in range(3)))
    for t in (2, 3):
        lines.append("Wall%d    Center %s    Velocity %s    Omega %s" % (
            t, " ".join(g(p.wall_center[t][d]) for d in range(3)),
            " ".join(g(p.wall_velocity[t][d]) for d in range(3)),
            " ".join(g(p.wall_omega[t][d]) for d in range(3))))
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def _pad_for_cells(extent_l0: float, min_pad: float, cutoff_l0: float = 3.6) -> float:
    """Padding (in l0, each side) >= min_pad that keeps extent/cut-off away from
    an integer, so the cell width stays clear of MaxRadius+MARGIN."""
    pad = min_pad
    while True:
        q = (extent_l0 + 2 * pad) / cutoff_l0
        if 0.05 < q - math.floor(q) < 0.95:
            return pad
        pad += 0.25


def _lattice(counts, l0, origin=(0.0, 0.0, 0.0)):
    axes = [(np.arange(c) + 0.5) * l0 + o for c, o in zip(counts, origin)]
    g = np.meshgrid(*axes, indexing="ij")
    return np.stack([a.ravel() for a in g], axis=1)


def droplet_2d(n: int = 40, l0: float = 0.004, seed: int = 0, box: float = 100.0, steps: int = 1000,
               rho=1000.0, mu=0.1, sigma=0.07, c_sound=10.0, dt=1.0e-5) -> Scene:
    """Square droplet (n x n type-0), no walls, no gravity (benchmark config 1)."""
    rng = np.random.default_rng(seed)
    xy = _lattice((n, n), l0, (-0.5 * n * l0, -0.5 * n * l0))
    xy += rng.uniform(-0.01 * l0, 0.01 * l0, xy.shape)
    xyz = np.zeros((len(xy), 3))
    xyz[:, :2] = xy
    half = 0.5 * (box + 2 * _pad_for_cells(box, 0.0) - box) + 0.5 * box
    p = make_params(dt=dt, density=rho, bulk_modulus=rho * c_sound ** 2, bulk_viscosity=mu, shear_viscosity=mu,
                    surface_tension=sigma, steps=steps)
    h = make_header(len(xyz), l0, (-half * l0, -half * l0, -0.5 * l0), (half * l0, half * l0, 0.5 * l0))
    return Scene("droplet_2d", 2, p, h, np.zeros(len(xyz), np.int32), xyz, np.zeros_like(xyz), steps,
                 {"seed": seed, "n": n, "l0": l0})


def dam_break_3d(fluid=(100, 100, 200), box=(300, 100, 240), l0: float = 0.005, walls: int = 3, seed: int = 0,
                 steps: int = 1000, rho=1000.0, mu=1.0e-3, c_sound=20.0, dt=2.0e-5, lid: bool = True) -> Scene:
    """Dam break (benchmark config 2): a fluid block of type 0 in the corner of
    a box of `box` cells, closed by `walls` layers of type-2 particles."""
    rng = np.random.default_rng(seed)
    f = _lattice(fluid, l0)
    f += rng.uniform(-0.01 * l0, 0.01 * l0, f.shape)
    outer = [b + 2 * walls for b in box]
    w = _lattice(outer, l0, tuple(-walls * l0 for _ in range(3)))
    inside = np.ones(len(w), bool)
    for d in range(3):
        lo_ok = w[:, d] > 0.0
        hi_ok = w[:, d] < box[d] * l0 if (lid or d != 2) else np.ones(len(w), bool)
        inside &= lo_ok & hi_ok
    w = w[~inside]
    xyz = np.concatenate([f, w])
    typ = np.concatenate([np.zeros(len(f), np.int32), np.full(len(w), 2, np.int32)])
    dmin, dmax = [], []
    for d in range(3):
        ext = box[d] + 2 * walls
        pad = _pad_for_cells(ext, 2.0)
        dmin.append(-(walls + pad) * l0)
        dmax.append((box[d] + walls + pad) * l0)
    p = make_params(dt=dt, density=rho, bulk_modulus=rho * c_sound ** 2, bulk_viscosity=mu, shear_viscosity=mu,
                    surface_tension=0.0, gravity=(0.0, 0.0, -9.81), steps=steps)
    h = make_header(len(xyz), l0, dmin, dmax)
    return Scene("dam_break_3d", 3, p, h, typ, xyz, np.zeros_like(xyz), steps,
                 {"seed": seed, "fluid": tuple(fluid), "box": tuple(box), "walls": walls, "l0": l0})


def two_fluid_column(n: int = 200, l0: float = 0.0025, walls: int = 2, seed: int = 0, steps: int = 500,
                     mu=0.01, sigma=0.05, c_sound=20.0, dt=1.0e-5, modes: int = 4) -> Scene:
    """Two-fluid column (benchmark config 3): n^3 fluid, lower half type 0
    (rho 500), upper half type 1 (rho 1000), interface displaced by a seeded sum
    of cosine modes of amplitude 2 l0; walls alternate types 2/3 by layer."""
    rng = np.random.default_rng(seed)
    f = _lattice((n, n, n), l0)
    L = n * l0
    kx = rng.integers(1, 5, modes)
    ky = rng.integers(1, 5, modes)
    ph = rng.uniform(0, 2 * np.pi, (modes, 2))
    amp = 2.0 * l0 / modes
    z0 = 0.5 * L + sum(amp * np.cos(2 * np.pi * kx[m] * f[:, 0] / L + ph[m, 0]) *
                       np.cos(2 * np.pi * ky[m] * f[:, 1] / L + ph[m, 1]) for m in range(modes))
    ftype = np.where(f[:, 2] > z0, 1, 0).astype(np.int32)
    f += rng.uniform(-0.01 * l0, 0.01 * l0, f.shape)
    outer = n + 2 * walls
    w = _lattice((outer,) * 3, l0, (-walls * l0,) * 3)
    layer = np.max(np.stack([np.maximum(-w[:, d] / l0, w[:, d] / l0 - n) for d in range(3)]), axis=0)
    keep = layer > 0
    w = w[keep]
    wtype = np.where(np.ceil(layer[keep]).astype(int) % 2 == 1, 2, 3).astype(np.int32)
    xyz = np.concatenate([f, w])
    typ = np.concatenate([ftype, wtype])
    pad = _pad_for_cells(outer, 2.0)
    dmin = [-(walls + pad) * l0] * 3
    dmax = [(n + walls + pad) * l0] * 3
    rho = [500.0, 1000.0, 1000.0, 1000.0]
    p = make_params(dt=dt, density=rho, bulk_modulus=[r * c_sound ** 2 for r in rho], bulk_viscosity=mu,
                    shear_viscosity=mu, surface_tension=sigma, gravity=(0.0, 0.0, -9.81), steps=steps)
    h = make_header(len(xyz), l0, dmin, dmax)
    return Scene("two_fluid_column", 3, p, h, typ, xyz, np.zeros_like(xyz), steps,
                 {"seed": seed, "n": n, "walls": walls, "l0": l0})


def droplet_batch_2d(count: int = 256, seed: int = 0, l0: float = 1.0e-3, lo: int = 20, hi: int = 140,
                     steps: int = 2000, dt: float = 5.0e-6, c_sound: float = 10.0) -> list[Scene]:
    """Uneven 2-D droplets (benchmark config 4): width/height ~ U[lo, hi]
    particles, mu log-uniform in [1e-3, 1], sigma uniform in [0.02, 0.08]."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        wdt, hgt = (int(v) for v in rng.integers(lo, hi + 1, 2))
        mu = float(10 ** rng.uniform(-3, 0))
        sigma = float(rng.uniform(0.02, 0.08))
        xy = _lattice((wdt, hgt), l0, (-0.5 * wdt * l0, -0.5 * hgt * l0))
        xy += rng.uniform(-0.01 * l0, 0.01 * l0, xy.shape)
        xyz = np.zeros((len(xy), 3))
        xyz[:, :2] = xy
        ex = max(wdt, hgt) + 40.0
        pad = _pad_for_cells(ex, 0.0)
        half = 0.5 * ex + pad
        p = make_params(dt=dt, density=1000.0, bulk_modulus=1000.0 * c_sound ** 2, bulk_viscosity=mu,
                        shear_viscosity=mu, surface_tension=sigma, steps=steps)
        h = make_header(len(xyz), l0, (-half * l0, -half * l0, -0.5 * l0), (half * l0, half * l0, 0.5 * l0))
        out.append(Scene("droplet_batch_2d[%d]" % k, 2, p, h, np.zeros(len(xyz), np.int32), xyz,
                         np.zeros_like(xyz), steps, {"seed": seed, "index": k, "w": wdt, "h": hgt, "mu": mu,
                                                     "sigma": sigma}))
    return out


def cuboid_grid(cuboids, spacing_domain, lower, upper):
    """The reference generator's lattice fill (generator/generator.cpp:170-193)
    through the library's generator (mph_generate_cuboids): for each cuboid
    (spacing, type, lower, upper, velocity), count = round(width/spacing) per
    axis with C rounding (halves away from zero), spacing = width/count,
    particles from lower + spacing/2 while below upper - 0.49 spacing.
    Returns (header, type, xyz, vel)."""
    from .solver import generate_cuboids
    cs = []
    for (sp, typ, lo, up, v) in cuboids:
        c = N.Cuboid()
        c.spacing, c.type = float(sp), int(typ)
        for d in range(3):
            c.lower[d], c.upper[d], c.velocity[d] = float(lo[d]), float(up[d]), float(v[d])
        cs.append(c)
    t, x, vel = generate_cuboids(cs)
    return make_header(len(t), spacing_domain, lower, upper), t, x, vel
