"""Inputs and timing for the reference's own executable.  TEST INFRASTRUCTURE ONLY.

Used by bench.py's CPU legs (the `cpu_baseline` of the main line and the
`--impl reference` arm) and by tests/.  Pure numpy + subprocess: nothing here
imports the product package or loads its library, so the process that times
the reference runs the reference's code and nothing of the product.

* ``dam_break_arrays``: the seeded 3-D dam-break scene (fluid block of type 0 in
  the corner of a box closed by type-2 wall layers), the same arrays as the
  product's scene generator (a CPU test compares them element for element);
  ``droplet_arrays`` and ``two_fluid_arrays``: the 2-D square droplet and the
  two-fluid column, likewise.
* ``write_data`` / ``write_grid``: the reference's *.data keys (readDataFile,
  source/main.cpp:502-521) and *.grid layout (readGridFile, main.cpp:541-640;
  the generator's writer, generator/generator.cpp:197-217).
* ``time_reference``: wall clock of the reference's step loop through
  oracle/_ref/ref_mph{2,3}d `time` (oracle/ref_harness.cpp).
* ``host_cores``: logical CPUs this process may use and the physical cores
  behind them.
"""
from __future__ import annotations

import json
import math
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")


def ref_available(dim: int) -> bool:
    return os.path.exists(os.path.join(REF_DIR, "ref_mph%dd" % dim))


def _pad_for_cells(extent_l0: float, min_pad: float, cutoff_l0: float = 3.6) -> float:
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


def dam_break_arrays(fluid=(100, 100, 200), box=(300, 100, 240), l0=0.005, walls=3, seed=0, steps=1000,
                     rho=1000.0, mu=1.0e-3, c_sound=20.0, dt=2.0e-5):
    """(params dict, header dict, type, xyz, vel) of the dam break: fluid on a
    lattice with a seeded uniform +-0.01 l0 jitter, `walls` closed layers of
    type-2 particles, domain padded so no pair interacts across the periodic
    boundary; K = rho c^2, lambda = mu, gravity -9.81 z, radii 3.5/1.7/3.5 l0."""
    rng = np.random.default_rng(seed)
    f = _lattice(fluid, l0)
    f += rng.uniform(-0.01 * l0, 0.01 * l0, f.shape)
    outer = [b + 2 * walls for b in box]
    w = _lattice(outer, l0, tuple(-walls * l0 for _ in range(3)))
    inside = np.ones(len(w), bool)
    for d in range(3):
        inside &= (w[:, d] > 0.0) & (w[:, d] < box[d] * l0)
    w = w[~inside]
    xyz = np.concatenate([f, w])
    typ = np.concatenate([np.zeros(len(f), np.int32), np.full(len(w), 2, np.int32)])
    dmin, dmax = [], []
    for d in range(3):
        pad = _pad_for_cells(box[d] + 2 * walls, 2.0)
        dmin.append(-(walls + pad) * l0)
        dmax.append((box[d] + walls + pad) * l0)
    four = lambda v: [float(v)] * 4  # noqa: E731
    params = {"dt": dt, "output_interval": 1.0e30, "vtk_output_interval": 1.0e30, "end_time": dt * (steps - 0.5),
              "radius_ratio_a": 3.5, "radius_ratio_p": 1.7, "radius_ratio_v": 3.5, "density": four(rho),
              "bulk_modulus": four(rho * c_sound ** 2), "bulk_viscosity": four(mu), "shear_viscosity": four(mu),
              "surface_tension": four(0.0), "interaction_ratio": [[1.0] * 4 for _ in range(4)],
              "gravity": [0.0, 0.0, -9.81], "wall_center": [[0.0] * 3 for _ in range(4)],
              "wall_velocity": [[0.0] * 3 for _ in range(4)], "wall_omega": [[0.0] * 3 for _ in range(4)]}
    header = {"time": 0.0, "n": len(xyz), "l0": l0, "dmin": dmin, "dmax": dmax}
    return params, header, typ, xyz, np.zeros_like(xyz)


def droplet_arrays(n=40, l0=0.004, seed=0, box=100.0, steps=1000, rho=1000.0, mu=0.1, sigma=0.07, c_sound=10.0,
                   dt=1.0e-5):
    """(params dict, header dict, type, xyz, vel) of the 2-D square droplet:
    n x n type-0 particles on a lattice with a seeded uniform +-0.01 l0 jitter,
    no walls, no gravity, surface tension sigma; the domain `box` cells wide,
    padded so no pair interacts across the periodic boundary."""
    rng = np.random.default_rng(seed)
    xy = _lattice((n, n), l0, (-0.5 * n * l0, -0.5 * n * l0))
    xy += rng.uniform(-0.01 * l0, 0.01 * l0, xy.shape)
    xyz = np.zeros((len(xy), 3))
    xyz[:, :2] = xy
    half = 0.5 * (box + 2 * _pad_for_cells(box, 0.0) - box) + 0.5 * box
    four = lambda v: [float(v)] * 4  # noqa: E731
    params = {"dt": dt, "output_interval": 1.0e30, "vtk_output_interval": 1.0e30, "end_time": dt * (steps - 0.5),
              "radius_ratio_a": 3.5, "radius_ratio_p": 1.7, "radius_ratio_v": 3.5, "density": four(rho),
              "bulk_modulus": four(rho * c_sound ** 2), "bulk_viscosity": four(mu), "shear_viscosity": four(mu),
              "surface_tension": four(sigma), "interaction_ratio": [[1.0] * 4 for _ in range(4)],
              "gravity": [0.0, 0.0, 0.0], "wall_center": [[0.0] * 3 for _ in range(4)],
              "wall_velocity": [[0.0] * 3 for _ in range(4)], "wall_omega": [[0.0] * 3 for _ in range(4)]}
    header = {"time": 0.0, "n": len(xyz), "l0": l0, "dmin": [-half * l0, -half * l0, -0.5 * l0],
              "dmax": [half * l0, half * l0, 0.5 * l0]}
    return params, header, np.zeros(len(xyz), np.int32), xyz, np.zeros_like(xyz)


def two_fluid_arrays(n=200, l0=0.0025, walls=2, seed=0, steps=500, mu=0.01, sigma=0.05, c_sound=20.0, dt=1.0e-5,
                     modes=4):
    """(params dict, header dict, type, xyz, vel) of the two-fluid column: n^3
    fluid, type 1 above an interface displaced by a seeded sum of cosine modes
    of amplitude 2 l0 and type 0 below, densities 500 / 1000, closed walls
    whose layers alternate types 2 and 3, gravity -9.81 z, surface tension."""
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
    rho = [500.0, 1000.0, 1000.0, 1000.0]
    params = {"dt": dt, "output_interval": 1.0e30, "vtk_output_interval": 1.0e30, "end_time": dt * (steps - 0.5),
              "radius_ratio_a": 3.5, "radius_ratio_p": 1.7, "radius_ratio_v": 3.5, "density": rho,
              "bulk_modulus": [r * c_sound ** 2 for r in rho], "bulk_viscosity": [float(mu)] * 4,
              "shear_viscosity": [float(mu)] * 4, "surface_tension": [float(sigma)] * 4,
              "interaction_ratio": [[1.0] * 4 for _ in range(4)], "gravity": [0.0, 0.0, -9.81],
              "wall_center": [[0.0] * 3 for _ in range(4)], "wall_velocity": [[0.0] * 3 for _ in range(4)],
              "wall_omega": [[0.0] * 3 for _ in range(4)]}
    header = {"time": 0.0, "n": len(xyz), "l0": l0, "dmin": [-(walls + pad) * l0] * 3,
              "dmax": [(n + walls + pad) * l0] * 3}
    return params, header, typ, xyz, np.zeros_like(xyz)


def write_data(path: str, p: dict) -> None:
    """*.data with the keys readDataFile parses (main.cpp:502-521)."""
    g = lambda x: "%.17g" % x  # noqa: E731
    four = lambda a: "  ".join(g(a[t]) for t in range(4))  # noqa: E731
    lines = ["#######",
             "Dt                      " + g(p["dt"]),
             "OutputInterval          " + g(p["output_interval"]),
             "VtkOutputInterval       " + g(p["vtk_output_interval"]),
             "EndTime                 " + g(p["end_time"]),
             "RadiusRatioA            " + g(p["radius_ratio_a"]),
             "RadiusRatioP            " + g(p["radius_ratio_p"]),
             "RadiusRatioV            " + g(p["radius_ratio_v"]),
             "Density                 " + four(p["density"]),
             "BulkModulus             " + four(p["bulk_modulus"]),
             "BulkViscosity           " + four(p["bulk_viscosity"]),
             "ShearViscosity          " + four(p["shear_viscosity"]),
             "SurfaceTension          " + four(p["surface_tension"])]
    for t in range(4):
        lines.append("InteractionRatio(Type%d) " % t + four(p["interaction_ratio"][t]))
    lines.append("Gravity                 " + " ".join(g(p["gravity"][d]) for d in range(3)))
    for t in (2, 3):
        lines.append("Wall%d    Center %s    Velocity %s    Omega %s" % (
            t, " ".join(g(p["wall_center"][t][d]) for d in range(3)),
            " ".join(g(p["wall_velocity"][t][d]) for d in range(3)),
            " ".join(g(p["wall_omega"][t][d]) for d in range(3))))
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def write_grid(path: str, h: dict, typ, xyz, vel) -> None:
    """*.grid: Time; N l0 xmin xmax ymin ymax zmin zmax; N lines of
    `type x y z  vx vy vz`, every real as %e."""
    typ = np.asarray(typ)
    xyz = np.asarray(xyz, np.float64)
    vel = np.asarray(vel, np.float64)
    with open(path, "w") as f:
        f.write("%e\n" % h["time"])
        f.write("%d %e %e %e %e %e %e %e\n" % (h["n"], h["l0"], h["dmin"][0], h["dmax"][0], h["dmin"][1],
                                                h["dmax"][1], h["dmin"][2], h["dmax"][2]))
        step = 1 << 16
        for a in range(0, len(typ), step):
            rows = zip(typ[a:a + step].tolist(), *xyz[a:a + step].T.tolist(), *vel[a:a + step].T.tolist())
            f.write("".join("%d %e %e %e  %e %e %e\n" % r for r in rows))


def host_cores() -> dict:
    """Logical CPUs this process may run on, and the physical cores (distinct
    (package, core) pairs of /sys topology) behind them."""
    try:
        cpus = sorted(os.sched_getaffinity(0))
    except AttributeError:
        cpus = list(range(os.cpu_count() or 1))
    phys = set()
    for c in cpus:
        base = "/sys/devices/system/cpu/cpu%d/topology/" % c
        try:
            pkg = open(base + "physical_package_id").read().strip()
            core = open(base + "core_id").read().strip()
            phys.add((pkg, core))
        except OSError:
            phys.add(("?", str(c)))
    model = ""
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return {"logical": len(cpus), "physical": len(phys), "model": model}


def time_reference(data_path: str, grid_path: str, dim: int, warmup: int, steps: int, threads: int,
                   max_seconds: float = 1.0e30, timeout: float = 900, rebuild_at: int = -1) -> dict:
    """Wall-clock the reference's step loop (ref_harness `time`); stops after the
    step that crosses max_seconds and reports the steps done.  rebuild_at=k
    makes the k-th timed step rebuild the neighbour lists."""
    exe = os.path.join(REF_DIR, "ref_mph%dd" % dim)
    with tempfile.TemporaryDirectory() as td:
        env = dict(os.environ, OMP_NUM_THREADS=str(threads))
        cmd = [exe, "time", data_path, grid_path, str(warmup), str(steps), str(threads), repr(float(max_seconds))]
        if rebuild_at >= 0:
            cmd.append("rebuild_at=%d" % rebuild_at)
        r = subprocess.run(cmd, check=True, cwd=td, env=env, timeout=timeout, capture_output=True, text=True)
        return json.loads(r.stdout.strip().splitlines()[-1])


def dam_break_files(td: str, seed: int = 0, **kw):
    """Write the dam break's *.data / *.grid into directory td; returns
    (data path, grid path, particles, fluid)."""
    p, h, t, x, v = dam_break_arrays(seed=seed, **kw)
    d, g = os.path.join(td, "dam.data"), os.path.join(td, "dam.grid")
    write_data(d, p)
    write_grid(g, h, t, x, v)
    return d, g, int(h["n"]), int(np.count_nonzero(t < 2))


def droplet_files(td: str, seed: int = 0, **kw):
    """Write the 2-D droplet's *.data / *.grid into directory td; returns
    (data path, grid path, particles)."""
    p, h, t, x, v = droplet_arrays(seed=seed, **kw)
    d, g = os.path.join(td, "drop.data"), os.path.join(td, "drop.grid")
    write_data(d, p)
    write_grid(g, h, t, x, v)
    return d, g, int(h["n"])


def two_fluid_files(td: str, seed: int = 0, **kw):
    """Write the two-fluid column's *.data / *.grid into directory td; returns
    (data path, grid path, particles, fluid)."""
    p, h, t, x, v = two_fluid_arrays(seed=seed, **kw)
    d, g = os.path.join(td, "column.data"), os.path.join(td, "column.grid")
    write_data(d, p)
    write_grid(g, h, t, x, v)
    return d, g, int(h["n"]), int(np.count_nonzero(t < 2))
