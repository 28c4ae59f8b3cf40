"""Regenerate the golden fixtures in tests/golden/ from the reference itself.

Run where the reference sources are checked out, with REF (or
MPH_REFERENCE_DIR) naming that checkout, after ``make -C oracle ref REF=...``.  Each case is a *.data/*.grid
pair; the fixture holds the reference's arrays after `steps` steps (its own
code via oracle/_ref/ref_mph{2,3}d, see oracle/ref_harness.cpp), compressed.

Cases:
  square_drop_skip  reference sample results/SquareDropSkip_l00400_rv35_rp17
                    (grid made by the reference's own generator), 300 steps
  bridge            reference sample results/Bridge_l00100_deg000_re35_mu01_g98,
                    300 steps
  moving_walls      the SquareDropSkip input with type-2 walls translating and
                    rotating (exercises main.cpp:994-1053), 200 steps
  droplet_2d        benchmark config 1 (40x40 droplet, sigma 0.07), 1000 steps
  dam_break_small   benchmark config 2 scaled to 8x8x16 fluid in a 24x8x20 box,
                    200 steps
  two_fluid_small   benchmark config 3 scaled to 10^3, interaction ratios != 1,
                    100 steps
  dam_break_1000    benchmark config 2 scaled to 16x12x24 fluid in a 48x12x29-cell
                    box (3 wall layers), started from the reference's own *.prof
                    after 600 steps (inside the collapse, where the lists are
                    rebuilt every few tens of steps), 1000 steps
  two_fluid_1000    benchmark config 3 scaled to 12^3 (surface tension, interaction
                    ratios != 1), started from the reference's *.prof after 300
                    steps, 1000 steps

generator/edge     a *.boid of the generator's edge cases and the reference
                    generator's *.grid of it (the two samples above keep their
                    *.boid beside the generator's *.grid as well)

The two 1000-step cases keep the neighbour list as SHA-256 digests of the
reference's NeighborPtr / NeighborInd bytes (the lists themselves would be
several MB); every other array is kept whole.
"""
from __future__ import annotations

import gzip
import hashlib
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from mphexplicit_b200 import scenes  # noqa: E402
from mphexplicit_b200.scenes import write_data_file  # noqa: E402
from oracle import pyoracle as po  # noqa: E402

REF = os.environ.get("REF") or os.environ.get("MPH_REFERENCE_DIR") or ""
LONG_CASES = ("dam_break_1000", "two_fluid_1000")
KEEP = ["particle_index", "type", "xyz", "vel", "force", "neighbor_count", "density_a", "vol_strain_p",
        "virial_pressure", "divergence_p", "pressure_p", "pressure_a", "gravity_center", "cell_index",
        "fluid_begin", "fluid_end", "wall_begin", "wall_end", "nptr", "nind"]


def sample_inputs(case_dir: str, out_dir: str) -> None:
    with tempfile.TemporaryDirectory() as td:
        shutil.copyfile(os.path.join(REF, "results", case_dir, "box.boid"), os.path.join(td, "box.boid"))
        shutil.copyfile(os.path.join(REF, "results", case_dir, "box.data"), os.path.join(td, "box.data"))
        subprocess.run([os.path.join(ROOT, "oracle", "_ref", "GeneratorForMph"), "box"], cwd=td, check=True,
                       stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        shutil.copyfile(os.path.join(td, "box.data"), os.path.join(out_dir, "case.data"))
        shutil.copyfile(os.path.join(td, "box.boid"), os.path.join(out_dir, "case.boid"))
        with open(os.path.join(td, "box.grid"), "rb") as f, gzip.GzipFile(os.path.join(out_dir, "case.grid.gz"), "wb",
                                                                           mtime=0) as g:
            g.write(f.read())


def scene_inputs(sc, out_dir: str) -> None:
    with tempfile.TemporaryDirectory() as td:
        sc.write(os.path.join(out_dir, "case.data"), os.path.join(td, "case.grid"))
        with open(os.path.join(td, "case.grid"), "rb") as f, gzip.GzipFile(os.path.join(out_dir, "case.grid.gz"), "wb",
                                                                           mtime=0) as g:
            g.write(f.read())


def preroll_inputs(sc, pre_steps: int, out_dir: str) -> None:
    """Inputs inside the developed flow: the scene's *.data, and as *.grid the
    reference's own *.prof after `pre_steps` steps (writeProfFile,
    main.cpp:672-696; the file its main() restarts from, main.cpp:371, 550)."""
    with tempfile.TemporaryDirectory() as td:
        d, g, prof = os.path.join(td, "case.data"), os.path.join(td, "case.grid"), os.path.join(td, "pre.prof")
        sc.write(d, g)
        po.run_reference(d, g, sc.dim, pre_steps, timeout=7200, prof=prof)
        shutil.copyfile(d, os.path.join(out_dir, "case.data"))
        with open(prof, "rb") as f, gzip.GzipFile(os.path.join(out_dir, "case.grid.gz"), "wb", mtime=0) as z:
            z.write(f.read())


def record(name: str, dim: int, steps: int) -> None:
    out_dir = os.path.join(HERE, name)
    with tempfile.TemporaryDirectory() as td:
        grid = os.path.join(td, "case.grid")
        with gzip.open(os.path.join(out_dir, "case.grid.gz"), "rb") as g, open(grid, "wb") as f:
            f.write(g.read())
        vtk = os.path.join(td, "case.vtk")
        prof = os.path.join(td, "case.prof")
        d = po.run_reference(os.path.join(out_dir, "case.data"), grid, dim, steps, virial=True, timeout=3600,
                             vtk=vtk, prof=prof)
        if name in ("square_drop_skip", "dam_break_small"):  # the reference's own output bytes
            for src, dst in ((vtk, "reference.vtk.gz"), (prof, "reference.prof.gz")):
                with open(src, "rb") as f, gzip.GzipFile(os.path.join(out_dir, dst), "wb", mtime=0) as g:
                    g.write(f.read())
    meta = np.array([dim, steps, d["rebuilds"], d["neighbor_ind_count"], d["total_cell_count"]] + d["cell_count"],
                    np.int64)
    keep = {k: d[k] for k in KEEP}
    if name in LONG_CASES:
        for k in ("nptr", "nind"):
            keep[k + "_sha256"] = np.array(hashlib.sha256(np.ascontiguousarray(keep.pop(k)).tobytes()).hexdigest())
    np.savez_compressed(os.path.join(out_dir, "reference.npz"), meta=meta, time=np.array(d["time"]),
                        n0a=np.array(d["n0a"]), n0p=np.array(d["n0p"]), **keep)
    print(name, "n", d["n"], "steps", steps, "rebuilds", d["rebuilds"], "NeighborIndCount",
          d["neighbor_ind_count"])


# A *.boid for the generator's edge cases: width/spacing ratios ending in .5
# (C round takes them away from zero), negative coordinates, a non-zero
# velocity, a cuboid of type 3, a comment and a blank line.
GENERATOR_BOID = """# generator edge cases
ParticleDistance 0.01
LowerDomain -0.2 -0.2 -0.1
UpperDomain  0.3  0.3  0.1

StartCuboid
  Spacing 0.01
  Type 0
  Lower -0.1 -0.05 -0.0125
  Upper  0.025 0.0 0.0125
  Velocity 0.5 -0.25 0.125
EndCuboid
StartCuboid
  Spacing 0.02
  Type 3
  Lower 0.1 0.1 -0.05
  Upper 0.15 0.13 0.05
  Velocity 0 0 0
EndCuboid
"""


def generator_case() -> None:
    """tests/golden/generator/edge.boid and the reference generator's *.grid of it."""
    out_dir = os.path.join(HERE, "generator")
    os.makedirs(out_dir, exist_ok=True)
    with open(os.path.join(out_dir, "edge.boid"), "w") as f:
        f.write(GENERATOR_BOID)
    with tempfile.TemporaryDirectory() as td:
        shutil.copyfile(os.path.join(out_dir, "edge.boid"), os.path.join(td, "edge.boid"))
        subprocess.run([os.path.join(ROOT, "oracle", "_ref", "GeneratorForMph"), "edge"], cwd=td, check=True,
                       stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        with open(os.path.join(td, "edge.grid"), "rb") as f, gzip.GzipFile(os.path.join(out_dir, "edge.grid.gz"),
                                                                           "wb", mtime=0) as g:
            g.write(f.read())


def long_cases() -> list:
    """The two 1000-step 3-D cases (inputs pre-rolled by the reference)."""
    cases = []
    sc = scenes.dam_break_3d(fluid=(16, 12, 24), box=(48, 12, 29), seed=5)
    os.makedirs(os.path.join(HERE, "dam_break_1000"), exist_ok=True)
    preroll_inputs(sc, 600, os.path.join(HERE, "dam_break_1000"))
    cases.append(("dam_break_1000", 3, 1000))
    sc = scenes.two_fluid_column(n=12, l0=0.0025, seed=6, steps=1000)
    rng = np.random.default_rng(6)
    for a in range(4):
        for b in range(4):
            sc.params.interaction_ratio[a][b] = float(rng.uniform(0.5, 1.5))
    os.makedirs(os.path.join(HERE, "two_fluid_1000"), exist_ok=True)
    preroll_inputs(sc, 300, os.path.join(HERE, "two_fluid_1000"))
    cases.append(("two_fluid_1000", 3, 1000))
    return cases


def main() -> None:
    if not REF or not os.path.isdir(os.path.join(REF, "source")):
        raise SystemExit("set REF (or MPH_REFERENCE_DIR) to the reference checkout")
    if sys.argv[1:] == ["generator"]:  # only the generator's fixtures
        generator_case()
        for name, src in (("square_drop_skip", "SquareDropSkip_l00400_rv35_rp17"),
                          ("bridge", "Bridge_l00100_deg000_re35_mu01_g98")):
            shutil.copyfile(os.path.join(REF, "results", src, "box.boid"), os.path.join(HERE, name, "case.boid"))
        return
    if sys.argv[1:] == ["long"]:  # only the two 1000-step cases
        for name, dim, steps in long_cases():
            record(name, dim, steps)
        return
    cases = []
    for name, src in (("square_drop_skip", "SquareDropSkip_l00400_rv35_rp17"),
                      ("bridge", "Bridge_l00100_deg000_re35_mu01_g98")):
        os.makedirs(os.path.join(HERE, name), exist_ok=True)
        sample_inputs(src, os.path.join(HERE, name))
        cases.append((name, 2, 300))
    # moving walls: the SquareDropSkip input with moving type-2 walls
    name = "moving_walls"
    os.makedirs(os.path.join(HERE, name), exist_ok=True)
    sample_inputs("SquareDropSkip_l00400_rv35_rp17", os.path.join(HERE, name))
    from mphexplicit_b200 import read_data_file  # noqa: E402
    p = read_data_file(os.path.join(HERE, name, "case.data"))
    p.wall_center[2][0], p.wall_center[2][1] = 1.5, 0.3
    p.wall_velocity[2][0], p.wall_velocity[2][1] = 0.05, 0.02
    p.wall_omega[2][2] = 0.7
    write_data_file(os.path.join(HERE, name, "case.data"), p)
    cases.append((name, 2, 200))
    for name, sc, steps in (
            ("droplet_2d", scenes.droplet_2d(n=40, seed=1), 1000),
            ("dam_break_small", scenes.dam_break_3d(fluid=(8, 8, 16), box=(24, 8, 20), seed=2), 200),
            ("two_fluid_small", scenes.two_fluid_column(n=10, l0=0.0025, seed=3, steps=100), 100)):
        if name == "two_fluid_small":
            rng = np.random.default_rng(3)
            for a in range(4):
                for b in range(4):
                    sc.params.interaction_ratio[a][b] = float(rng.uniform(0.5, 1.5))
        os.makedirs(os.path.join(HERE, name), exist_ok=True)
        scene_inputs(sc, os.path.join(HERE, name))
        cases.append((name, sc.dim, steps))
    generator_case()
    cases += long_cases()
    for name, dim, steps in cases:
        record(name, dim, steps)


if __name__ == "__main__":
    main()
