"""The scene generator (mph_read_boid_file / mph_generate_cuboids /
mph_generate_grid_file and the mph_generate command) against the reference's
pre-processor GeneratorForMph (generator/generator.cpp).

* the reference's two sample *.boid files and an edge-case *.boid (width /
  spacing ratios ending in .5, negative coordinates, velocities, type 3):
  the *.grid bytes equal the reference generator's, committed as fixtures
  (tests/golden/make_golden.py) and, where the reference build is present,
  produced live;
* malformed *.boid files return MPH_ERR_IO with a reason (the reference
  prints a message and goes on, or never returns).
"""
import gzip
import os
import subprocess
import tempfile

import numpy as np
import pytest

import mphexplicit_b200 as M
from mphexplicit_b200 import scenes
from mphexplicit_b200 import _native as N
from tests.common import GOLDEN

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_GEN = os.path.join(ROOT, "oracle", "_ref", "GeneratorForMph")
GEN_BIN = os.path.join(ROOT, "mphexplicit_b200", "bin", "mph_generate")
CASES = [("square_drop_skip", "case"), ("bridge", "case"), ("generator", "edge")]


def _golden_grid(folder, stem):
    with gzip.open(os.path.join(GOLDEN, folder, stem + ".grid.gz"), "rb") as g:
        return g.read()


@pytest.mark.parametrize("folder,stem", CASES)
def test_grid_bytes_equal_reference_generator(folder, stem):
    boid = os.path.join(GOLDEN, folder, stem + ".boid")
    with tempfile.TemporaryDirectory() as td:
        out = os.path.join(td, "out.grid")
        n = M.generate_grid_file(boid, out)
        got = open(out, "rb").read()
    want = _golden_grid(folder, stem)
    assert got == want
    assert n == int(want.split(b"\n")[1].split()[0])


@pytest.mark.parametrize("folder,stem", CASES)
def test_cli_equals_reference_generator(folder, stem):
    """`mph_generate <stem>` reads <stem>.boid and writes <stem>.grid, as
    `GeneratorForMph <stem>` does; also against the live reference build."""
    with tempfile.TemporaryDirectory() as td:
        with open(os.path.join(GOLDEN, folder, stem + ".boid"), "rb") as f:
            text = f.read()
        with open(os.path.join(td, "s.boid"), "wb") as f:
            f.write(text)
        subprocess.run([GEN_BIN, "s"], cwd=td, check=True, capture_output=True)
        got = open(os.path.join(td, "s.grid"), "rb").read()
        assert got == _golden_grid(folder, stem)
        if os.path.exists(REF_GEN):
            os.rename(os.path.join(td, "s.grid"), os.path.join(td, "mine.grid"))
            subprocess.run([REF_GEN, "s"], cwd=td, check=True, capture_output=True)
            assert got == open(os.path.join(td, "s.grid"), "rb").read()


def test_boid_reader_and_lattice_half_ratios():
    b, cub = M.read_boid_file(os.path.join(GOLDEN, "generator", "edge.boid"))
    assert b.particle_distance == 0.01 and b.cuboid_count == 2 and len(cub) == 2
    assert list(b.lower_domain) == [-0.2, -0.2, -0.1] and list(b.upper_domain) == [0.3, 0.3, 0.1]
    c = cub[0]
    assert c.type == 0 and c.spacing == 0.01 and list(c.velocity) == [0.5, -0.25, 0.125]
    # width/spacing = 12.5 in x: C round gives 13 points (Python's round would give 12)
    t, x, v = M.generate_cuboids(cub[:1])
    nx = len(np.unique(x[:, 0]))
    assert nx == 13
    assert np.all(t == 0) and np.all(v == [0.5, -0.25, 0.125])
    # scenes.cuboid_grid goes through the same generator
    h, t2, x2, v2 = scenes.cuboid_grid([(c.spacing, c.type, list(c.lower), list(c.upper), list(c.velocity))],
                                       0.01, b.lower_domain, b.upper_domain)
    assert np.array_equal(x2, x) and np.array_equal(t2, t) and h.particle_count == len(t)


@pytest.mark.parametrize("text,why", [
    ("ParticleDistance 0.1\nLowerDomain 0 0 0\nUpperDomain 1 1 1\nStartCuboid\n Spacing 0.1\n Type 0\n",
     "EndCuboid"),
    ("ParticleDistance 0.1\nLowerDomain 0 0 0\nUpperDomain 1 1 1\nStartCuboid\n Spacing 0.1\n Colour 3\nEndCuboid\n",
     "unknown cuboid key"),
    ("ParticleDistance 0.1\nLowerDomain 0 0 0\nStartCuboid\n Spacing 0.1 Type 0 Lower 0 0 0 Upper 1 1 1 "
     "Velocity 0 0 0\nEndCuboid\n", "UpperDomain"),
    ("ParticleDistance 0.1\nLowerDomain 0 0 0\nUpperDomain 1 1 1\nStartCuboid\n Spacing 0.1\n Type 0\n"
     " Lower 0 0 0\nEndCuboid\n", "needs Spacing"),
])
def test_malformed_boid_is_an_error(text, why):
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "bad.boid")
        with open(p, "w") as f:
            f.write(text)
        with pytest.raises(M.MphError) as e:
            M.generate_grid_file(p, os.path.join(td, "bad.grid"))
        assert e.value.code == N.MPH_ERR_IO and why in str(e.value)
        r = subprocess.run([GEN_BIN, os.path.join(td, "bad")], capture_output=True, text=True)
        assert r.returncode != 0 and why in r.stderr


def test_missing_boid_file():
    with pytest.raises(M.MphError) as e:
        M.read_boid_file("/nonexistent/x.boid")
    assert e.value.code == N.MPH_ERR_IO
