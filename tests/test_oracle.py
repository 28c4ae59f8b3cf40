"""The CPU oracle (oracle/mph_oracle.c) pinned against the reference.

* against every committed golden fixture (the reference's own arrays after k
  steps, tests/golden/make_golden.py), bit for bit;
* against the reference run here on fresh seeded scenes, when the reference
  build (oracle/_ref) is present;
* against the known-answer lattice constants N0a/N0p.
"""
import os
import tempfile

import numpy as np
import pytest

from mphexplicit_b200 import read_data_file, read_grid_file, scenes
from oracle import pyoracle as po
from tests.common import (micro_cases, CASES, CELL_KEYS, FIELD_KEYS, STATE_KEYS, GoldenCase, assert_same,
                          csr_digests)


def run_oracle(case: GoldenCase):
    p = read_data_file(case.data)
    g = read_grid_file(case.grid)
    o = po.Oracle(p, g.header, g.type, g.xyz, g.vel, case.dim)
    o.step(case.steps)
    o.virial()
    return o


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_golden(name):
    case = GoldenCase(name)
    o = run_oracle(case)
    s, f, c = o.state(), o.fields(), o.cells()
    for k in STATE_KEYS:
        assert_same(s[k], case.ref[k], k)
    for k in FIELD_KEYS:
        assert_same(f[k], case.ref[k], k)
    for k in CELL_KEYS:
        assert_same(c[k], case.ref[k], k)
    ptr, ind = o.neighbors()
    assert_same(ptr, case.ref["nptr"], "NeighborPtr")
    assert_same(ind, case.ref["nind"], "NeighborInd")
    assert o.rebuilds == case.rebuilds
    assert o.constants().n0a == float(case.ref["n0a"])
    assert o.constants().n0p == float(case.ref["n0p"])


def test_oracle_matches_golden_two_fluid_1000_steps():
    """The 1000-step 3-D two-fluid case (surface tension, interaction ratios
    != 1, 7 rebuilds) bit for bit; its neighbour list through the digests.
    (The 1000-step dam break, 22k particles, is compared on the GPU only.)"""
    case = GoldenCase("two_fluid_1000")
    o = run_oracle(case)
    s, f, c = o.state(), o.fields(), o.cells()
    for k in STATE_KEYS:
        assert_same(s[k], case.ref[k], k)
    for k in FIELD_KEYS:
        assert_same(f[k], case.ref[k], k)
    for k in CELL_KEYS:
        assert_same(c[k], case.ref[k], k)
    ptr, ind = o.neighbors()
    assert csr_digests(ptr, ind) == (str(case.ref["nptr_sha256"]), str(case.ref["nind_sha256"]))
    assert o.rebuilds == case.rebuilds


# Known-answer lattice sums (main.cpp:861-949), values printed by the reference.
@pytest.mark.parametrize("dim,ra,rp,n0a,n0a_count,n0p,n0p_count", [
    (2, 3.5, 1.75, 0.97430960741661099, None, 0.55001609129137918, None),
    (2, 3.5, 1.7, 0.9743096, 36, 0.5228945, 8),
    (3, 3.5, 1.7, 0.9907023, 178, 0.6591169, 18),
])
def test_lattice_constants(dim, ra, rp, n0a, n0a_count, n0p, n0p_count):
    from mphexplicit_b200 import default_params, make_header
    p = default_params()
    p.radius_ratio_a, p.radius_ratio_p, p.radius_ratio_v = ra, rp, ra
    h = make_header(1, 0.004, (-1, -1, -1), (1, 1, 1))
    c = po.constants(p, h, dim)
    assert abs(c.n0a - n0a) < 5e-7 and abs(c.n0p - n0p) < 5e-7
    if n0a_count is not None:
        assert c.n0a_count == n0a_count and c.n0p_count == n0p_count


def _fresh_scenes():
    yield scenes.droplet_2d(n=16, seed=11, steps=40), 40
    yield scenes.dam_break_3d(fluid=(6, 6, 10), box=(14, 6, 14), walls=3, seed=12), 40
    sc = scenes.two_fluid_column(n=8, seed=13, steps=30)
    yield sc, 30


@pytest.mark.skipif(not (po.ref_available(2) and po.ref_available(3)), reason="reference build absent")
def test_oracle_matches_reference_fresh():
    with tempfile.TemporaryDirectory() as td:
        for sc, steps in _fresh_scenes():
            d, g = os.path.join(td, "a.data"), os.path.join(td, "a.grid")
            sc.write(d, g)
            ref = po.run_reference(d, g, sc.dim, steps, virial=True)
            gr = read_grid_file(g)
            o = po.Oracle(read_data_file(d), gr.header, gr.type, gr.xyz, gr.vel, sc.dim)
            o.step(steps)
            o.virial()
            s = o.state()
            for k in STATE_KEYS:
                assert_same(s[k], ref[k], f"{sc.name}:{k}")
            assert o.rebuilds == ref["rebuilds"]


def test_oracle_rejects_bad_geometry():
    # cells narrower than MaxRadius+MARGIN: the reference asserts (main.cpp:1347)
    p = scenes.make_params(dt=1e-5, density=1000.0, bulk_modulus=1e5, bulk_viscosity=0.1, shear_viscosity=0.1,
                           surface_tension=0.0)
    from mphexplicit_b200 import make_header
    h = make_header(2, 1.0, (0, 0, 0), (36.0, 36.0, 36.0))  # W/(3.6) = 10 exactly -> width may round below
    p.radius_ratio_a = p.radius_ratio_v = 3.5
    p.radius_ratio_p = 1.7
    c = po.constants(p, h, 3)
    rm = c.max_radius + 0.1
    ranges = [int(np.ceil(rm / c.cell_width[d])) for d in range(3)]
    t = np.zeros(2, np.int32)
    x = np.array([[1.0, 1.0, 1.0], [2.0, 1.0, 1.0]])
    if max(ranges) > 1:
        with pytest.raises(ValueError):
            po.Oracle(p, h, t, x, np.zeros_like(x), 3)
    else:
        po.Oracle(p, h, t, x, np.zeros_like(x), 3).close()


@pytest.mark.skipif(not (po.ref_available(2) and po.ref_available(3)), reason="reference build absent")
@pytest.mark.parametrize("k", range(6))
def test_oracle_matches_reference_micro(k):
    """Micro-cases (pairs at every radius, a lone particle, an isolated wall,
    every periodic face, a thin 2-D grid) against the reference itself."""
    (name, sc), steps = list(micro_cases())[k]
    with tempfile.TemporaryDirectory() as td:
        d, g = os.path.join(td, "a.data"), os.path.join(td, "a.grid")
        sc.write(d, g)
        ref = po.run_reference(d, g, sc.dim, steps, virial=True)
        gr = read_grid_file(g)
        o = po.Oracle(read_data_file(d), gr.header, gr.type, gr.xyz, gr.vel, sc.dim)
        o.step(steps)
        o.virial()
        s = o.state()
        for key in STATE_KEYS:
            assert_same(s[key], ref[key], f"{name}:{key}")
        assert o.rebuilds == ref["rebuilds"]
