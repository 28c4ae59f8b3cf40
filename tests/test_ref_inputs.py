"""The reference arm's inputs (oracle/ref_inputs.py) equal the product's scene.

bench.py's CPU legs time the reference on files written by oracle/ref_inputs,
which loads nothing of the product.  These tests pin that those files hold
the same scene as the one the GPU arm steps: the same arrays element for
element, the same *.data bytes and the same *.grid bytes as the product's
writers; and that the timing command of the reference harness reports the
steps, warm-up and the forced neighbour rebuild it was asked for (the rebuild
is a timing device only: it reorders the particles, so the state after it is
not compared with anything).
"""
import os
import tempfile

import numpy as np
import pytest

from mphexplicit_b200 import scenes
from oracle import ref_inputs as RI


@pytest.mark.parametrize("fluid,box,seed", [((6, 5, 7), (14, 6, 12), 0), ((9, 4, 5), (20, 7, 9), 3)])
def test_dam_break_arrays_equal_product_scene(fluid, box, seed):
    sc = scenes.dam_break_3d(fluid=fluid, box=box, seed=seed)
    p, h, t, x, v = RI.dam_break_arrays(fluid=fluid, box=box, seed=seed)
    assert np.array_equal(t, sc.type)
    assert np.array_equal(x, sc.xyz)
    assert np.array_equal(v, sc.vel)
    assert h["n"] == sc.n and h["l0"] == sc.header.particle_spacing
    for d in range(3):
        assert h["dmin"][d] == sc.header.domain_min[d] and h["dmax"][d] == sc.header.domain_max[d]
    with tempfile.TemporaryDirectory() as td:
        d1, g1 = os.path.join(td, "a.data"), os.path.join(td, "a.grid")
        d2, g2 = os.path.join(td, "b.data"), os.path.join(td, "b.grid")
        sc.write(d1, g1)                       # the product's writers (C ABI)
        RI.write_data(d2, p)
        RI.write_grid(g2, h, t, x, v)
        assert open(d1, "rb").read() == open(d2, "rb").read()
        assert open(g1, "rb").read() == open(g2, "rb").read()


@pytest.mark.parametrize("n,seed", [(40, 0), (12, 5)])
def test_droplet_arrays_equal_product_scene(n, seed):
    sc = scenes.droplet_2d(n=n, seed=seed)
    p, h, t, x, v = RI.droplet_arrays(n=n, seed=seed)
    assert np.array_equal(t, sc.type) and np.array_equal(x, sc.xyz) and np.array_equal(v, sc.vel)
    with tempfile.TemporaryDirectory() as td:
        d1, g1 = os.path.join(td, "a.data"), os.path.join(td, "a.grid")
        d2, g2 = os.path.join(td, "b.data"), os.path.join(td, "b.grid")
        sc.write(d1, g1)
        RI.write_data(d2, p)
        RI.write_grid(g2, h, t, x, v)
        assert open(d1, "rb").read() == open(d2, "rb").read()
        assert open(g1, "rb").read() == open(g2, "rb").read()


def test_two_fluid_arrays_equal_product_scene():
    sc = scenes.two_fluid_column(n=10, seed=4)
    p, h, t, x, v = RI.two_fluid_arrays(n=10, seed=4)
    assert np.array_equal(t, sc.type) and np.array_equal(x, sc.xyz) and np.array_equal(v, sc.vel)
    with tempfile.TemporaryDirectory() as td:
        d1, g1 = os.path.join(td, "a.data"), os.path.join(td, "a.grid")
        d2, g2 = os.path.join(td, "b.data"), os.path.join(td, "b.grid")
        sc.write(d1, g1)
        RI.write_data(d2, p)
        RI.write_grid(g2, h, t, x, v)
        assert open(d1, "rb").read() == open(d2, "rb").read()
        assert open(g1, "rb").read() == open(g2, "rb").read()


def test_host_cores():
    c = RI.host_cores()
    assert c["logical"] >= 1 and 1 <= c["physical"] <= c["logical"]


@pytest.mark.skipif(not RI.ref_available(3), reason="reference build absent")
def test_time_reference_forced_rebuild():
    with tempfile.TemporaryDirectory() as td:
        d, g, n, nf = RI.dam_break_files(td, fluid=(6, 5, 7), box=(14, 6, 12))
        r = RI.time_reference(d, g, 3, 1, 3, 1, rebuild_at=1)
        assert r["steps"] == 3 and r["warmup"] == 1 and r["rebuilds"] == 1
        assert r["particles"] == n and r["fluid"] == nf
        r = RI.time_reference(d, g, 3, 0, 2, 1)
        assert r["rebuilds"] == 0


@pytest.mark.skipif(not RI.ref_available(2), reason="reference build absent")
def test_time_reference_droplet_2d():
    """The reference's 2-D build steps the droplet the bench times it on."""
    with tempfile.TemporaryDirectory() as td:
        d, g, n = RI.droplet_files(td, n=12, seed=1)
        r = RI.time_reference(d, g, 2, 1, 5, 1)
        assert r["steps"] == 5 and r["particles"] == n == 144 and r["seconds"] > 0.0


@pytest.mark.skipif(not RI.ref_available(3), reason="reference build absent")
def test_time_reference_two_fluid_column():
    """... and the two-fluid column (scaled down)."""
    with tempfile.TemporaryDirectory() as td:
        d, g, n, nf = RI.two_fluid_files(td, n=8, seed=2)
        r = RI.time_reference(d, g, 3, 0, 2, 2)
        assert r["steps"] == 2 and r["particles"] == n and r["fluid"] == nf == 512
