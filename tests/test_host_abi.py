"""Host side of the C ABI, without a GPU: symbols, file formats, set-up
constants and argument validation (no kernel launches)."""
import os
import re
import tempfile

import numpy as np
import pytest

import mphexplicit_b200 as M
from mphexplicit_b200 import _native as N
from mphexplicit_b200 import scenes
from oracle import pyoracle as po
from tests.common import GoldenCase, assert_same

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "mph_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(mph_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    lib = N.load()
    names = declared_symbols()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) <= set(N.SIGNATURES), set(names) - set(N.SIGNATURES)
    assert b"sm_100a" in lib.mph_version()


def test_read_sample_data_file():
    case = GoldenCase("square_drop_skip")
    p = M.read_data_file(case.data)
    assert p.dt == 5.0e-4 and p.end_time == 1.0 and p.vtk_output_interval == 5.0e-2
    assert list(p.density) == [1.0e3] * 4 and list(p.bulk_modulus) == [1.0e6] * 4
    assert list(p.bulk_viscosity) == [2.0e3] * 4 and list(p.shear_viscosity) == [1.0e3] * 4
    assert (p.radius_ratio_a, p.radius_ratio_p, p.radius_ratio_v) == (3.5, 1.75, 3.5)
    assert list(p.gravity) == [0.0, -1.0, 0.0]
    assert all(p.interaction_ratio[a][b] == 1.0 for a in range(4) for b in range(4))


def test_data_file_round_trip_and_unknown_lines():
    p = scenes.make_params(dt=1.2345678901234567e-5, density=[500.0, 1000.0, 1e3, 2e3], bulk_modulus=1e5,
                           bulk_viscosity=0.3, shear_viscosity=0.1, surface_tension=0.0725, gravity=(0.1, -9.8, 0.3))
    p.wall_velocity[2][0] = 0.25
    p.wall_omega[3][2] = -1.5
    p.wall_center[3][1] = 0.125
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "x.data")
        scenes.write_data_file(path, p)
        with open(path, "a") as f:
            f.write("NotAKey 1 2 3\n")
        q = M.read_data_file(path)
    for name, _ in N.Params._fields_:
        a, b = getattr(p, name), getattr(q, name)
        assert np.array_equal(np.ctypeslib.as_array(a) if not isinstance(a, float) else a,
                              np.ctypeslib.as_array(b) if not isinstance(b, float) else b), name


def test_missing_files_raise_io_error():
    with pytest.raises(M.MphError) as e:
        M.read_data_file("/nonexistent/x.data")
    assert e.value.code == N.MPH_ERR_IO
    with pytest.raises(M.MphError) as e:
        M.read_grid_file("/nonexistent/x.grid")
    assert e.value.code == N.MPH_ERR_IO


def test_truncated_grid_file_is_an_error():
    case = GoldenCase("square_drop_skip")
    lines = open(case.grid).read().splitlines()
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "t.grid")
        open(path, "w").write("\n".join(lines[:100]) + "\n")
        with pytest.raises(M.MphError) as e:
            M.read_grid_file(path)
        assert e.value.code == N.MPH_ERR_IO


def test_grid_round_trip():
    sc = scenes.dam_break_3d(fluid=(4, 4, 4), box=(8, 6, 8), walls=2, seed=3)
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "a.grid")
        M.write_grid_file(path, sc.header, sc.type, sc.xyz, sc.vel)
        g = M.read_grid_file(path)
        path2 = os.path.join(td, "b.grid")
        M.write_grid_file(path2, g.header, g.type, g.xyz, g.vel)
        assert open(path).read() == open(path2).read()
    assert np.array_equal(g.type, sc.type)
    assert np.allclose(g.xyz, sc.xyz, rtol=1e-6, atol=1e-12)


@pytest.mark.parametrize("name", ["square_drop_skip", "dam_break_small"])
def test_writers_match_reference_bytes(name):
    """VTK and prof text from the reference's own writers after k steps equals
    ours given the same (oracle) arrays: same formats, same float casts."""
    case = GoldenCase(name)
    p = M.read_data_file(case.data)
    g = M.read_grid_file(case.grid)
    o = po.Oracle(p, g.header, g.type, g.xyz, g.vel, case.dim)
    o.step(case.steps)
    o.virial()
    s = o.state()
    with tempfile.TemporaryDirectory() as td:
        vtk = os.path.join(td, "x.vtk")
        M.write_vtk_arrays(vtk, s)
        assert open(vtk, "rb").read() == case.reference_bytes("vtk")
        prof = os.path.join(td, "x.prof")
        h = g.header
        h.time = o.time
        M.write_grid_file(prof, h, s["type"], s["xyz"], s["vel"])
        assert open(prof, "rb").read() == case.reference_bytes("prof")


@pytest.mark.parametrize("dim,make", [
    (2, lambda: scenes.droplet_2d(n=10)),
    (3, lambda: scenes.dam_break_3d(fluid=(4, 4, 4), box=(10, 8, 10))),
    (3, lambda: scenes.two_fluid_column(n=6)),
])
def test_constants_match_oracle(dim, make):
    sc = make()
    sc.params.wall_omega[2][2] = 0.3
    sc.params.wall_omega[3][0] = -0.2
    a = M.compute_constants(sc.params, sc.header, dim)
    b = po.constants(sc.params, sc.header, dim)
    for name, _ in N.Constants._fields_:
        va, vb = getattr(a, name), getattr(b, name)
        if isinstance(va, (int, float)):
            assert va == vb, name
        else:
            assert_same(np.ctypeslib.as_array(va), np.ctypeslib.as_array(vb), name)


def test_create_validates_before_touching_the_device():
    sc = scenes.droplet_2d(n=4)
    bad = sc.type.copy()
    bad[0] = 7
    with pytest.raises(M.MphError) as e:
        M.Solver(sc.params, sc.header, bad, sc.xyz, sc.vel, dim=2)
    assert e.value.code == N.MPH_ERR_ARG
    x = sc.xyz.copy()
    x[1, 0] = np.nan
    with pytest.raises(M.MphError) as e:
        M.Solver(sc.params, sc.header, sc.type, x, sc.vel, dim=2)
    assert e.value.code == N.MPH_ERR_NONFINITE
    with pytest.raises(M.MphError) as e:
        M.Solver(sc.params, sc.header, sc.type, sc.xyz, sc.vel, dim=4)
    assert e.value.code == N.MPH_ERR_ARG
    # a domain narrower than one cell of MaxRadius+MARGIN: no cell grid
    p = sc.params
    p.radius_ratio_a = p.radius_ratio_v = 60.0  # 0.24 m radius in a 0.2 m wide domain
    h = M.make_header(sc.n, sc.header.particle_spacing, (-0.1, -0.1, -0.002), (0.1, 0.1, 0.002))
    with pytest.raises(M.MphError) as e:
        M.Solver(p, h, sc.type, sc.xyz, sc.vel, dim=2)
    assert e.value.code == N.MPH_ERR_GEOMETRY
    # a width that is an exact multiple of the cut-off can round the cell width
    # below MaxRadius+MARGIN; the reference asserts then (main.cpp:1347-1349)
    l0 = sc.header.particle_spacing
    p.radius_ratio_a = p.radius_ratio_v = 3.5
    for k in range(3, 400):
        rm = 3.5 * l0 + 0.1 * l0
        w = k * rm
        h = M.make_header(sc.n, l0, (-0.5 * w, -0.5 * w, -0.002), (0.5 * w, 0.5 * w, 0.002))
        c = M.compute_constants(p, h, 2)
        if min(c.cell_width[0], c.cell_width[1]) < c.max_radius + 0.1 * l0:
            with pytest.raises(M.MphError) as e:
                M.Solver(p, h, sc.type, sc.xyz, sc.vel, dim=2)
            assert e.value.code == N.MPH_ERR_GEOMETRY
            break


def test_benchmark_scene_sizes():
    # config 2: 100x100x200 fluid, 3 wall layers around a closed 300x100x240 box
    f = 100 * 100 * 200
    w = 306 * 106 * 246 - 300 * 100 * 240
    assert (f, w) == (2_000_000, 779_256)
    sc = scenes.dam_break_3d(fluid=(10, 10, 20), box=(30, 10, 24))
    assert sc.n_fluid == 2000 and sc.n - sc.n_fluid == 36 * 16 * 30 - 30 * 10 * 24
    c = M.compute_constants(sc.params, sc.header, 3)
    rm = c.max_radius + 0.1 * sc.header.particle_spacing
    assert all(c.cell_width[d] > rm for d in range(3))
    d1 = scenes.droplet_2d()
    assert d1.n == 1600 and d1.dim == 2
    assert np.array_equal(scenes.droplet_2d(seed=5).xyz, scenes.droplet_2d(seed=5).xyz)
    b = scenes.droplet_batch_2d(count=8, seed=1)
    assert len(b) == 8 and all(20 * 20 <= s.n <= 140 * 140 for s in b)


def test_batch_rejects_bad_scenes_before_touching_the_gpu():
    """mph_batch_create validates every scene on the host first."""
    good = scenes.droplet_batch_2d(count=2, seed=1, lo=10, hi=12)
    with pytest.raises(ValueError):
        M.Batch([])
    moving = scenes.droplet_batch_2d(count=1, seed=2, lo=10, hi=12)[0]
    moving.params.wall_velocity[2][0] = 0.1
    with pytest.raises(M.MphError) as e:
        M.Batch([good[0], moving])
    assert e.value.code == N.MPH_ERR_ARG and "static walls" in str(e.value)
    tiny = scenes.droplet_2d(n=4, box=6.0)  # fewer than 3 cells per axis
    with pytest.raises(M.MphError) as e:
        M.Batch([good[1], tiny])
    assert e.value.code == N.MPH_ERR_GEOMETRY and "scene 1" in str(e.value)
    bad = scenes.droplet_batch_2d(count=1, seed=3, lo=10, hi=12)[0]
    bad.type[0] = 7
    with pytest.raises(M.MphError) as e:
        M.Batch([bad])
    assert e.value.code == N.MPH_ERR_ARG
    nan = scenes.droplet_batch_2d(count=1, seed=4, lo=10, hi=12)[0]
    nan.xyz[3, 1] = np.nan
    with pytest.raises(M.MphError):
        M.Batch([nan])
    mixed_dim = scenes.dam_break_3d(fluid=(4, 4, 4), box=(8, 6, 8))
    with pytest.raises(ValueError):
        M.Batch([good[0], mixed_dim])


def test_checkpoint_file_round_trip_is_exact_and_rejects_bad_files():
    rng = np.random.default_rng(5)
    sc = scenes.dam_break_3d(fluid=(4, 4, 5), box=(8, 6, 8), seed=2)
    sc.params.wall_center[2][:] = [0.1, 0.2, 0.3]
    n = sc.n
    hdr = M.make_header(n, 0.005, [-0.1] * 3, [0.2] * 3, time=0.123456789012345678)
    ck = M.Checkpoint(sc.params, hdr, 3, 4242, sc.type, rng.permutation(n).astype(np.int32),
                      rng.standard_normal((n, 3)), rng.standard_normal((n, 3)) * 1e-3)
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "state.ckpt")
        M.write_checkpoint_arrays(path, ck)
        got = M.read_checkpoint(path)
        assert got.dim == 3 and got.step == 4242 and got.header.time == hdr.time
        assert got.header.particle_count == n
        for k in ("type", "particle_index", "xyz", "vel"):
            assert np.array_equal(getattr(got, k), getattr(ck, k)), k
        assert list(got.params.wall_center[2]) == [0.1, 0.2, 0.3] and got.params.dt == sc.params.dt
        raw = open(path, "rb").read()
        open(path, "wb").write(raw[:-8])  # truncated
        with pytest.raises(M.MphError) as e:
            M.read_checkpoint(path)
        assert e.value.code == N.MPH_ERR_IO
        open(path, "wb").write(b"NOTACKPT" + raw[8:])  # foreign
        with pytest.raises(M.MphError):
            M.read_checkpoint(path)
        with pytest.raises(M.MphError):
            M.read_checkpoint(os.path.join(td, "missing.ckpt"))


def test_create_rejects_bad_modes_before_any_device_call():
    """mph_create checks its mode before it touches the device: an unknown
    mode, and the cell-walk flag on a form other than the mixed ones."""
    import ctypes as C
    lib = N.load()
    sc = scenes.dam_break_3d(fluid=(6, 5, 7), box=(14, 6, 12))
    t = np.ascontiguousarray(sc.type, np.int32)
    x = np.ascontiguousarray(sc.xyz, np.float64)
    v = np.ascontiguousarray(sc.vel, np.float64)
    for mode in (7, N.MODE_FP64 | N.MIXED_CELL_WALK, N.MODE_LEARNED | N.MIXED_CELL_WALK):
        ctx = C.c_void_p()
        rc = lib.mph_create(C.byref(sc.params), C.byref(sc.header), 3, mode, t.ctypes.data_as(C.POINTER(C.c_int)),
                            x.ctypes.data_as(C.POINTER(C.c_double)), v.ctypes.data_as(C.POINTER(C.c_double)),
                            C.byref(ctx))
        assert rc == N.MPH_ERR_ARG and not ctx.value, mode
