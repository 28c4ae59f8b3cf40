"""CUDA FP64 form vs the reference, through the C ABI (needs a B200).

The FP64 form keeps the reference's operation order, its bitonic cell sort and
its neighbour-list order, so every comparison here is bit-exact:
  * golden fixtures: the reference's own arrays after k steps;
  * fresh seeded scenes: the CPU oracle (itself pinned to the reference);
  * output files: byte-identical *.vtk / *.prof text;
  * full-size benchmark scene (2.78 M particles): two steps against the oracle.
"""
import os
import tempfile

import numpy as np
import pytest

import mphexplicit_b200 as M
from mphexplicit_b200 import _native as N
from mphexplicit_b200 import scenes
from oracle import pyoracle as po
from tests.common import (CASES, CELL_KEYS, FIELD_KEYS, LONG_CASES, STATE_KEYS, GoldenCase, assert_same, csr_digests,
                          micro_cases)

pytestmark = pytest.mark.gpu


def solver_for(case: GoldenCase, mode="fp64", layout="auto") -> M.Solver:
    s = M.Solver.from_files(case.data, case.grid, dim=case.dim, mode=mode)
    if layout != "auto":
        s.set_sweep_layout(layout)
    return s


# The golden cases are small: "auto" runs the warp-per-particle sweeps on
# them, "thread" the thread-per-particle ones the large scenes use.
@pytest.mark.parametrize("layout", ["auto", "thread"])
@pytest.mark.parametrize("name", CASES)
def test_fp64_matches_reference_golden(name, layout):
    case = GoldenCase(name)
    s = solver_for(case, layout=layout)
    s.step(case.steps)
    s.synchronize()
    s.compute_virial()
    st, f, c = s.state(), s.fields(), s.cells()
    for k in STATE_KEYS:
        assert_same(st[k], case.ref[k], k)
    for k in FIELD_KEYS:
        if k == "gravity_center" and not any(s.params.surface_tension[t] for t in range(4)):
            continue  # not computed without surface tension (every term is zero then)
        assert_same(f[k], case.ref[k], k)
    for k in CELL_KEYS:
        assert_same(c[k], case.ref[k], k)
    ptr, ind = s.neighbors()
    assert_same(ptr, case.ref["nptr"], "NeighborPtr")
    assert_same(ind, case.ref["nind"], "NeighborInd")
    info = s.info()
    assert info["rebuild_count"] == case.rebuilds
    assert info["neighbor_ind_count"] == case.neighbor_ind_count
    assert info["time"] == float(case.ref["time"])
    s.close()


@pytest.mark.parametrize("layout", ["auto", "thread"])
@pytest.mark.parametrize("name", LONG_CASES)
def test_fp64_matches_reference_golden_1000_steps(name, layout):
    """3-D, 1000 steps from inside the developed flow (dozens of neighbour
    rebuilds), against the reference's own arrays: bit for bit (stricter than
    the 1e-10 relative bound on the FP64 state)."""
    case = GoldenCase(name)
    s = solver_for(case, layout=layout)
    s.step(case.steps)
    s.synchronize()
    s.compute_virial()
    st, f, c = s.state(), s.fields(), s.cells()
    for k in STATE_KEYS:
        assert_same(st[k], case.ref[k], k)
    for k in FIELD_KEYS:
        if k == "gravity_center" and not any(s.params.surface_tension[t] for t in range(4)):
            continue
        assert_same(f[k], case.ref[k], k)
    for k in CELL_KEYS:
        assert_same(c[k], case.ref[k], k)
    ptr, ind = s.neighbors()
    dp, di = csr_digests(ptr, ind)
    assert dp == str(case.ref["nptr_sha256"]), "NeighborPtr differs"
    assert di == str(case.ref["nind_sha256"]), "NeighborInd differs"
    info = s.info()
    assert info["rebuild_count"] == case.rebuilds and case.rebuilds >= (30 if name == "dam_break_1000" else 5)
    assert info["neighbor_ind_count"] == case.neighbor_ind_count
    assert info["time"] == float(case.ref["time"])
    s.close()


def test_startup_matches_oracle():
    case = GoldenCase("bridge")
    p = M.read_data_file(case.data)
    g = M.read_grid_file(case.grid)
    o = po.Oracle(p, g.header, g.type, g.xyz, g.vel, 2)
    s = M.Solver(p, g.header, g.type, g.xyz, g.vel, dim=2)
    a, b = s.state(), o.state()
    for k in ["particle_index", "type", "xyz", "vel", "neighbor_count", "density_a", "vol_strain_p"]:
        assert_same(a[k], b[k], k)
    for k in CELL_KEYS:
        assert_same(s.cells()[k], o.cells()[k], k)
    assert_same(s.fields()["gravity_center"], o.fields()["gravity_center"], "gc")


def _fresh():
    yield scenes.droplet_2d(n=24, seed=21, steps=60), 60, {}
    yield scenes.dam_break_3d(fluid=(16, 12, 24), box=(40, 12, 30), walls=3, seed=22), 30, {}
    sc = scenes.two_fluid_column(n=14, seed=23, steps=40)
    yield sc, 25, {"ratio": True}
    sc = scenes.dam_break_3d(fluid=(10, 6, 10), box=(24, 6, 16), walls=2, seed=24)
    sc.params.wall_omega[2][1] = 0.4
    sc.params.wall_velocity[2][0] = 0.03
    sc.params.wall_center[2][2] = 0.02
    yield sc, 30, {}


@pytest.mark.parametrize("k", range(4))
def test_fp64_matches_oracle_fresh(k):
    sc, steps, opt = list(_fresh())[k]
    if opt.get("ratio"):
        rng = np.random.default_rng(k)
        for a in range(4):
            for b in range(4):
                sc.params.interaction_ratio[a][b] = float(rng.uniform(0.6, 1.4))
    o = po.Oracle.from_scene(sc)
    s = M.Solver(sc.params, sc.header, sc.type, sc.xyz, sc.vel, dim=sc.dim)
    o.step(steps)
    s.step(steps)
    o.virial()
    s.compute_virial()
    a, b = s.state(), o.state()
    for key in STATE_KEYS:
        assert_same(a[key], b[key], f"{sc.name}:{key}")
    assert s.info()["rebuild_count"] == o.rebuilds


@pytest.mark.parametrize("k", range(6))
def test_fp64_matches_oracle_micro(k):
    """Pairs at every kernel radius, a lone particle, a wall out of every fluid
    particle's reach, motion and interaction across all periodic faces, a
    thin 2-D grid: bit-exact against the oracle (pinned to the reference on
    the same cases)."""
    (name, sc), steps = list(micro_cases())[k]
    o = po.Oracle.from_scene(sc)
    s = M.Solver(sc.params, sc.header, sc.type, sc.xyz, sc.vel, dim=sc.dim)
    o.step(steps)
    s.step(steps)
    o.virial()
    s.compute_virial()
    a, b = s.state(), o.state()
    for key in STATE_KEYS:
        assert_same(a[key], b[key], f"{name}:{key}")
    assert s.info()["rebuild_count"] == o.rebuilds
    s.close()


@pytest.mark.parametrize("name", ["square_drop_skip", "dam_break_small"])
def test_output_files_match_reference_bytes(name):
    case = GoldenCase(name)
    s = solver_for(case)
    s.step(case.steps)
    s.compute_virial()
    with tempfile.TemporaryDirectory() as td:
        vtk, prof = os.path.join(td, "a.vtk"), os.path.join(td, "a.prof")
        s.write_vtk(vtk)
        s.write_prof(prof)
        assert open(vtk, "rb").read() == case.reference_bytes("vtk")
        assert open(prof, "rb").read() == case.reference_bytes("prof")


def test_state_round_trip_and_step_continuity():
    """get_state -> set_state leaves the trajectory unchanged (host-resident use)."""
    sc = scenes.dam_break_3d(fluid=(8, 8, 12), box=(20, 8, 16), seed=5)
    a = M.Solver(sc.params, sc.header, sc.type, sc.xyz, sc.vel, dim=3)
    b = M.Solver(sc.params, sc.header, sc.type, sc.xyz, sc.vel, dim=3)
    x = np.zeros((sc.n, 3))
    v = np.zeros((sc.n, 3))
    for _ in range(20):
        a.step(1)
        a.get_xv(x, v)
        a.set_state(x, v)
        b.step(1)
    for key in STATE_KEYS:
        assert_same(a.state()[key], b.state()[key], key)


def _host_xv(n, pinned):
    if not pinned:
        return np.zeros((n, 3)), np.zeros((n, 3))
    import torch
    return (torch.zeros((n, 3), dtype=torch.float64, pin_memory=True).numpy(),
            torch.zeros((n, 3), dtype=torch.float64, pin_memory=True).numpy())


@pytest.mark.parametrize("name,pinned", [("dam_break_small", True), ("two_fluid_small", True),
                                         ("moving_walls", False), ("droplet_2d", True)])
def test_step_read_state_is_step_then_get_state(name, pinned):
    """The overlapped step-and-read (force sweep in ranges on two streams, the
    copies behind it) returns the bits of step + get_state, and a host loop of
    step_read_state + set_state stays on the reference's trajectory."""
    case = GoldenCase(name)
    a, b = solver_for(case), solver_for(case)
    x, v = _host_xv(a.n, pinned)
    xb, vb = np.zeros((b.n, 3)), np.zeros((b.n, 3))
    done, m = 0, 1
    while done < case.steps:
        m = min(m, case.steps - done)
        a.step_read_state(m, x, v)
        b.step(m)
        b.get_xv(xb, vb)
        assert_same(x, xb, "xyz")
        assert_same(v, vb, "vel")
        a.set_state(x, v)
        done += m
        m = m * 2 + 1
    a.synchronize()
    a.compute_virial()
    st = a.state()
    for key in STATE_KEYS:
        assert_same(st[key], case.ref[key], key)


def test_step_read_state_mixed_form():
    """The mixed form has no overlapped path: it steps, then copies."""
    case = GoldenCase("dam_break_small")
    a, b = solver_for(case, "mixed"), solver_for(case, "mixed")
    x, v = _host_xv(a.n, True)
    xb, vb = np.zeros((b.n, 3)), np.zeros((b.n, 3))
    for m in (1, 4):
        a.step_read_state(m, x, v)
        b.step(m)
        b.get_xv(xb, vb)
        assert_same(x, xb, "xyz")
        assert_same(v, vb, "vel")


def test_checkpoint_restart_is_the_reference_restart_exactly():
    """A checkpoint keeps the state in the order of the *.prof file of that
    time with the wall centres reached; restarting from it equals the
    reference (oracle) restarted from the same state, bit for bit, and the
    file maps every particle back to its original id."""
    case = GoldenCase("moving_walls")
    s = solver_for(case)
    s.step(37)
    before = s.state()
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "run.ckpt")
        s.write_checkpoint(path)
        ck = M.read_checkpoint(path)
        r = M.Solver.from_checkpoint(path)
    assert ck.step == 37 and ck.header.time == s.info()["time"]
    assert np.array_equal(ck.particle_index, before["particle_index"])
    assert np.array_equal(ck.xyz, before["xyz"]) and np.array_equal(ck.vel, before["vel"])
    assert any(ck.params.wall_center[t][k] != s.params.wall_center[t][k] for t in (2, 3) for k in range(3))
    o = po.Oracle(ck.params, ck.header, ck.type, ck.xyz, ck.vel, ck.dim)
    r.step(25)
    o.step(25)
    got, ref = r.state(), o.state()
    for key in STATE_KEYS:
        assert_same(got[key], ref[key], key)
    r.close()
    s.close()


def test_nonfinite_state_is_reported_not_trapped():
    """A NaN velocity injected from the host is caught by the device-side
    finiteness flag and returned as MPH_ERR_NONFINITE; the context stays usable."""
    sc = scenes.droplet_2d(n=12, seed=3)
    s = M.Solver(sc.params, sc.header, sc.type, sc.xyz, sc.vel, dim=2)
    st = s.state()
    v = st["vel"].copy()
    v[5, 0] = np.nan
    s.set_state(st["xyz"], v)
    with pytest.raises(M.MphError) as e:
        s.step(2)
        s.synchronize()
    assert e.value.code == N.MPH_ERR_NONFINITE
    s.close()
    t = M.Solver(sc.params, sc.header, sc.type, sc.xyz, sc.vel, dim=2)  # device still fine
    t.step(3)
    t.synchronize()


def test_neighbor_table_grows_on_compression():
    """Squeezing particles closer than the lattice spacing makes lists longer
    than the initial table; the build grows it and stays exact."""
    sc = scenes.droplet_2d(n=20, seed=9)
    c = sc.xyz.mean(axis=0)
    sc.xyz[:] = c + (sc.xyz - c) * 0.6
    o = po.Oracle.from_scene(sc)
    s = M.Solver(sc.params, sc.header, sc.type, sc.xyz, sc.vel, dim=2)
    assert s.info()["max_neighbor_count"] > 100
    assert_same(s.state()["neighbor_count"], o.state()["neighbor_count"], "ncount")
    p1, i1 = s.neighbors()
    p2, i2 = o.neighbors()
    assert_same(i1, i2, "nind")


INFO_KEYS = ("step", "rebuild_count", "time", "max_neighbor_count", "neighbor_capacity")


@pytest.mark.parametrize("name", ["dam_break_small", "two_fluid_small", "moving_walls", "droplet_2d", "bridge"])
def test_step_graphs_match_host_path(name):
    """With mph_set_step_graphs, several FP64 steps per mph_step run as graph
    launches whose conditional nodes take the rebuild test on the device; the
    host path (one flag read per step) gives the same bits, rebuilds, step
    count and time."""
    case = GoldenCase(name)
    a, b = solver_for(case), solver_for(case)
    a.set_step_graphs(True)
    b.set_step_graphs(False)
    done = 0
    for m in (1, 2, 7, 13, case.steps):
        m = min(m, case.steps - done)
        if m <= 0:
            break
        a.step(m)
        b.step(m)
        done += m
    a.synchronize()
    b.synchronize()
    ia, ib = a.info(), b.info()
    for k in INFO_KEYS:
        assert ia[k] == ib[k], (k, ia[k], ib[k])
    if name in ("dam_break_small", "moving_walls"):
        assert ia["rebuild_count"] > 0
    sa, sb = a.state(), b.state()
    for key in STATE_KEYS:
        if key != "virial_pressure":
            assert_same(sa[key], sb[key], key)
    fa, fb = a.fields(), b.fields()
    for key in FIELD_KEYS:
        assert_same(fa[key], fb[key], key)


def test_step_graphs_grow_the_table_mid_batch():
    """A list that outgrows its table inside a batch of graph launches stops
    the batch after that step's reorder; the host grows the table, builds the
    list again and finishes the steps: the same bits as the host path."""
    sc = scenes.droplet_2d(n=20, seed=9)
    a = M.Solver(sc.params, sc.header, sc.type, sc.xyz, sc.vel, dim=2)
    b = M.Solver(sc.params, sc.header, sc.type, sc.xyz, sc.vel, dim=2)
    a.set_step_graphs(True)
    b.set_step_graphs(False)
    cap0 = a.info()["neighbor_capacity"]
    for s in (a, b):
        st = s.state()
        c = st["xyz"].mean(axis=0)
        s.set_state(c + (st["xyz"] - c) * 0.6, st["vel"])
        s.step(6)
        s.synchronize()
    ia, ib = a.info(), b.info()
    assert ia["neighbor_capacity"] > cap0
    for k in INFO_KEYS:
        assert ia[k] == ib[k], (k, ia[k], ib[k])
    sa, sb = a.state(), b.state()
    for key in STATE_KEYS:
        if key != "virial_pressure":
            assert_same(sa[key], sb[key], key)


def test_full_size_dam_break_two_steps():
    """Benchmark config 2 at full size (2.0 M fluid + 0.78 M wall): two steps,
    bit-exact against the oracle, and the expected interior neighbour count."""
    sc = scenes.dam_break_3d()
    assert sc.n == 2_779_256
    s = M.Solver(sc.params, sc.header, sc.type, sc.xyz, sc.vel, dim=3)
    s.step(2)
    a = s.state()
    o = po.Oracle.from_scene(sc)
    o.step(2)
    b = o.state()
    for key in ["particle_index", "type", "xyz", "vel", "neighbor_count", "density_a", "vol_strain_p", "force"]:
        assert_same(a[key], b[key], key)
    fluid = a["type"] < 2
    assert np.median(a["neighbor_count"][fluid]) >= 180


def test_exact_division_matches_hardware_ieee():
    """The FP64 kernels divide with div_rn (Markstein's method on a correctly
    rounded reciprocal); it must equal the hardware IEEE quotient bit for bit."""
    import ctypes as C
    lib = N.load()
    mism = C.c_longlong(-1)
    first = (C.c_double * 2)()
    assert lib.mph_check_exact_division(10_000_000_000, 12345, C.byref(mism), first) == 0
    assert mism.value == 0, (mism.value, first[0], first[1])
