"""Mixed-precision forms vs the FP64 form (bit-identical to the reference).

MPH_MODE_MIXED: every pair term in FP32 operations (cell-relative, exact FP32
displacements, Kahan sums; the DensityP terms as double-float pairs of FP32
numbers), FP64 integration.  MPH_MODE_MIXED_P64: the same with the density
sweep's pressure pairs (DensityP, DivergenceP) in FP64.
Errors are relative L2 norms of the fluid velocity against the FP64 form,
matched by ParticleIndex; the tolerances below are the contract of each form.
"""
import numpy as np
import pytest

import mphexplicit_b200 as M
from mphexplicit_b200 import scenes
from tests.common import by_original_id, micro_cases, rel_l2

pytestmark = pytest.mark.gpu

# relative L2 velocity error bounds after the given steps ("_walk": the same
# form with the table-free cell-walk force sweep, MPH_MIXED_CELL_WALK)
TOL = {"mixed": 1e-4, "mixed_p64": 1e-4, "mixed_walk": 1e-4, "mixed_p64_walk": 1e-4}
MODES = list(TOL)


def run(sc, steps, mode):
    s = M.Solver(sc.params, sc.header, sc.type, sc.xyz, sc.vel, dim=sc.dim, mode=mode)
    s.step(steps)
    s.synchronize()
    st = s.state()
    info = s.info()
    cons = s.conserved_sums()
    s.close()
    return st, info, cons


def vel_error(a, b):
    fl = by_original_id(a, "type") < 2
    return rel_l2(by_original_id(b, "vel")[fl], by_original_id(a, "vel")[fl])


CASES = [
    ("droplet_2d", lambda: scenes.droplet_2d(seed=4), 1000),
    ("dam_break", lambda: scenes.dam_break_3d(fluid=(16, 12, 24), box=(40, 12, 30), seed=5), 400),
    ("two_fluid_ratio", lambda: scenes.two_fluid_column(n=12, seed=6), 200),
]


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("name,make,steps", CASES)
def test_mixed_error_against_fp64(name, make, steps, mode):
    sc = make()
    if name == "two_fluid_ratio":
        rng = np.random.default_rng(6)
        for a in range(4):
            for b in range(4):
                sc.params.interaction_ratio[a][b] = float(rng.uniform(0.7, 1.3))
    ref, rinfo, _ = run(sc, steps, "fp64")
    got, ginfo, _ = run(sc, steps, mode)
    err = vel_error(ref, got)
    assert err <= TOL[mode], f"{name} {mode}: relative L2 velocity error {err:.3e}"
    assert rel_l2(by_original_id(got, "xyz"), by_original_id(ref, "xyz")) < 1e-6
    assert abs(ginfo["rebuild_count"] - rinfo["rebuild_count"]) <= 2
    # output fields are filled on read-back and close to the FP64 ones
    assert np.allclose(by_original_id(got, "density_a"), by_original_id(ref, "density_a"), rtol=1e-4, atol=1e-6)
    same = np.mean(by_original_id(got, "neighbor_count") == by_original_id(ref, "neighbor_count"))
    assert same > 0.99


def test_mixed_momentum_free_droplet():
    """No walls, no gravity: total momentum stays at its initial zero."""
    sc = scenes.droplet_2d(seed=8)
    for mode in MODES:
        _, _, cons = run(sc, 500, mode)
        mass = cons[0]
        assert np.all(np.abs(cons[1:3]) < 1e-7 * mass), (mode, cons)


def test_mixed_full_size_dam_break_1000_steps():
    """Benchmark config 2 at full size: both mixed forms stay within 1e-4
    relative L2 velocity error of the FP64 form (bit-identical to the
    reference) after 1000 steps."""
    sc = scenes.dam_break_3d()
    ref, _, _ = run(sc, 1000, "fp64")
    for mode in MODES:
        got, _, _ = run(sc, 1000, mode)
        err = vel_error(ref, got)
        assert err <= 1e-4, (mode, err)


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("k", range(6))
def test_mixed_micro_cases(k, mode):
    """The micro-cases (pairs at every radius, a lone particle, an isolated
    wall, every periodic face, a thin 2-D grid) within the form's tolerance."""
    (name, sc), steps = list(micro_cases())[k]
    ref, rinfo, _ = run(sc, steps, "fp64")
    got, ginfo, _ = run(sc, steps, mode)
    err = vel_error(ref, got)
    assert err <= TOL[mode], f"{name} {mode}: {err:.3e}"
    assert rel_l2(by_original_id(got, "xyz"), by_original_id(ref, "xyz")) < 1e-6
    assert np.array_equal(by_original_id(got, "neighbor_count"), by_original_id(ref, "neighbor_count"))


@pytest.mark.parametrize("name,make,steps", CASES)
def test_cell_walk_matches_table_sweep(name, make, steps):
    """The cell-walk force sweep evaluates the same pair terms as the table
    sweep: after a few steps the two mixed runs agree far inside the form's
    bound (they differ only in FP32 summation order and in which pairs take
    the exact hi/lo displacement)."""
    sc = make()
    a, _, _ = run(sc, 20, "mixed")
    b, _, _ = run(sc, 20, "mixed_walk")
    assert vel_error(a, b) < 1e-5, vel_error(a, b)


@pytest.mark.parametrize("mode", ["mixed", "mixed_p64"])
@pytest.mark.parametrize("name", ["dam_break", "two_fluid_ratio"])
def test_mixed_virial_close_to_fp64(name, mode):
    """mph_compute_virial in the mixed forms (FP32 pair terms over the form's
    own table) against the FP64 virial (bit-identical to the reference) after
    the same steps; surface tension and interaction ratios in the two-fluid
    case."""
    sc = dict((n, m) for n, m, _ in CASES)[name]()
    if name == "two_fluid_ratio":
        rng = np.random.default_rng(6)
        for a in range(4):
            for b in range(4):
                sc.params.interaction_ratio[a][b] = float(rng.uniform(0.7, 1.3))
    out = {}
    for md in ("fp64", mode):
        s = M.Solver(sc.params, sc.header, sc.type, sc.xyz, sc.vel, dim=sc.dim, mode=md)
        s.step(20)
        s.compute_virial()
        out[md] = s.state()
        s.close()
    a = by_original_id(out[mode], "virial_pressure")
    b = by_original_id(out["fp64"], "virial_pressure")
    assert np.any(a != 0.0)
    assert rel_l2(a, b) < 2e-3, rel_l2(a, b)


def test_cli_mixed_vtk_has_the_virial():
    """The drop-in executable in a mixed form writes VirialPressureAtParticle
    computed by the mixed virial (non-zero, close to the FP64 run's)."""
    import os
    import re
    import subprocess
    import tempfile
    from tests.common import GoldenCase
    case = GoldenCase("dam_break_small")
    exe = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "mphexplicit_b200", "bin",
                       "mph_b200")

    def virial_section(path):
        text = open(path).read()
        sec = text.split("SCALARS VirialPressureAtParticle float 1\nLOOKUP_TABLE default\n", 1)[1]
        return np.array(sec.split("\n\n", 1)[0].split(), float)

    got = {}
    with tempfile.TemporaryDirectory() as td:
        text = open(case.data).read()
        for key, val in (("OutputInterval", "1.0"), ("VtkOutputInterval", "1.0e-4"), ("EndTime", "1.5e-4")):
            text = re.sub(r"^%s\s+\S+" % key, "%s %s" % (key, val), text, flags=re.M)
        data = os.path.join(td, "case.data")
        open(data, "w").write(text)
        for mode in ("fp64", "mixed_p64"):
            r = subprocess.run([exe, data, case.grid, "p%03d.prof", mode + "%03d.vtk", "run.log", "1",
                                "--dim=3", "--mode=" + mode], cwd=td, capture_output=True, text=True, timeout=300)
            assert r.returncode == 0, r.stdout + r.stderr
            got[mode] = virial_section(os.path.join(td, mode + "005.vtk"))
    assert np.any(got["mixed_p64"] != 0.0)
    # the two forms sort the particles differently: compare the distributions
    a, b = np.sort(got["mixed_p64"]), np.sort(got["fp64"])
    assert rel_l2(a, b) < 5e-3, rel_l2(a, b)
