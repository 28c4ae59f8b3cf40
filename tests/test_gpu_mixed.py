"""Mixed-precision forms vs the FP64 form (bit-identical to the reference).

MPH_MODE_MIXED: every pair term in FP32 (cell-relative, exact FP32
displacements, Kahan sums), FP64 integration.  MPH_MODE_MIXED_P64: the same with
the density sweep's pressure pairs (DensityP, DivergenceP) in FP64.
Errors are relative L2 norms of the fluid velocity against the FP64 form,
matched by ParticleIndex; the tolerances below are the contract of each form.
"""
import numpy as np
import pytest

import mphexplicit_b200 as M
from mphexplicit_b200 import scenes
from tests.common import by_original_id, micro_cases, rel_l2

pytestmark = pytest.mark.gpu

# relative L2 velocity error bounds after the given steps
TOL = {"mixed": 2e-3, "mixed_p64": 1e-4}


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


@pytest.mark.parametrize("mode", ["mixed", "mixed_p64"])
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
    for mode in ("mixed", "mixed_p64"):
        _, _, cons = run(sc, 500, mode)
        mass = cons[0]
        assert np.all(np.abs(cons[1:3]) < 1e-7 * mass), (mode, cons)


def test_mixed_p64_full_size_dam_break_1000_steps():
    """Benchmark config 2 at full size: the FP64-pressure-core mixed form stays
    within 1e-4 relative L2 velocity error of the FP64 form after 1000 steps."""
    sc = scenes.dam_break_3d()
    ref, _, _ = run(sc, 1000, "fp64")
    got, _, _ = run(sc, 1000, "mixed_p64")
    err = vel_error(ref, got)
    assert err <= 1e-4, err


@pytest.mark.parametrize("mode", ["mixed", "mixed_p64"])
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
