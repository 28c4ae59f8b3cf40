"""Batched form (mph_batch_*): many uneven scenes stepped together.

Every scene of a batch takes the reference step with the pair arithmetic of
MPH_MODE_MIXED_P64 (FP64 density pairs, FP32 force pairs) and FP64
integration, so its contract is that form's: relative L2 velocity error
against the FP64 form (bit-identical to the reference) within TOL after the
given steps.  A particle's pair sums run over
its neighbour cells in a fixed order, so a batch is deterministic, a scene's
result does not depend on the other scenes in the batch, and replaying steps
through CUDA graphs or as direct launches gives the same bits.
"""
import numpy as np
import pytest

import mphexplicit_b200 as M
from mphexplicit_b200 import scenes
from oracle import pyoracle as po
from tests.common import by_original_id, micro_cases, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-4  # relative L2 velocity error against the FP64 form (MPH_MODE_MIXED_P64's bound)


def small_droplets(count=6, seed=3):
    return scenes.droplet_batch_2d(count=count, seed=seed, lo=10, hi=26)


def small_dams(count=3, seed=5):
    out = []
    rng = np.random.default_rng(seed)
    for k in range(count):
        fx, fy, fz = (int(v) for v in rng.integers(5, 10, 3))
        out.append(scenes.dam_break_3d(fluid=(fx, fy, fz), box=(fx + 8, fy + 2, fz + 4), seed=seed + k))
    return out


def fp64_state(sc, steps):
    s = M.Solver(sc.params, sc.header, sc.type, sc.xyz, sc.vel, dim=sc.dim, mode="fp64")
    s.step(steps)
    st = s.state()
    s.close()
    return by_original_id(st, "xyz"), by_original_id(st, "vel")


def run_batch(scs, steps, tiles=None, profile=False):
    b = M.Batch(scs, tiles=tiles)
    if profile:
        b.profile(True)
    b.step(steps)
    b.synchronize()
    xyz, vel = b.state()
    info = b.info()
    b.close()
    return xyz, vel, info


def check_against_fp64(scs, steps, xyz, vel, offsets):
    for k, sc in enumerate(scs):
        a, e = int(offsets[k]), int(offsets[k + 1])
        rx, rv = fp64_state(sc, steps)
        fl = sc.type < 2
        err = rel_l2(vel[a:e][fl], rv[fl])
        assert err <= TOL, f"scene {k}: relative L2 velocity error {err:.3e}"
        assert rel_l2(xyz[a:e], rx) < 1e-6


def offsets_of(scs):
    return np.concatenate([[0], np.cumsum([sc.n for sc in scs])])


def test_batch_droplets_2d_against_fp64():
    scs = small_droplets()
    steps = 300
    xyz, vel, info = run_batch(scs, steps)
    assert info["steps"] == steps and info["scenes"] == len(scs)
    check_against_fp64(scs, steps, xyz, vel, offsets_of(scs))


def test_batch_dam_breaks_3d_against_fp64():
    scs = small_dams()
    steps = 200
    xyz, vel, info = run_batch(scs, steps)
    assert info["scene_rebuilds"] >= 0
    check_against_fp64(scs, steps, xyz, vel, offsets_of(scs))


def test_batch_against_oracle():
    """One scene straight against the CPU oracle (the reference restated)."""
    sc = scenes.droplet_batch_2d(count=1, seed=11, lo=12, hi=16)[0]
    steps = 200
    xyz, vel, _ = run_batch([sc], steps)
    o = po.Oracle.from_scene(sc)
    o.step(steps)
    st = o.state()
    rv = by_original_id(st, "vel")
    assert rel_l2(vel, rv) <= TOL
    assert rel_l2(xyz, by_original_id(st, "xyz")) < 1e-6


def test_batch_deterministic_and_independent_of_other_scenes():
    scs = small_droplets(count=5, seed=7)
    off = offsets_of(scs)
    x1, v1, _ = run_batch(scs, 120)
    x2, v2, _ = run_batch(scs, 120)
    assert np.array_equal(x1, x2) and np.array_equal(v1, v2)
    xs, vs, _ = run_batch([scs[3]], 120)
    assert np.array_equal(xs, x1[off[3]:off[4]]) and np.array_equal(vs, v1[off[3]:off[4]])


def test_batch_graph_replay_equals_direct_launches():
    scs = small_droplets(count=4, seed=9)
    steps = 2 * M._native.BATCH_GRAPH_STEPS + 5
    xg, vg, _ = run_batch(scs, steps)
    xd, vd, _ = run_batch(scs, steps, profile=True)
    assert np.array_equal(xg, xd) and np.array_equal(vg, vd)


def test_batch_tile_shapes_agree():
    """Other tile shapes and CTA sizes give the same flow within FP32 rounding."""
    scs = small_droplets(count=4, seed=13)
    steps = 100
    xr, vr, _ = run_batch(scs, steps, tiles=(8, 8, 1, 256))
    fl = np.concatenate([sc.type for sc in scs]) < 2
    for tiles in [(4, 4, 1, 128), (16, 8, 1, 256), (64, 64, 1, 256)]:
        x, v, info = run_batch(scs, steps, tiles=tiles)
        assert rel_l2(v[fl], vr[fl]) < 1e-4, tiles
        assert rel_l2(x, xr) < 1e-8, tiles


def test_batch_tiles_larger_than_shared_memory_are_split():
    """A 64x64-cell tile of ~100x100-particle droplets does not fit in shared
    memory: the sweeps split it on the device and the flow is unchanged."""
    scs = scenes.droplet_batch_2d(count=2, seed=19, lo=90, hi=100)
    steps = 60
    xr, vr, _ = run_batch(scs, steps, tiles=(8, 8, 1, 256))
    x, v, info = run_batch(scs, steps, tiles=(64, 64, 1, 256))
    assert info["tile_splits"] > 0
    assert info["capacity"] < max(sc.n for sc in scs)
    fl = np.concatenate([sc.type for sc in scs]) < 2
    assert rel_l2(v[fl], vr[fl]) < 1e-4
    assert rel_l2(x, xr) < 1e-8


def test_batch_autotune_keeps_state_and_picks_a_timed_shape():
    scs = small_droplets(count=6, seed=17)
    b = M.Batch(scs)
    b.step(20)
    x0, v0 = b.state()
    trials = b.autotune(steps=16)
    assert len(trials) >= 4 and all(t["ms_per_step"] > 0 for t in trials)
    x1, v1 = b.state()
    assert np.array_equal(x0, x1) and np.array_equal(v0, v1)
    info = b.info()
    best = min(trials, key=lambda t: t["ms_per_step"])
    assert tuple(info["tile"][:2]) == tuple(best["tile"][:2]) and info["threads"] == best["threads"]
    assert info["ctas_per_sm"] == best["ctas_per_sm"] and info["capacity"] == best["capacity"]
    assert info["steps"] == 20
    b.step(30)
    xa, va = b.state()
    b.close()
    # the same steps without the autotuner: default shape, then the chosen one
    c = M.Batch(scs)
    c.step(20)
    c.set_tiles(best["tile"][0], best["tile"][1], best["tile"][2], best["threads"], best["ctas_per_sm"])
    c.step(30)
    xb, vb = c.state()
    c.close()
    assert np.array_equal(xa, xb) and np.array_equal(va, vb)


def test_batch_momentum_free_droplets():
    """No walls, no gravity: every droplet keeps zero total momentum."""
    scs = small_droplets(count=4, seed=21)
    xyz, vel, _ = run_batch(scs, 300)
    off = offsets_of(scs)
    for k, sc in enumerate(scs):
        v = vel[off[k]:off[k + 1]]
        mom = np.abs(v.sum(axis=0)) * sc.params.density[0]
        assert np.all(mom < 1e-8 * np.abs(v).sum() * sc.params.density[0] + 1e-12), (k, mom)


@pytest.mark.parametrize("dim", [2, 3])
def test_batch_micro_cases_against_fp64(dim):
    """The micro-cases of one dimension as one batch: lone particles, an
    isolated wall, pairs across every periodic face and at every radius."""
    cases = [(sc, steps) for (name, sc), steps in micro_cases() if sc.dim == dim]
    steps = min(st for _, st in cases)
    scs = [sc for sc, _ in cases]
    xyz, vel, _ = run_batch(scs, steps)
    off = offsets_of(scs)
    for k, sc in enumerate(scs):
        rx, rv = fp64_state(sc, steps)
        a, e = int(off[k]), int(off[k + 1])
        fl = sc.type < 2
        err = rel_l2(vel[a:e][fl], rv[fl])
        assert err <= TOL, (sc.name, err)
        assert rel_l2(xyz[a:e], rx) < 1e-6, sc.name
