"""The learned form: the edge-MLP tensor-core kernels against the CPU oracle
(oracle/mlp_oracle.py), training, and the learned step with its judge and
fallback against the FP64 form."""
import numpy as np
import pytest

import mphexplicit_b200 as M
from mphexplicit_b200 import learned as LR
from mphexplicit_b200 import scenes
from oracle import mlp_oracle as O
from tests.common import by_original_id, rel_l2

pytestmark = pytest.mark.gpu

# BF16 operands with FP32 accumulation in a different order than the oracle's:
# a few rounding points flip, so outputs and gradients agree to ~1e-3 relative
TOL_OUT = 1e-2
TOL_GRAD = 2e-2


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.parametrize("n", [100, 128 * 3 + 5, 128 * 148 * 2 + 77])
def test_mlp_forward_and_gradient_match_oracle(n):
    m = LR.Model(seed=0)
    p = O.random_params(11)
    m.set_params(p)
    m.set_scales(0.7, 3.0)
    s = O.random_samples(n, n)
    f = m.predict(s)
    assert _rel(f, O.predict_forces(p, s, 0.7, 3.0)) < TOL_OUT
    g, loss = m.gradient(s)
    gr, lr = O.gradient(p, s, 0.7, 3.0)
    assert abs(loss - lr) < TOL_OUT * lr
    for a, b in [(O.OFF_W1, O.OFF_B1), (O.OFF_B1, O.OFF_W2), (O.OFF_W2, O.OFF_B2), (O.OFF_B2, O.OFF_W3),
                 (O.OFF_W3, O.OFF_B3), (O.OFF_B3, O.OFF_W4), (O.OFF_W4, O.OFF_B4), (O.OFF_B4, O.NPARAM)]:
        assert _rel(g[a:b], gr[a:b]) < TOL_GRAD, (a, _rel(g[a:b], gr[a:b]))
    m.close()


@pytest.mark.parametrize("kernel", [0, 1])
def test_bounded_wait_runs_out_and_model_stays_usable(kernel):
    """The training (0) and inference (1) kernels with their MMA groups
    withheld and a wait limit of 64 polls: the mbarrier wait runs out with
    nothing in flight, the kernel sets the error flag and frees its tensor
    memory, the call reports MPH_ERR_DEVICE; the same model then computes the
    same outputs and gradients as before."""
    from mphexplicit_b200 import _native as N
    m = LR.Model(seed=0)
    p = O.random_params(7)
    m.set_params(p)
    m.set_scales(0.7, 3.0)
    s = O.random_samples(300, 5)
    f0 = m.predict(s)
    g0, l0 = m.gradient(s)
    st, msg = m.check_wait(kernel, 64)
    assert st == N.MPH_ERR_DEVICE and "timed out" in msg, (st, msg)
    assert np.array_equal(m.predict(s), f0)
    g1, l1 = m.gradient(s)
    assert np.array_equal(g1, g0) and l1 == l0
    m.close()


def test_mlp_params_round_trip_and_padding():
    m = LR.Model(seed=3)
    p = m.params()
    assert p.size == O.NPARAM
    assert np.all(p[O.OFF_W1:O.OFF_B1].reshape(O.H, O.KIN)[:, O.NIN:] == 0)
    q = O.random_params(5)
    m.set_params(q)
    assert np.array_equal(m.params(), q)
    m.close()


def test_mlp_training_fits_a_viscous_pair_law():
    """Adam on the tensor-core gradient fits f = (u.e) e (1 - r/3.5)^2 / r."""
    rng = np.random.default_rng(0)
    n = 1 << 17
    s = O.random_samples(n, 9, valid_frac=1.0)
    d = s[:, 0:3].astype(np.float64)
    r = np.maximum(np.linalg.norm(d, axis=1), 0.3)
    s[:, 3] = r
    e = d / r[:, None]
    u = s[:, 4:7].astype(np.float64)
    w = np.clip(1.0 - r / 3.5, 0.0, None) ** 2 / r
    f = (np.sum(u * e, axis=1) * w)[:, None] * e
    s[:, 8:11] = f
    ds = LR.Dataset(n)
    ds.append(s)
    m = LR.Model(seed=1)
    m.fit_scales(ds)
    loss0 = m.gradient(s[:8192])[1]
    loss = m.train(ds, epochs=60, batch=1024, lr=2e-3, seed=2)
    assert loss < loss0 / 20, (loss0, loss)
    test = s[rng.choice(n, 4096, replace=False)]
    assert _rel(m.predict(test), test[:, 8:11]) < 0.2
    m.close()
    ds.close()


def _scene():
    # a viscous dam break (mu = 0.05 Pa s) so that the replaced terms matter
    sc = scenes.dam_break_3d(fluid=(16, 12, 24), box=(40, 12, 30), seed=5, mu=0.05)
    return sc


def _run(sc, mode, steps, model=None, judge=10, tol=1e-2):
    s = M.Solver(sc.params, sc.header, sc.type, sc.xyz, sc.vel, dim=sc.dim, mode=mode)
    if model is not None:
        s.set_learned(model, judge, tol)
    s.step(steps)
    st = s.state()
    stats = s.learned_stats() if mode == "learned" else None
    s.close()
    return st, stats


def test_learned_fallback_everywhere_is_the_fp64_step():
    """With a zero tolerance every judgement falls back: the run is the FP64
    step, bit for bit."""
    sc = _scene()
    m = LR.Model(seed=0)
    ref, _ = _run(sc, "fp64", 30)
    got, stats = _run(sc, "learned", 30, m, judge=10, tol=1e-300)
    assert stats["learned_steps"] == 0 and stats["fallbacks"] == 3 and stats["plain_steps"] == 30
    for k in ("xyz", "vel"):
        assert np.array_equal(by_original_id(got, k), by_original_id(ref, k))
    m.close()


def test_untrained_model_falls_back():
    """An untrained network (random weights) on a flowing scene: every judgement
    sees the replaced terms' error far over the tolerance and takes the plain
    step, so the run equals the FP64 step bit for bit."""
    sc = _scene()
    s = M.Solver(sc.params, sc.header, sc.type, sc.xyz, sc.vel, dim=sc.dim, mode="fp64")
    s.step(40)  # into the flow: the replaced (viscous) terms are non-zero
    st = s.state()
    s.close()
    o = np.argsort(st["particle_index"], kind="stable")
    flowing = scenes.Scene(sc.name, sc.dim, sc.params, sc.header, st["type"][o], st["xyz"][o], st["vel"][o], 30)
    m = LR.Model(seed=4)
    ref, _ = _run(flowing, "fp64", 30)
    got, stats = _run(flowing, "learned", 30, m, judge=10, tol=1e-2)
    assert stats["judged"] == 3 and stats["fallbacks"] == 3 and stats["learned_steps"] == 0, stats
    assert stats["last_term_error"] > 1e-2 and stats["max_accepted_error"] == 0.0, stats
    for k in ("xyz", "vel"):
        assert np.array_equal(by_original_id(got, k), by_original_id(ref, k))
    m.close()


def test_learned_step_gains_over_dropping_the_terms():
    """Train on the solver's own FP64 trajectory, then run the learned form:
    its velocities stay closer to the FP64 form than the same step with the
    replaced terms dropped (a zero network), and its judge records the errors."""
    sc = _scene()
    steps = 60
    s = M.Solver(sc.params, sc.header, sc.type, sc.xyz, sc.vel, dim=sc.dim, mode="fp64")
    ds = LR.Dataset(1 << 20)
    for k in range(6):
        s.collect_samples(ds, 1 << 17, seed=k)
        s.step(10)
    ref = s.state()
    s.close()
    samp = ds.read(0, 4096)
    assert np.mean(samp[:, 11]) > 0.5 and np.all(np.isfinite(samp))
    m = LR.Model(seed=0)
    m.fit_scales(ds)
    m.train(ds, epochs=20, batch=4096, lr=2e-3, seed=1)
    got, stats = _run(sc, "learned", steps, m, judge=10, tol=1.0)
    zero = LR.Model(seed=0)
    zero.set_params(np.zeros(O.NPARAM, np.float32))
    zero.set_scales(*m.scales())
    base, _ = _run(sc, "learned", steps, zero, judge=10 ** 6, tol=1e30)
    fl = by_original_id(ref, "type") < 2
    e_learned = rel_l2(by_original_id(got, "vel")[fl], by_original_id(ref, "vel")[fl])
    e_zero = rel_l2(by_original_id(base, "vel")[fl], by_original_id(ref, "vel")[fl])
    assert stats["judged"] == 6 and stats["learned_steps"] == steps
    assert stats["max_term_error"] < 0.5, (stats, e_learned, e_zero)
    assert e_learned < 0.5 * e_zero, (stats, e_learned, e_zero)
    m.close()
    zero.close()
    ds.close()
