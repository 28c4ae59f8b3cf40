"""The CPU oracle of the edge MLP (oracle/mlp_oracle.py) against finite
differences, so that it can check the tensor-core kernels' gradients."""
import numpy as np

from oracle import mlp_oracle as O


def test_fp64_gradient_matches_finite_differences():
    p = O.random_params(1).astype(np.float64)
    s = O.random_samples(24, 2)
    g, loss = O.gradient(p, s, 0.5, 2.0, bf16_on=False)
    rng = np.random.default_rng(3)
    real = [k for k in range(O.NPARAM) if g[k] != 0.0]
    for k in rng.choice(real, 40, replace=False):
        h = 1e-6 * max(1.0, abs(p[k]))
        pp, pm = p.copy(), p.copy()
        pp[k] += h
        pm[k] -= h
        fd = (O.gradient(pp, s, 0.5, 2.0, False)[1] - O.gradient(pm, s, 0.5, 2.0, False)[1]) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(g[k])) + 1e-9, (k, fd, g[k])


def test_bf16_rounding_points_stay_close_to_fp64():
    p = O.random_params(4)
    s = O.random_samples(512, 5)
    g64, l64 = O.gradient(p, s, 0.5, 2.0, bf16_on=False)
    g16, l16 = O.gradient(p, s, 0.5, 2.0, bf16_on=True)
    assert abs(l16 - l64) < 2e-2 * l64
    assert np.linalg.norm(g16 - g64) < 3e-2 * np.linalg.norm(g64)


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.0e-5, 65504.0], np.float32)
    b = O.bf16(x)
    assert b[0] == 1.0 and b[1] == 1.0  # halfway to 1.0078125 ties to even (1.0)
    assert b[2] == np.float32(1.0078125)
    assert np.all(np.abs(b - x) <= np.abs(x) * 2.0 ** -8)


def test_padding_parameters_have_no_gradient():
    p = O.random_params(6)
    g, _ = O.gradient(p, O.random_samples(64, 7), 1.0, 1.0)
    assert np.all(g[O.OFF_W1:O.OFF_B1].reshape(O.H, O.KIN)[:, O.NIN:] == 0)
    assert np.all(g[O.OFF_W4:O.OFF_B4].reshape(O.KOUT, O.H)[O.NOUT:] == 0)
    assert np.all(g[O.OFF_B4 + O.NOUT:] == 0)
