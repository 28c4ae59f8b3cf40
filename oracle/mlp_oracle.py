"""CPU oracle of the learned form's edge MLP (test infrastructure only: used
by tests/ to check the tensor-core kernels of csrc/k_mlp.cu; never by the
library).

The network has no reference counterpart (the reference has no learned
terms); this is a restatement of the same arithmetic in numpy.  `forward` /
`gradient` with bf16=True round to BF16 where the kernels do (inputs,
weights, Z = pre-activation, H = SiLU(Z) at the rounding points of the
kernels' packed form, dY, dZ) and accumulate in FP64 (the
kernels accumulate in FP32 on the tensor cores); with bf16=False everything is
FP64, which `tests/` checks against finite differences.

Parameter vector (FP32): W1[128][16], b1[128], W2[128][128], b2, W3[128][128],
b3, W4[16][128], b4[16]; input columns >= 9 and output rows >= 3 are padding.
Sample: 12 floats (dx, dy, dz, r)/l0, (ux, uy, uz, type_i + 4 type_j),
(fx, fy, fz, valid).
"""
from __future__ import annotations

import numpy as np

H, KIN, KOUT, NIN, NOUT = 128, 16, 16, 9, 3
OFF_W1 = 0
OFF_B1 = OFF_W1 + H * KIN
OFF_W2 = OFF_B1 + H
OFF_B2 = OFF_W2 + H * H
OFF_W3 = OFF_B2 + H
OFF_B3 = OFF_W3 + H * H
OFF_W4 = OFF_B3 + H
OFF_B4 = OFF_W4 + KOUT * H
NPARAM = OFF_B4 + KOUT


def bf16(x) -> np.ndarray:
    """Round FP32 values to BF16 (nearest, ties to even), returned as FP32."""
    a = np.ascontiguousarray(np.asarray(x, np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).reshape(a.shape)


def unpack(p: np.ndarray) -> dict:
    p = np.asarray(p, np.float64)
    return {"W1": p[OFF_W1:OFF_B1].reshape(H, KIN), "b1": p[OFF_B1:OFF_W2],
            "W2": p[OFF_W2:OFF_B2].reshape(H, H), "b2": p[OFF_B2:OFF_W3],
            "W3": p[OFF_W3:OFF_B3].reshape(H, H), "b3": p[OFF_B3:OFF_W4],
            "W4": p[OFF_W4:OFF_B4].reshape(KOUT, H), "b4": p[OFF_B4:NPARAM]}


def pack(d: dict) -> np.ndarray:
    return np.concatenate([d["W1"].ravel(), d["b1"], d["W2"].ravel(), d["b2"], d["W3"].ravel(), d["b3"],
                           d["W4"].ravel(), d["b4"]]).astype(np.float64)


def features(samples: np.ndarray, velocity_scale: float, force_scale: float):
    """Scaled inputs [n, 16], scaled targets [n, 3], valid mask [n]."""
    s = np.asarray(samples, np.float32).reshape(-1, 12)
    n = len(s)
    x = np.zeros((n, KIN), np.float32)
    inv_u = np.float32(1.0 / velocity_scale)
    inv_f = np.float32(1.0 / force_scale)
    x[:, 0:3] = s[:, 0:3]
    x[:, 3:6] = s[:, 4:7] * inv_u
    x[:, 6] = s[:, 3]
    tt = s[:, 7].astype(np.int64)
    x[:, 7] = (tt & 3).astype(np.float32)
    x[:, 8] = (tt >> 2).astype(np.float32)
    valid = s[:, 11] != 0
    x[~valid] = 0.0
    t = s[:, 8:11] * inv_f
    return x, t.astype(np.float32), valid


def _silu(z):
    return z / (1.0 + np.exp(-z))


def _dsilu(z):
    sg = 1.0 / (1.0 + np.exp(-z))
    return sg * (1.0 + z * (1.0 - sg))


def _silu_bf16x2(z):
    """SiLU with the rounding points of the kernels' packed BF16 form (z is
    already BF16): hz = z/2 (exact), t = bf16(tanh(hz)), h = bf16(hz + hz t)."""
    hz = 0.5 * z
    t = bf16(np.tanh(hz).astype(np.float32)).astype(np.float64)
    return bf16((hz + hz * t).astype(np.float32)).astype(np.float64)


def _round(a, on):
    return bf16(a).astype(np.float64) if on else np.asarray(a, np.float64)


def forward(params, samples, velocity_scale=1.0, force_scale=1.0, bf16_on=True):
    """Scaled outputs [n, 3] and the intermediates for `gradient`."""
    P = unpack(params)
    x, t, valid = features(samples, velocity_scale, force_scale)
    r = lambda a: _round(a, bf16_on)  # noqa: E731
    X = r(x)
    Wb = {k: (r(P[k].astype(np.float32)) if bf16_on else P[k]) for k in ("W1", "W2", "W3", "W4")}
    Z, Hs = [], [X]
    h = X
    for W, b in (("W1", "b1"), ("W2", "b2"), ("W3", "b3")):
        z = r((h @ Wb[W].T + P[b]).astype(np.float32) if bf16_on else h @ Wb[W].T + P[b])
        h = _silu_bf16x2(z) if bf16_on else _silu(z)
        Z.append(z)
        Hs.append(h)
    y = (h @ Wb["W4"].T + P["b4"])[:, :NOUT]
    return y, {"X": X, "Z": Z, "H": Hs, "Wb": Wb, "t": t.astype(np.float64), "valid": valid}


def gradient(params, samples, velocity_scale=1.0, force_scale=1.0, bf16_on=True):
    """(gradient [NPARAM], loss) of mean((y - t)^2) over valid samples x 3
    (n counts every sample, as in the kernels)."""
    y, c = forward(params, samples, velocity_scale, force_scale, bf16_on)
    n = len(y)
    r = (lambda a: bf16(np.asarray(a, np.float32)).astype(np.float64)) if bf16_on else (lambda a: a)
    dy = np.where(c["valid"][:, None], y - c["t"], 0.0)
    if bf16_on:
        dy = dy.astype(np.float32).astype(np.float64)
    loss = float((dy * dy).sum() / (3.0 * n))
    dyp = np.zeros((n, KOUT))
    dyp[:, :NOUT] = dy
    dyb = r(dyp)
    Wb, Z, Hs = c["Wb"], c["Z"], c["H"]
    g = {}
    g["W4"] = dyb.T @ Hs[3]
    g["b4"] = dyp.sum(0)
    dh = dyb @ Wb["W4"]
    for layer in (3, 2, 1):
        z = Z[layer - 1]
        dz = r(dh * _dsilu(z)) if bf16_on else dh * _dsilu(z)
        g["W%d" % layer] = dz.T @ Hs[layer - 1]
        g["b%d" % layer] = dz.sum(0)
        if layer > 1:
            dh = dz @ Wb["W%d" % layer]
    scale = 2.0 / (3.0 * n)
    out = pack({k: v * scale for k, v in g.items()})
    # padding parameters carry no gradient
    out[OFF_W1:OFF_B1].reshape(H, KIN)[:, NIN:] = 0.0
    out[OFF_W4:OFF_B4].reshape(KOUT, H)[NOUT:, :] = 0.0
    out[OFF_B4 + NOUT:] = 0.0
    return out, loss


def predict_forces(params, samples, velocity_scale, force_scale, bf16_on=True) -> np.ndarray:
    """Pair forces in N (zero for invalid samples)."""
    y, c = forward(params, samples, velocity_scale, force_scale, bf16_on)
    return np.where(c["valid"][:, None], y * force_scale, 0.0)


def random_params(seed: int, gain: float = 1.0) -> np.ndarray:
    """Parameters with variance ~1/fan_in and zero padding."""
    rng = np.random.default_rng(seed)
    d = {"W1": rng.uniform(-1, 1, (H, KIN)) * np.sqrt(3.0 / NIN) * gain,
         "W2": rng.uniform(-1, 1, (H, H)) * np.sqrt(3.0 / H) * gain,
         "W3": rng.uniform(-1, 1, (H, H)) * np.sqrt(3.0 / H) * gain,
         "W4": rng.uniform(-1, 1, (KOUT, H)) * np.sqrt(3.0 / H) * 0.5 * gain,
         "b1": rng.uniform(-0.1, 0.1, H), "b2": rng.uniform(-0.1, 0.1, H), "b3": rng.uniform(-0.1, 0.1, H),
         "b4": rng.uniform(-0.1, 0.1, KOUT)}
    d["W1"][:, NIN:] = 0.0
    d["W4"][NOUT:, :] = 0.0
    d["b4"][NOUT:] = 0.0
    return pack(d).astype(np.float32)


def random_samples(n: int, seed: int, valid_frac: float = 0.9) -> np.ndarray:
    """Samples with pair-like inputs and targets of order one."""
    rng = np.random.default_rng(seed)
    s = np.zeros((n, 12), np.float32)
    d = rng.normal(0, 1.5, (n, 3))
    s[:, 0:3] = d
    s[:, 3] = np.linalg.norm(d, axis=1)
    s[:, 4:7] = rng.normal(0, 0.3, (n, 3))
    s[:, 7] = rng.integers(0, 2, n) + 4 * rng.choice([0, 2], n)
    s[:, 8:11] = rng.normal(0, 1.0, (n, 3))
    s[:, 11] = (rng.random(n) < valid_frac).astype(np.float32)
    return s
