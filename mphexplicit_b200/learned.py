"""The learned form's edge-MLP surrogate and its training data (C ABI
mph_model_* / mph_dataset_*; kernels in csrc/k_mlp.cu).

Model: 9 inputs -> 128 -> 128 -> 128 -> 3 with SiLU, BF16 weights and
activations, FP32 accumulation on the tcgen05 tensor cores.  A sample is 12
floats: (dx, dy, dz, r)/l0, (ux, uy, uz, type_i + 4 type_j), (fx, fy, fz, valid)
with u = v_j - v_i and f the FP64 viscous + surface-tension force of j on i.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .solver import MphError, _check


def _fp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _mcheck(st: int, handle) -> None:
    if st != N.MPH_OK:
        buf = C.create_string_buffer(1024)
        N.load().mph_model_last_error(handle, buf, 1024)
        raise MphError(st, buf.value.decode(errors="replace"))


class Dataset:
    """Training samples in device memory."""

    def __init__(self, capacity: int):
        self._lib = N.load()
        h = C.c_void_p()
        _check(self._lib.mph_dataset_create(int(capacity), C.byref(h)))
        self.handle = h

    def __len__(self) -> int:
        return int(self._lib.mph_dataset_size(self.handle))

    def append(self, samples: np.ndarray) -> None:
        a = np.ascontiguousarray(samples, np.float32).reshape(-1, N.SAMPLE_FLOATS)
        _check(self._lib.mph_dataset_append(self.handle, _fp(a), len(a)))

    def read(self, first: int = 0, count: int | None = None) -> np.ndarray:
        count = len(self) - first if count is None else count
        out = np.empty((count, N.SAMPLE_FLOATS), np.float32)
        _check(self._lib.mph_dataset_read(self.handle, int(first), int(count), _fp(out)))
        return out

    def close(self) -> None:
        if getattr(self, "handle", None):
            self._lib.mph_dataset_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Model:
    """The edge-MLP surrogate on the current CUDA device."""

    def __init__(self, seed: int = 0):
        self._lib = N.load()
        h = C.c_void_p()
        _check(self._lib.mph_model_create(int(seed), C.byref(h)))
        self.handle = h
        self.n_params = int(self._lib.mph_model_param_count())

    def params(self) -> np.ndarray:
        out = np.empty(self.n_params, np.float32)
        _mcheck(self._lib.mph_model_get_params(self.handle, _fp(out)), self.handle)
        return out

    def set_params(self, p: np.ndarray) -> None:
        a = np.ascontiguousarray(p, np.float32)
        if a.size != self.n_params:
            raise MphError(N.MPH_ERR_ARG, "expected %d parameters" % self.n_params)
        _mcheck(self._lib.mph_model_set_params(self.handle, _fp(a)), self.handle)

    def set_scales(self, velocity_scale: float, force_scale: float) -> None:
        _mcheck(self._lib.mph_model_set_scales(self.handle, float(velocity_scale), float(force_scale)), self.handle)

    def scales(self) -> tuple[float, float]:
        u, f = C.c_double(), C.c_double()
        _mcheck(self._lib.mph_model_get_scales(self.handle, C.byref(u), C.byref(f)), self.handle)
        return u.value, f.value

    def fit_scales(self, ds: Dataset) -> None:
        _mcheck(self._lib.mph_model_fit_scales(self.handle, ds.handle), self.handle)

    def gradient(self, samples: np.ndarray) -> tuple[np.ndarray, float]:
        """Gradient of the mean squared error of the scaled outputs, and the loss."""
        a = np.ascontiguousarray(samples, np.float32).reshape(-1, N.SAMPLE_FLOATS)
        g = np.empty(self.n_params, np.float32)
        loss = C.c_double()
        _mcheck(self._lib.mph_model_gradient(self.handle, _fp(a), len(a), _fp(g), C.byref(loss)), self.handle)
        return g, loss.value

    def predict(self, samples: np.ndarray) -> np.ndarray:
        """Pair forces (N) of the samples, [n, 3]."""
        a = np.ascontiguousarray(samples, np.float32).reshape(-1, N.SAMPLE_FLOATS)
        out = np.empty((len(a), 4), np.float32)
        _mcheck(self._lib.mph_model_predict(self.handle, _fp(a), len(a), _fp(out)), self.handle)
        return out[:, :3]

    def train(self, ds: Dataset, epochs: int = 4, batch: int = 16384, lr: float = 2e-3, seed: int = 0) -> float:
        loss = C.c_double()
        _mcheck(self._lib.mph_model_train(self.handle, ds.handle, int(epochs), int(batch), float(lr), int(seed),
                                          C.byref(loss)), self.handle)
        return loss.value

    def check_wait(self, kernel: int, polls: int) -> tuple[int, str]:
        """mph_model_check_wait: the training (0) or inference (1) kernel with
        its tensor-core work withheld and a wait limit of `polls`; returns the
        status (MPH_ERR_DEVICE when the bounded wait ran out as it should) and
        the model's error message."""
        st = self._lib.mph_model_check_wait(self.handle, int(kernel), int(polls))
        buf = C.create_string_buffer(256)
        self._lib.mph_model_last_error(self.handle, buf, 256)
        return st, buf.value.decode(errors="replace")

    def close(self) -> None:
        if getattr(self, "handle", None):
            self._lib.mph_model_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
