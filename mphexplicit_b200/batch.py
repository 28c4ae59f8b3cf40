"""Batched form: many independent MPH-WC scenes stepped together.

A thin host mirror of the mph_batch_* C ABI (include/mph_b200.h).  Every
scene keeps its own *.data parameters, *.grid particles and cell grid; one
``step`` advances all of them by their own dt with the pair arithmetic of
MPH_MODE_MIXED_P64 (FP64 density pairs, FP32 force pairs) and FP64
integration, as persistent (scene, cell tile) sweeps
replayed through CUDA graphs.  ``autotune`` picks the tile shape on the batch
itself without advancing it.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np

from . import _native as N
from .solver import MphError


def _bcheck(st: int, handle=None) -> None:
    if st != N.MPH_OK:
        buf = C.create_string_buffer(1024)
        N.load().mph_batch_last_error(handle, buf, 1024)
        raise MphError(st, buf.value.decode(errors="replace"))


class Batch:
    """Scenes of one dimension (objects with params, header, type, xyz, vel,
    dim, as made by mphexplicit_b200.scenes) on the current CUDA device."""

    def __init__(self, scenes: Sequence, tiles: tuple | None = None):
        if not scenes:
            raise ValueError("a batch needs at least one scene")
        dims = {int(s.dim) for s in scenes}
        if len(dims) != 1:
            raise ValueError("all scenes of a batch must have the same dimension")
        self.dim = dims.pop()
        self._lib = N.load()
        S = len(scenes)
        self.counts = np.array([int(s.header.particle_count) for s in scenes], np.int64)
        self.offsets = np.concatenate([[0], np.cumsum(self.counts)])
        params = (N.Params * S)(*[s.params for s in scenes])
        headers = (N.GridHeader * S)(*[s.header for s in scenes])
        typ = np.ascontiguousarray(np.concatenate([np.asarray(s.type, np.int32) for s in scenes]))
        xyz = np.ascontiguousarray(np.concatenate([np.asarray(s.xyz, np.float64).reshape(-1, 3) for s in scenes]))
        vel = np.ascontiguousarray(np.concatenate([np.asarray(s.vel, np.float64).reshape(-1, 3) for s in scenes]))
        self.type = typ
        h = C.c_void_p()
        st = self._lib.mph_batch_create(S, params, headers, self.dim, typ.ctypes.data_as(C.POINTER(C.c_int)),
                                        xyz.ctypes.data_as(C.POINTER(C.c_double)),
                                        vel.ctypes.data_as(C.POINTER(C.c_double)), C.byref(h))
        _bcheck(st)
        self.handle = h
        if tiles is not None:
            self.set_tiles(*tiles)

    @property
    def n(self) -> int:
        return int(self.offsets[-1])

    @property
    def n_fluid(self) -> int:
        return int(np.count_nonzero(self.type < 2))

    @property
    def stream_handle(self) -> int:
        return int(self._lib.mph_batch_stream(self.handle) or 0)

    def step(self, nsteps: int = 1) -> None:
        _bcheck(self._lib.mph_batch_step(self.handle, int(nsteps)), self.handle)

    def synchronize(self) -> None:
        _bcheck(self._lib.mph_batch_synchronize(self.handle), self.handle)

    def set_tiles(self, tx: int, ty: int, tz: int = 1, threads: int = 256, ctas_per_sm: int = 0) -> None:
        _bcheck(self._lib.mph_batch_set_tiles(self.handle, int(tx), int(ty), int(tz), int(threads), int(ctas_per_sm)),
                self.handle)

    def autotune(self, steps: int = 32) -> list[dict]:
        cap = 64
        trials = (N.BatchTrial * cap)()
        cnt = C.c_int(0)
        _bcheck(self._lib.mph_batch_autotune(self.handle, int(steps), trials, cap, C.byref(cnt)), self.handle)
        return [{"tile": tuple(trials[k].tile), "threads": trials[k].threads, "ctas_per_sm": trials[k].ctas_per_sm,
                 "capacity": trials[k].capacity, "ms_per_step": trials[k].ms_per_step}
                for k in range(min(cnt.value, cap))]

    def info(self) -> dict:
        i = N.BatchInfo()
        _bcheck(self._lib.mph_batch_get_info(self.handle, C.byref(i)), self.handle)
        return {k: (tuple(getattr(i, k)) if k == "tile" else getattr(i, k)) for k, _ in N.BatchInfo._fields_}

    def state(self) -> tuple[np.ndarray, np.ndarray]:
        """Positions and velocities of all scenes, each in its input order,
        concatenated (n, 3)."""
        xyz = np.empty((self.n, 3), np.float64)
        vel = np.empty((self.n, 3), np.float64)
        _bcheck(self._lib.mph_batch_get_state(self.handle, xyz.ctypes.data_as(C.POINTER(C.c_double)),
                                              vel.ctypes.data_as(C.POINTER(C.c_double))), self.handle)
        return xyz, vel

    def scene_state(self, xyz: np.ndarray, vel: np.ndarray, s: int) -> tuple[np.ndarray, np.ndarray]:
        a, b = int(self.offsets[s]), int(self.offsets[s + 1])
        return xyz[a:b], vel[a:b]

    def profile(self, on: bool) -> None:
        _bcheck(self._lib.mph_batch_profile_enable(self.handle, 1 if on else 0), self.handle)

    def profile_read(self) -> dict:
        cap = 32
        out = (N.KernelStat * cap)()
        cnt = C.c_int(0)
        _bcheck(self._lib.mph_batch_profile_read(self.handle, out, cap, C.byref(cnt)), self.handle)
        return {out[k].name.decode(): (out[k].launches, out[k].total_ms) for k in range(min(cnt.value, cap))}

    def close(self) -> None:
        if getattr(self, "handle", None):
            self._lib.mph_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
