"""Python access to the test oracle.  TEST INFRASTRUCTURE ONLY.

* ``Oracle``: the C restatement in ``oracle/mph_oracle.c`` (``liboracle.so``),
  driven through ctypes.  Used by tests/, ``__graft_entry__.smoke()`` and the
  CPU-baseline leg of ``bench.py`` -- never by the product.
* ``run_reference``: the reference solver's own code (``oracle/_ref/ref_mph2d``
  / ``ref_mph3d``, compiled from its sources by ``oracle/Makefile``), run as a
  subprocess on a *.data/*.grid pair; returns its arrays.
"""
from __future__ import annotations

import ctypes as C
import json
import os
import subprocess
import tempfile

import numpy as np

from mphexplicit_b200 import _native as N

from .ref_inputs import ref_available, time_reference  # noqa: F401  (re-exported for tests and bench)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB):
        build()
    lib = C.CDLL(LIB)
    P = C.c_void_p
    dp = C.POINTER(C.c_double)
    ip = C.POINTER(C.c_int)
    lib.oracle_create.restype = P
    lib.oracle_create.argtypes = [C.POINTER(N.Params), C.POINTER(N.GridHeader), C.c_int, ip, dp, dp]
    lib.oracle_step.argtypes = [P, C.c_int]
    lib.oracle_virial.argtypes = [P]
    lib.oracle_destroy.argtypes = [P]
    lib.oracle_particle_count.restype = C.c_int
    lib.oracle_particle_count.argtypes = [P]
    lib.oracle_rebuild_count.restype = C.c_longlong
    lib.oracle_rebuild_count.argtypes = [P]
    lib.oracle_neighbor_ind_count.restype = C.c_longlong
    lib.oracle_neighbor_ind_count.argtypes = [P]
    lib.oracle_time.restype = C.c_double
    lib.oracle_time.argtypes = [P]
    lib.oracle_get_constants.argtypes = [P, C.POINTER(N.Constants)]
    lib.oracle_compute_constants.restype = C.c_int
    lib.oracle_compute_constants.argtypes = [C.POINTER(N.Params), C.POINTER(N.GridHeader), C.c_int,
                                             C.POINTER(N.Constants)]
    lib.oracle_get_state.argtypes = [P, ip, ip, dp, dp, dp, ip, dp, dp, dp]
    lib.oracle_get_fields.argtypes = [P, dp, dp, dp, dp]
    lib.oracle_get_cells.argtypes = [P, ip, ip, ip, ip, ip]
    lib.oracle_get_neighbors.argtypes = [P, C.POINTER(C.c_longlong), ip]
    _lib = lib
    return lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def constants(params, header, dim) -> N.Constants:
    c = N.Constants()
    st = load().oracle_compute_constants(C.byref(params), C.byref(header), dim, C.byref(c))
    if st != 0:
        raise ValueError("oracle_compute_constants failed: %d" % st)
    return c


class Oracle:
    """CPU restatement of the reference step (same call sequence as main())."""

    def __init__(self, params, header, type_, xyz, vel, dim):
        lib = load()
        self._lib = lib
        self._t = np.ascontiguousarray(type_, np.int32)
        self._x = np.ascontiguousarray(xyz, np.float64)
        self._v = np.ascontiguousarray(vel, np.float64)
        self.params, self.header, self.dim = params, header, dim
        self._s = lib.oracle_create(C.byref(params), C.byref(header), dim, _ip(self._t), _dp(self._x),
                                    _dp(self._v))
        if not self._s:
            raise ValueError("oracle_create failed (bad input or geometry)")
        self.n = lib.oracle_particle_count(self._s)

    @classmethod
    def from_scene(cls, scene):
        return cls(scene.params, scene.header, scene.type, scene.xyz, scene.vel, scene.dim)

    def step(self, n=1):
        self._lib.oracle_step(self._s, int(n))

    def virial(self):
        self._lib.oracle_virial(self._s)

    @property
    def rebuilds(self):
        return self._lib.oracle_rebuild_count(self._s)

    @property
    def time(self):
        return self._lib.oracle_time(self._s)

    def constants(self):
        c = N.Constants()
        self._lib.oracle_get_constants(self._s, C.byref(c))
        return c

    def state(self):
        n = self.n
        o = {"particle_index": np.zeros(n, np.int32), "type": np.zeros(n, np.int32), "xyz": np.zeros((n, 3)),
             "vel": np.zeros((n, 3)), "force": np.zeros((n, 3)), "neighbor_count": np.zeros(n, np.int32),
             "density_a": np.zeros(n), "vol_strain_p": np.zeros(n), "virial_pressure": np.zeros(n)}
        self._lib.oracle_get_state(self._s, _ip(o["particle_index"]), _ip(o["type"]), _dp(o["xyz"]),
                                   _dp(o["vel"]), _dp(o["force"]), _ip(o["neighbor_count"]),
                                   _dp(o["density_a"]), _dp(o["vol_strain_p"]), _dp(o["virial_pressure"]))
        return o

    def fields(self):
        n = self.n
        o = {"divergence_p": np.zeros(n), "pressure_p": np.zeros(n), "pressure_a": np.zeros(n),
             "gravity_center": np.zeros((n, 3))}
        self._lib.oracle_get_fields(self._s, _dp(o["divergence_p"]), _dp(o["pressure_p"]), _dp(o["pressure_a"]),
                                    _dp(o["gravity_center"]))
        return o

    def cells(self):
        tot = self.constants().total_cell_count
        o = {"cell_index": np.zeros(self.n, np.int32), "fluid_begin": np.zeros(tot, np.int32),
             "fluid_end": np.zeros(tot, np.int32), "wall_begin": np.zeros(tot, np.int32),
             "wall_end": np.zeros(tot, np.int32)}
        self._lib.oracle_get_cells(self._s, _ip(o["cell_index"]), _ip(o["fluid_begin"]), _ip(o["fluid_end"]),
                                   _ip(o["wall_begin"]), _ip(o["wall_end"]))
        return o

    def neighbors(self):
        ptr = np.zeros(self.n + 1, np.int64)
        self._lib.oracle_get_neighbors(self._s, ptr.ctypes.data_as(C.POINTER(C.c_longlong)), None)
        ind = np.zeros(max(int(ptr[-1]), 1), np.int32)
        self._lib.oracle_get_neighbors(self._s, ptr.ctypes.data_as(C.POINTER(C.c_longlong)), _ip(ind))
        return ptr, ind[: int(ptr[-1])]

    def close(self):
        if getattr(self, "_s", None):
            self._lib.oracle_destroy(self._s)
            self._s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
def read_dump(path: str) -> dict:
    """Parse the binary dump written by oracle/ref_harness.cpp."""
    raw = open(path, "rb").read()
    off = 0

    def take(dtype, count):
        nonlocal off
        a = np.frombuffer(raw, dtype=dtype, count=count, offset=off)
        off += a.nbytes
        return a.copy()

    magic, ver, n, tot = take(np.int32, 4)
    assert magic == 0x4D504852 and ver == 1
    nic, rebuilds = take(np.int64, 2)
    time_, n0a, n0p = take(np.float64, 3)
    hi = take(np.int32, 8)
    d = {"n": int(n), "total_cell_count": int(tot), "neighbor_ind_count": int(nic), "rebuilds": int(rebuilds),
         "time": float(time_), "n0a": float(n0a), "n0p": float(n0p), "cell_count": hi[:3].tolist(),
         "fluid_begin_all": int(hi[3]), "fluid_end_all": int(hi[4]), "wall_begin_all": int(hi[5]),
         "wall_end_all": int(hi[6])}
    d["particle_index"] = take(np.int32, n)
    d["type"] = take(np.int32, n)
    d["xyz"] = take(np.float64, 3 * n).reshape(n, 3)
    d["vel"] = take(np.float64, 3 * n).reshape(n, 3)
    d["force"] = take(np.float64, 3 * n).reshape(n, 3)
    d["neighbor_count"] = take(np.int32, n)
    d["density_a"] = take(np.float64, n)
    d["vol_strain_p"] = take(np.float64, n)
    d["divergence_p"] = take(np.float64, n)
    d["pressure_p"] = take(np.float64, n)
    d["pressure_a"] = take(np.float64, n)
    d["gravity_center"] = take(np.float64, 3 * n).reshape(n, 3)
    d["virial_pressure"] = take(np.float64, n)
    d["cell_index"] = take(np.int32, n)
    d["fluid_begin"] = take(np.int32, tot)
    d["fluid_end"] = take(np.int32, tot)
    d["wall_begin"] = take(np.int32, tot)
    d["wall_end"] = take(np.int32, tot)
    d["nptr"] = take(np.int64, n + 1)
    d["nind"] = take(np.int32, int(nic))
    return d


def run_reference(data_path: str, grid_path: str, dim: int, nsteps: int, virial: bool = False,
                  timeout: float = 600, vtk: str | None = None, prof: str | None = None) -> dict:
    """Run the reference's own code for nsteps on the given files; return its
    arrays (and let it write its own VTK / prof files when paths are given)."""
    exe = os.path.join(REF_DIR, "ref_mph%dd" % dim)
    with tempfile.TemporaryDirectory() as td:
        out = os.path.join(td, "dump.bin")
        cmd = [exe, "dump", data_path, grid_path, str(nsteps), out] + (["virial"] if virial else [])
        cmd += (["vtk=" + os.path.abspath(vtk)] if vtk else []) + (["prof=" + os.path.abspath(prof)] if prof else [])
        env = dict(os.environ, OMP_NUM_THREADS=os.environ.get("OMP_NUM_THREADS", "1"))
        subprocess.run(cmd, check=True, cwd=td, env=env, timeout=timeout, stdout=subprocess.DEVNULL,
                       stderr=subprocess.DEVNULL)
        return read_dump(out)


def time_oracle(scene, warmup: int, steps: int, max_seconds: float = 1.0e30) -> dict:
    """Wall-clock the C restatement's step loop (used when oracle/_ref is absent)."""
    import time as _t
    o = Oracle.from_scene(scene)
    o.step(warmup)
    rb0 = o.rebuilds
    t0 = _t.perf_counter()
    done = 0
    while done < steps:
        o.step(1)
        done += 1
        if _t.perf_counter() - t0 > max_seconds:
            break
    sec = _t.perf_counter() - t0
    return {"seconds": sec, "steps": done, "particles": o.n, "fluid": int((scene.type < 2).sum()),
            "rebuilds": o.rebuilds - rb0, "threads": int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))}
