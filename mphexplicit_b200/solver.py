"""Python mirror of the reference solver's interface, over the C ABI.

The reference (Masahiro-Kondo-AIST/MphExplicit) is a program, not a library:
its interface is the command line (source/main.cpp:290-307), the *.data /
*.grid / *.prof / *.vtk files and the per-step call sequence of its main loop
(main.cpp:374-452).  This module offers the same pieces:

* ``read_data_file`` / ``read_grid_file`` / ``write_grid_file``: readDataFile,
  readGridFile, writeProfFile;
* ``Solver``: set-up + start-up (main.cpp:324-364) on construction,
  ``step`` = one loop body (386-431) + ``Time += Dt`` (449), ``write_vtk`` /
  ``write_prof`` = writeVtkFile / writeProfFile, ``compute_virial`` =
  calculateVirialStressAtParticle;
* ``run``: the whole main() loop with the reference's output schedule.

Errors raise ``MphError`` with the library's status code and message (the
reference exits instead).
"""
from __future__ import annotations

import ctypes as C
import time as _time
from dataclasses import dataclass

import numpy as np

from . import _native as N


class MphError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"mph error {code}: {msg}")
        self.code = code


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def _check(st: int, ctx=None) -> None:
    if st != N.MPH_OK:
        buf = C.create_string_buffer(1024)
        N.load().mph_last_error(ctx, buf, 1024)
        raise MphError(st, buf.value.decode(errors="replace"))


@dataclass
class Grid:
    """Contents of a *.grid / *.prof file, in file order."""

    header: N.GridHeader
    type: np.ndarray  # int32 [n]
    xyz: np.ndarray   # float64 [n, 3]
    vel: np.ndarray   # float64 [n, 3]


def default_params() -> N.Params:
    p = N.Params()
    _check(N.load().mph_params_defaults(C.byref(p)))
    return p


def read_data_file(path: str) -> N.Params:
    """readDataFile (main.cpp:489-539): unknown lines are ignored."""
    p = default_params()
    bad = C.c_int(0)
    _check(N.load().mph_read_data_file(str(path).encode(), C.byref(p), C.byref(bad)))
    return p


def read_grid_file(path: str) -> Grid:
    """readGridFile (main.cpp:541-640)."""
    lib = N.load()
    h = N.GridHeader()
    _check(lib.mph_read_grid_header(str(path).encode(), C.byref(h)))
    n = h.particle_count
    t = np.zeros(n, np.int32)
    x = np.zeros((n, 3), np.float64)
    v = np.zeros((n, 3), np.float64)
    _check(lib.mph_read_grid_file(str(path).encode(), C.byref(h), n, _ip(t), _dp(x), _dp(v)))
    return Grid(h, t, x, v)


def make_header(n: int, l0: float, dmin, dmax, time: float = 0.0) -> N.GridHeader:
    h = N.GridHeader()
    h.time = time
    h.particle_count = int(n)
    h.particle_spacing = float(l0)
    for d in range(3):
        h.domain_min[d] = float(dmin[d])
        h.domain_max[d] = float(dmax[d])
    return h


def write_grid_file(path: str, header: N.GridHeader, type_, xyz, vel) -> None:
    """writeProfFile format (main.cpp:672-696)."""
    t = np.ascontiguousarray(type_, np.int32)
    x = np.ascontiguousarray(xyz, np.float64)
    v = np.ascontiguousarray(vel, np.float64)
    _check(N.load().mph_write_grid_file(str(path).encode(), C.byref(header), _ip(t), _dp(x), _dp(v)))


def _gen_check(st: int) -> None:
    if st != N.MPH_OK:
        buf = C.create_string_buffer(512)
        N.load().mph_generator_last_error(buf, 512)
        raise MphError(st, buf.value.decode(errors="replace"))


def read_boid_file(path: str):
    """The reference generator's readfile (generator/generator.cpp:49-164):
    returns (Boid, [Cuboid, ...])."""
    lib = N.load()
    b = N.Boid()
    cnt = C.c_int(0)
    st = lib.mph_read_boid_file(str(path).encode(), C.byref(b), None, 0, C.byref(cnt))
    if st not in (N.MPH_OK, N.MPH_ERR_CAPACITY):
        _gen_check(st)
    arr = (N.Cuboid * max(cnt.value, 1))()
    _gen_check(lib.mph_read_boid_file(str(path).encode(), C.byref(b), arr, cnt.value, C.byref(cnt)))
    return b, [arr[k] for k in range(cnt.value)]


def generate_cuboids(cuboids):
    """genparticle (generator.cpp:170-193): (type, xyz, vel) of the cuboids'
    lattices in the reference's order."""
    lib = N.load()
    arr = (N.Cuboid * max(len(cuboids), 1))(*cuboids)
    n = C.c_longlong(0)
    _gen_check(lib.mph_generate_cuboids(arr, len(cuboids), None, None, None, 0, C.byref(n)))
    t = np.zeros(n.value, np.int32)
    x = np.zeros((n.value, 3), np.float64)
    v = np.zeros((n.value, 3), np.float64)
    _gen_check(lib.mph_generate_cuboids(arr, len(cuboids), _ip(t), _dp(x), _dp(v), n.value, C.byref(n)))
    return t, x, v


def generate_grid_file(boid_path: str, grid_path: str) -> int:
    """The whole generator (GeneratorForMph): *.boid in, *.grid out; returns
    the particle count."""
    n = C.c_longlong(0)
    _gen_check(N.load().mph_generate_grid_file(str(boid_path).encode(), str(grid_path).encode(), C.byref(n)))
    return int(n.value)


def write_vtk_arrays(path: str, state: dict) -> None:
    """writeVtkFile (main.cpp:698-834) from host arrays (keys as Solver.state())."""
    t = np.ascontiguousarray(state["type"], np.int32)
    nc = np.ascontiguousarray(state["neighbor_count"], np.int32)
    f64 = {k: np.ascontiguousarray(state[k], np.float64) for k in
           ("xyz", "vel", "force", "density_a", "vol_strain_p", "virial_pressure")}
    _check(N.load().mph_write_vtk_arrays(str(path).encode(), len(t), _ip(t), _dp(f64["xyz"]), _dp(f64["vel"]),
                                         _dp(f64["force"]), _ip(nc), _dp(f64["density_a"]),
                                         _dp(f64["vol_strain_p"]), _dp(f64["virial_pressure"])))


def format_e(values, as_float: bool = False) -> bytes:
    """values as "%e\\n" lines, formatted by the device (each value cast to
    float first when as_float, as writeVtkFile prints its fields)."""
    v = np.ascontiguousarray(values, np.float64).ravel()
    cap = 15 * len(v)
    out = C.create_string_buffer(max(cap, 1))
    n = C.c_longlong(0)
    _check(N.load().mph_format_e(v.ctypes.data_as(C.c_void_p), len(v), int(bool(as_float)), out, cap, C.byref(n)))
    return out.raw[:n.value]


@dataclass
class Checkpoint:
    """Contents of an exact checkpoint (mph_write_checkpoint): the particles in
    the order of the *.prof file the reference would write at that time."""
    params: N.Params
    header: N.GridHeader
    dim: int
    step: int
    type: np.ndarray
    particle_index: np.ndarray
    xyz: np.ndarray
    vel: np.ndarray


def write_checkpoint_arrays(path: str, ck: Checkpoint) -> None:
    t = np.ascontiguousarray(ck.type, np.int32)
    pi = np.ascontiguousarray(ck.particle_index, np.int32)
    x = np.ascontiguousarray(ck.xyz, np.float64)
    v = np.ascontiguousarray(ck.vel, np.float64)
    _check(N.load().mph_write_checkpoint_arrays(path.encode(), C.byref(ck.params), C.byref(ck.header), int(ck.dim),
                                                int(ck.step), _ip(t), _ip(pi), _dp(x), _dp(v)))


def read_checkpoint(path: str) -> Checkpoint:
    lib = N.load()
    p, h = N.Params(), N.GridHeader()
    dim, step = C.c_int(0), C.c_longlong(0)
    _check(lib.mph_read_checkpoint_header(path.encode(), C.byref(p), C.byref(h), C.byref(dim), C.byref(step)))
    n = h.particle_count
    t, pi = np.zeros(n, np.int32), np.zeros(n, np.int32)
    x, v = np.zeros((n, 3)), np.zeros((n, 3))
    _check(lib.mph_read_checkpoint(path.encode(), C.byref(p), C.byref(h), C.byref(dim), C.byref(step), n, _ip(t),
                                   _ip(pi), _dp(x), _dp(v)))
    return Checkpoint(p, h, dim.value, step.value, t, pi, x, v)


def compute_constants(params: N.Params, header: N.GridHeader, dim: int) -> N.Constants:
    c = N.Constants()
    _check(N.load().mph_compute_constants(C.byref(params), C.byref(header), dim, C.byref(c)))
    return c


_MODES = {"fp64": N.MODE_FP64, "mixed": N.MODE_MIXED, "mixed_p64": N.MODE_MIXED_P64, "learned": N.MODE_LEARNED,
          # the mixed forms with the table-free (cell-walk) force sweep
          "mixed_walk": N.MODE_MIXED | N.MIXED_CELL_WALK, "mixed_p64_walk": N.MODE_MIXED_P64 | N.MIXED_CELL_WALK}


class Solver:
    """One simulation on the current CUDA device (a context of the C ABI)."""

    def __init__(self, params: N.Params, header: N.GridHeader, type_, xyz, vel, dim: int = 3,
                 mode: str = "fp64"):
        lib = N.load()
        self._lib = lib
        self.dim = dim
        self.mode = mode
        t = np.ascontiguousarray(type_, np.int32)
        x = np.ascontiguousarray(xyz, np.float64).reshape(-1, 3)
        v = np.ascontiguousarray(vel, np.float64).reshape(-1, 3)
        if not (len(t) == len(x) == len(v) == header.particle_count):
            raise MphError(N.MPH_ERR_ARG, "array lengths differ from header.particle_count")
        self.params = params
        self.header = header
        self.n = header.particle_count
        ctx = C.c_void_p()
        _check(lib.mph_create(C.byref(params), C.byref(header), dim, _MODES[mode], _ip(t), _dp(x), _dp(v),
                              C.byref(ctx)))
        self._ctx = ctx

    @classmethod
    def from_files(cls, data: str, grid: str, dim: int = 3, mode: str = "fp64") -> "Solver":
        g = read_grid_file(grid)
        return cls(read_data_file(data), g.header, g.type, g.xyz, g.vel, dim=dim, mode=mode)

    @classmethod
    def from_checkpoint(cls, path: str, mode: str = "fp64") -> "Solver":
        """Restart from an exact checkpoint (the reference's restart from the
        *.prof file of that time, without its text rounding)."""
        ck = read_checkpoint(path)
        return cls(ck.params, ck.header, ck.type, ck.xyz, ck.vel, dim=ck.dim, mode=mode)

    def write_checkpoint(self, path: str) -> None:
        _check(self._lib.mph_write_checkpoint(self._ctx, path.encode()), self._ctx)

    # -- stepping --------------------------------------------------------
    def step(self, nsteps: int = 1) -> None:
        _check(self._lib.mph_step(self._ctx, int(nsteps)), self._ctx)

    def synchronize(self) -> None:
        _check(self._lib.mph_synchronize(self._ctx), self._ctx)

    # -- learned form ----------------------------------------------------
    def set_learned(self, model, judge_interval: int = 20, tolerance: float = 1e-2) -> None:
        """Attach an edge-MLP model (mphexplicit_b200.learned.Model) to a
        "learned" solver; the plain FP64 step judges every judge_interval steps."""
        _check(self._lib.mph_set_learned(self._ctx, model.handle, int(judge_interval), float(tolerance)), self._ctx)
        self._model = model  # the context keeps a reference

    def learned_stats(self) -> dict:
        i = N.LearnedInfo()
        _check(self._lib.mph_learned_stats(self._ctx, C.byref(i)), self._ctx)
        return {k: getattr(i, k) for k, _ in N.LearnedInfo._fields_}

    def collect_samples(self, dataset, count: int, seed: int = 0) -> None:
        """Append `count` random edges of the current state to the dataset."""
        _check(self._lib.mph_collect_samples(self._ctx, dataset.handle, int(count), int(seed)), self._ctx)

    # -- read-back -------------------------------------------------------
    def info(self) -> dict:
        i = N.Info()
        _check(self._lib.mph_get_info(self._ctx, C.byref(i)), self._ctx)
        return {k: getattr(i, k) for k, _ in N.Info._fields_}

    def constants(self) -> N.Constants:
        c = N.Constants()
        _check(self._lib.mph_get_constants(self._ctx, C.byref(c)), self._ctx)
        return c

    def state(self) -> dict:
        """Particle arrays in the current (cell-sorted) order, as the reference holds them."""
        n = self.n
        out = {
            "particle_index": np.zeros(n, np.int32),
            "type": np.zeros(n, np.int32),
            "xyz": np.zeros((n, 3)),
            "vel": np.zeros((n, 3)),
            "force": np.zeros((n, 3)),
            "neighbor_count": np.zeros(n, np.int32),
            "density_a": np.zeros(n),
            "vol_strain_p": np.zeros(n),
            "virial_pressure": np.zeros(n),
        }
        _check(self._lib.mph_get_state(
            self._ctx, _ip(out["particle_index"]), _ip(out["type"]), _dp(out["xyz"]), _dp(out["vel"]),
            _dp(out["force"]), _ip(out["neighbor_count"]), _dp(out["density_a"]), _dp(out["vol_strain_p"]),
            _dp(out["virial_pressure"])), self._ctx)
        return out

    def get_xv(self, xyz: np.ndarray, vel: np.ndarray) -> None:
        """Positions and velocities only, into caller arrays (sorted order)."""
        _check(self._lib.mph_get_state(self._ctx, None, None, _dp(xyz), _dp(vel), None, None, None, None, None),
               self._ctx)

    def set_sweep_layout(self, layout: str) -> None:
        """FP64 pair sweeps: "auto" (by size), "thread" or "warp" per particle."""
        code = {"auto": 0, "thread": 1, "warp": 2}[layout]
        _check(self._lib.mph_set_sweep_layout(self._ctx, code), self._ctx)

    def set_step_graphs(self, enable: bool) -> None:
        """Graph launches for several FP64 steps (default) or the host path."""
        _check(self._lib.mph_set_step_graphs(self._ctx, 1 if enable else 0), self._ctx)

    def step_read_state(self, nsteps: int, xyz: np.ndarray | None, vel: np.ndarray | None) -> None:
        """step(nsteps), then the positions and velocities after it into caller
        arrays (sorted order, C-contiguous float64 [n, 3]); the FP64 form copies
        them while its last step still computes (pinned arrays overlap fully)."""
        for a in (xyz, vel):
            if a is not None and not (a.dtype == np.float64 and a.flags.c_contiguous and a.size == 3 * self.n):
                raise ValueError("xyz / vel must be C-contiguous float64 arrays of n x 3")
        _check(self._lib.mph_step_read_state(self._ctx, int(nsteps), _dp(xyz) if xyz is not None else None,
                                             _dp(vel) if vel is not None else None), self._ctx)

    def set_state(self, xyz: np.ndarray, vel: np.ndarray) -> None:
        _check(self._lib.mph_set_state(self._ctx, _dp(np.ascontiguousarray(xyz, np.float64)),
                                       _dp(np.ascontiguousarray(vel, np.float64))), self._ctx)

    def fields(self) -> dict:
        n = self.n
        out = {"divergence_p": np.zeros(n), "pressure_p": np.zeros(n), "pressure_a": np.zeros(n),
               "gravity_center": np.zeros((n, 3))}
        _check(self._lib.mph_get_fields(self._ctx, _dp(out["divergence_p"]), _dp(out["pressure_p"]),
                                        _dp(out["pressure_a"]), _dp(out["gravity_center"])), self._ctx)
        return out

    def cells(self) -> dict:
        tot = self.constants().total_cell_count
        out = {"cell_index": np.zeros(self.n, np.int32), "fluid_begin": np.zeros(tot, np.int32),
               "fluid_end": np.zeros(tot, np.int32), "wall_begin": np.zeros(tot, np.int32),
               "wall_end": np.zeros(tot, np.int32)}
        _check(self._lib.mph_get_cells(self._ctx, _ip(out["cell_index"]), _ip(out["fluid_begin"]),
                                       _ip(out["fluid_end"]), _ip(out["wall_begin"]), _ip(out["wall_end"])),
               self._ctx)
        return out

    def neighbors(self) -> tuple[np.ndarray, np.ndarray]:
        """(NeighborPtr[n+1], NeighborInd[...]) of the last rebuild."""
        ptr = np.zeros(self.n + 1, np.int64)
        _check(self._lib.mph_get_neighbors(self._ctx, ptr.ctypes.data_as(C.POINTER(C.c_longlong)), None, 0),
               self._ctx)
        ind = np.zeros(max(int(ptr[-1]), 1), np.int32)
        _check(self._lib.mph_get_neighbors(self._ctx, ptr.ctypes.data_as(C.POINTER(C.c_longlong)), _ip(ind),
                                           len(ind)), self._ctx)
        return ptr, ind[: int(ptr[-1])]

    def compute_virial(self) -> None:
        _check(self._lib.mph_compute_virial(self._ctx), self._ctx)

    def conserved_sums(self) -> np.ndarray:
        out = np.zeros(5)
        _check(self._lib.mph_conserved_sums(self._ctx, _dp(out)), self._ctx)
        return out

    # -- measurement hooks ------------------------------------------------
    @property
    def stream_handle(self) -> int:
        """cudaStream_t of this context (for CUDA events recorded by the caller)."""
        return int(self._lib.mph_stream(self._ctx) or 0)

    def launch_count(self) -> int:
        return int(self._lib.mph_launch_count(self._ctx))

    def profile(self, enable: bool) -> None:
        _check(self._lib.mph_profile_enable(self._ctx, 1 if enable else 0), self._ctx)

    def profile_read(self) -> dict:
        """{kernel name: (launches, total ms)} since profile(True)."""
        buf = (N.KernelStat * 64)()
        cnt = C.c_int(0)
        _check(self._lib.mph_profile_read(self._ctx, buf, 64, C.byref(cnt)), self._ctx)
        return {buf[k].name.decode(): (int(buf[k].launches), float(buf[k].total_ms)) for k in range(cnt.value)}

    def write_vtk(self, path: str) -> None:
        _check(self._lib.mph_write_vtk(self._ctx, str(path).encode()), self._ctx)

    def write_prof(self, path: str) -> None:
        _check(self._lib.mph_write_prof(self._ctx, str(path).encode()), self._ctx)

    def write_vtk_async(self, path: str) -> None:
        """Formats the current state on the device and writes the file from
        the context's writer thread while stepping continues."""
        _check(self._lib.mph_write_vtk_async(self._ctx, str(path).encode()), self._ctx)

    def write_prof_async(self, path: str) -> None:
        _check(self._lib.mph_write_prof_async(self._ctx, str(path).encode()), self._ctx)

    def output_wait(self) -> None:
        """Returns once every file written behind the step is on disk."""
        _check(self._lib.mph_output_wait(self._ctx), self._ctx)

    def close(self) -> None:
        if getattr(self, "_ctx", None):
            self._lib.mph_destroy(self._ctx)
            self._ctx = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def run(data: str, grid: str, prof: str = "sample%03d.prof", vtk: str = "sample%03d.vtk",
        log: str | None = None, dim: int = 3, mode: str = "fp64", startup_vtk: str | None = "output.vtk") -> dict:
    """The reference's main() loop (main.cpp:357-452) with its output schedule."""
    params = read_data_file(data)
    g = read_grid_file(grid)
    s = Solver(params, g.header, g.type, g.xyz, g.vel, dim=dim, mode=mode)
    if startup_vtk:
        s.write_vtk(startup_vtk)
    t = g.header.time
    dt = params.dt
    out_next = 0.0
    vtk_next = 0.0
    istep = int(t / dt)
    steps = 0
    t_step = 0.0
    lines = []
    while t < params.end_time + 1.0e-5 * dt:
        if t + 1.0e-5 * dt >= out_next:
            s.write_prof_async(prof % istep)
            lines.append("@ Prof Output Time : %e" % t)
            out_next += params.output_interval
        a = _time.perf_counter()
        s.step(1)
        s.synchronize()
        t_step += _time.perf_counter() - a
        steps += 1
        if t + 1.0e-5 * dt >= vtk_next:
            if mode == "fp64":
                s.compute_virial()
            s.write_vtk_async(vtk % istep)
            lines.append("@ Vtk Output Time : %e" % t)
            vtk_next += params.vtk_output_interval
        t += dt
        istep += 1
    s.output_wait()
    info = s.info()
    s.close()
    if log:
        with open(log, "w") as f:
            f.write("\n".join(lines) + "\n")
    return {"steps": steps, "seconds": t_step, "info": info}
