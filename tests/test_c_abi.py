"""The C ABI from a C program (CPU only): tests/c_abi_probe.c, compiled as C99
with warnings as errors against include/mph_b200.h and linked with the
library, reads a golden case and writes a VTK; its results must equal what the
same entry points give through ctypes."""
import os
import subprocess
import tempfile

import numpy as np

import mphexplicit_b200 as M
from tests.common import GoldenCase

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "mphexplicit_b200")


def test_c_program_calls_the_host_entry_points():
    case = GoldenCase("square_drop_skip")
    with tempfile.TemporaryDirectory() as td:
        exe = os.path.join(td, "probe")
        subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
                        os.path.join(ROOT, "tests", "c_abi_probe.c"), "-o", exe, "-L", LIBDIR, "-lmph_b200",
                        "-Wl,-rpath," + LIBDIR], check=True, capture_output=True, text=True)
        vtk = os.path.join(td, "c.vtk")
        r = subprocess.run([exe, case.data, case.grid, vtk, str(case.dim)], capture_output=True, text=True,
                           timeout=120)
        assert r.returncode == 0, r.stdout + r.stderr
        out = dict(line.split(" ", 1) for line in r.stdout.strip().splitlines())

        p = M.read_data_file(case.data)
        g = M.read_grid_file(case.grid)
        c = M.compute_constants(p, g.header, case.dim)
        assert out["particles"].split()[0] == str(g.header.particle_count)
        assert float(out["particles"].split()[-1]) == p.dt
        assert out["cells"] == "%d %d %d total %d" % (c.cell_count[0], c.cell_count[1], c.cell_count[2],
                                                      c.total_cell_count)
        assert float(out["max_radius"]) == c.max_radius
        assert out["write_vtk"] == "0"
        st = {"type": g.type, "xyz": g.xyz, "vel": g.vel, "force": g.vel,
              "neighbor_count": np.zeros(len(g.type), np.int32)}
        for k in ("density_a", "vol_strain_p", "virial_pressure"):
            st[k] = np.zeros(len(g.type))
        py_vtk = os.path.join(td, "py.vtk")
        M.write_vtk_arrays(py_vtk, st)
        assert open(vtk, "rb").read() == open(py_vtk, "rb").read()
        # dim 4 is rejected before any device work, with a message
        assert out["create_dim4"] == "%d ctx_null 1" % M._native.MPH_ERR_ARG
        assert out["error_message"].strip()
