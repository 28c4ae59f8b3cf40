"""The device writers of *.prof / *.vtk (needs a B200).

writeProfFile / writeVtkFile (main.cpp:672-834) print every value with glibc's
"%e"; the device formatter must give the same bytes for every double:
random bit patterns over the whole exponent range, subnormals, exact decimal
ties (rounded to even), the neighbours of ties and of powers of ten, and the
special values.  The files written through the context must equal the host
writers' bytes on the same state, in every form, also when written behind
the step."""
import ctypes as C
import os
import tempfile

import numpy as np
import pytest

import mphexplicit_b200 as M
from mphexplicit_b200 import scenes

pytestmark = pytest.mark.gpu

_libc = C.CDLL(None)
_libc.snprintf.restype = C.c_int


def printf_e(values) -> bytes:
    buf = C.create_string_buffer(64)
    out = []
    for v in values:
        n = _libc.snprintf(buf, 64, b"%e\n", C.c_double(float(v)))
        out.append(buf.raw[:n])
    return b"".join(out)


def tie_values() -> np.ndarray:
    """Dyadic values whose decimal expansion has exactly 8 significant digits
    ending in 5: k/2^j with k odd has j decimals, the last one a 5."""
    vals = []
    for j, lo, hi in [(7, 1, 10), (6, 10, 100), (10, 0.001, 0.01), (8, 0.1, 1), (4, 1000, 10000), (3, 10000, 100000)]:
        ks = np.arange(int(np.ceil(lo * 2 ** j)), int(hi * 2 ** j))
        ks = ks[ks % 2 == 1]
        vals.append(ks[:: max(1, len(ks) // 400)] / 2.0 ** j)
    ints = np.array([12345675.0, 12345665.0, 99999995.0, 10000005.0, 10000015.0, 2.5e7 + 5, 98765435.0])
    big = np.array([12345675.0 * 2.0 ** 40, 3.0 * 2.0 ** 60, 1125899906842624.0 * 5])  # large dyadic integers
    return np.concatenate(vals + [ints, big])


def edge_values(rng) -> np.ndarray:
    ties = tie_values()
    near = np.concatenate([np.nextafter(ties, np.inf), np.nextafter(ties, -np.inf)])
    p10 = 10.0 ** np.arange(-307, 308, dtype=np.float64)
    near10 = np.concatenate([p10, np.nextafter(p10, np.inf), np.nextafter(p10, -np.inf), p10 * 9.9999995,
                             p10 * 9.99999949999, p10 * 9.9999995000001, [1e308, np.nextafter(1e308, 0)]])
    special = np.array([0.0, -0.0, np.inf, -np.inf, np.nan, 5e-324, -5e-324, 2.2250738585072014e-308,
                        2.225073858507201e-308, 1.7976931348623157e308, -1.7976931348623157e308, 1.0, -1.0, 0.5,
                        9999999.5, 999999.5, 9.9999995, 0.1, 1e-5, 1e22, 1e23, 3.4028234663852886e38,
                        3.4028235677973366e38, 1.401298464324817e-45, 7e-46, 1e-40])
    sub = rng.integers(1, 2 ** 52, size=2000, dtype=np.int64).view(np.float64)
    return np.concatenate([ties, -ties, near, near10, -near10, special, sub])


def random_bits(rng, n) -> np.ndarray:
    v = rng.integers(0, 2 ** 63, size=n, dtype=np.int64)
    v ^= rng.integers(0, 2, size=n, dtype=np.int64) << 63
    v = v.view(np.float64)
    return v[np.isfinite(v)]


@pytest.mark.parametrize("as_float", [False, True])
def test_format_e_equals_printf(as_float):
    rng = np.random.default_rng(7)
    vals = np.concatenate([edge_values(rng), random_bits(rng, 60000),
                           rng.normal(0, 1, 20000), rng.normal(0, 1e4, 20000) * rng.random(20000)])
    with np.errstate(over="ignore"):
        expect_vals = vals.astype(np.float32).astype(np.float64) if as_float else vals
    got = M.format_e(vals, as_float=as_float)
    want = printf_e(expect_vals)
    if got != want:
        g, w = got.split(b"\n"), want.split(b"\n")
        bad = [i for i in range(min(len(g), len(w))) if g[i] != w[i]]
        i = bad[0] if bad else min(len(g), len(w))
        raise AssertionError(f"{len(bad)} lines differ; first {vals[i]!r}: {g[i] if i < len(g) else None} "
                             f"vs {w[i] if i < len(w) else None}")


def test_format_e_ties_round_to_even():
    got = M.format_e([1.0078125, 1.0234375, 12345675.0, 12345665.0, 0.0029296875]).split(b"\n")
    assert got[:5] == [b"1.007812e+00", b"1.023438e+00", b"1.234568e+07", b"1.234566e+07", b"2.929688e-03"]


def _host_bytes(s, td, time):
    st = s.state()
    vtk, prof = os.path.join(td, "host.vtk"), os.path.join(td, "host.prof")
    M.write_vtk_arrays(vtk, st)
    h = M.GridHeader()
    C.memmove(C.byref(h), C.byref(s.header), C.sizeof(h))
    h.time = time
    M.write_grid_file(prof, h, st["type"], st["xyz"], st["vel"])
    return open(vtk, "rb").read(), open(prof, "rb").read()


@pytest.mark.parametrize("mode", ["fp64", "mixed", "mixed_p64"])
def test_device_files_equal_host_writers(mode):
    sc = scenes.dam_break_3d(fluid=(12, 8, 14), box=(24, 10, 18), seed=11)
    s = M.Solver(sc.params, sc.header, sc.type, sc.xyz, sc.vel, dim=3, mode=mode)
    s.step(25)
    if mode == "fp64":
        s.compute_virial()
    with tempfile.TemporaryDirectory() as td:
        vtk, prof = os.path.join(td, "dev.vtk"), os.path.join(td, "dev.prof")
        s.write_vtk(vtk)
        s.write_prof(prof)
        hv, hp = _host_bytes(s, td, s.info()["time"])
        assert open(vtk, "rb").read() == hv
        assert open(prof, "rb").read() == hp
    s.close()


def test_async_writes_are_snapshots_of_the_call():
    """Files written behind the step hold the state at the call, whatever
    steps follow before they reach the disk."""
    sc = scenes.dam_break_3d(fluid=(10, 8, 12), box=(20, 8, 16), seed=3)
    a = M.Solver(sc.params, sc.header, sc.type, sc.xyz, sc.vel, dim=3)
    b = M.Solver(sc.params, sc.header, sc.type, sc.xyz, sc.vel, dim=3)
    with tempfile.TemporaryDirectory() as td:
        for k in range(4):
            a.step(7)
            a.compute_virial()
            a.write_vtk_async(os.path.join(td, "a%d.vtk" % k))
            a.write_prof_async(os.path.join(td, "a%d.prof" % k))
        a.step(5)
        a.output_wait()
        for k in range(4):
            b.step(7)
            b.compute_virial()
            hv, hp = _host_bytes(b, td, b.info()["time"])
            assert open(os.path.join(td, "a%d.vtk" % k), "rb").read() == hv, k
            assert open(os.path.join(td, "a%d.prof" % k), "rb").read() == hp, k
    a.close()
    b.close()


def test_write_failure_is_reported_and_context_survives():
    sc = scenes.dam_break_3d(fluid=(6, 6, 8), box=(12, 8, 12), seed=1)
    s = M.Solver(sc.params, sc.header, sc.type, sc.xyz, sc.vel, dim=3)
    with tempfile.TemporaryDirectory() as td:
        s.write_vtk_async(os.path.join(td, "missing_dir", "x.vtk"))
        with pytest.raises(M.MphError):
            s.output_wait()
        s.step(3)
        s.write_prof(os.path.join(td, "ok.prof"))
        assert os.path.getsize(os.path.join(td, "ok.prof")) > 0
    s.close()


def test_text_buffers_reused():
    sc = scenes.dam_break_3d(fluid=(4, 4, 4), box=(10, 8, 10), seed=2)
    s = M.Solver(sc.params, sc.header, sc.type, sc.xyz, sc.vel, dim=3)
    with tempfile.TemporaryDirectory() as td:
        s.write_vtk(os.path.join(td, "a.vtk"))
        s.write_vtk(os.path.join(td, "b.vtk"))  # both text buffers in turn
        s.write_vtk(os.path.join(td, "c.vtk"))
        assert open(os.path.join(td, "a.vtk"), "rb").read() == open(os.path.join(td, "c.vtk"), "rb").read()
    assert M.format_e([]) == b""
    s.close()


def test_cli_output_schedule_writes_behind_the_step():
    """The drop-in executable (same arguments as MphExplicit) writes its *.prof
    and *.vtk files behind the step; every file equals the host writers' bytes
    on the FP64 state of that step, on the reference's schedule
    (main.cpp:374-452)."""
    import re
    import subprocess
    from tests.common import GoldenCase
    case = GoldenCase("square_drop_skip")
    exe = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "mphexplicit_b200", "bin",
                       "mph_b200")
    with tempfile.TemporaryDirectory() as td:
        text = open(case.data).read()
        for key, val in (("OutputInterval", "1.0e-2"), ("VtkOutputInterval", "5.0e-3"), ("EndTime", "3.0e-2")):
            text = re.sub(r"^%s\s+\S+" % key, "%s %s" % (key, val), text, flags=re.M)
        data = os.path.join(td, "case.data")
        open(data, "w").write(text)
        r = subprocess.run([exe, data, case.grid, "p%03d.prof", "v%03d.vtk", "run.log", "1", "--dim=%d" % case.dim],
                           cwd=td, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stdout + r.stderr
        p = M.read_data_file(data)
        g = M.read_grid_file(case.grid)
        s = M.Solver(p, g.header, g.type, g.xyz, g.vel, dim=case.dim)
        t, dt, out_next, vtk_next, istep = g.header.time, p.dt, 0.0, 0.0, int(g.header.time / p.dt)
        checked = 0
        while t < p.end_time + 1.0e-5 * dt:
            if t + 1.0e-5 * dt >= out_next:
                _, hp = _host_bytes(s, td, t)
                assert open(os.path.join(td, "p%03d.prof" % istep), "rb").read() == hp, istep
                out_next += p.output_interval
                checked += 1
            s.step(1)
            if t + 1.0e-5 * dt >= vtk_next:
                s.compute_virial()
                hv, _ = _host_bytes(s, td, t)
                assert open(os.path.join(td, "v%03d.vtk" % istep), "rb").read() == hv, istep
                vtk_next += p.vtk_output_interval
                checked += 1
            t += dt
            istep += 1
        assert checked >= 9
        s.close()
