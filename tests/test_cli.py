"""The drop-in executable's failures before any device work (CPU only):
a missing *.data or *.grid ends with status 1 and a line naming the file and
the reason, in the log file and on stderr; an unknown option ends with
status 2 and the usage."""
import os
import subprocess
import tempfile

from tests.common import GoldenCase

EXE = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "mphexplicit_b200", "bin",
                   "mph_b200")


def _run(args, cwd):
    return subprocess.run([EXE] + args, cwd=cwd, capture_output=True, text=True, timeout=120)


def test_missing_files_and_unknown_options():
    case = GoldenCase("square_drop_skip")
    with tempfile.TemporaryDirectory() as td:
        missing = os.path.join(td, "missing.data")
        r = _run([missing, case.grid, "p%03d.prof", "v%03d.vtk", "run.log", "1", "--dim=2"], td)
        assert r.returncode == 1
        assert missing in r.stderr and "could not be opened" in r.stderr
        assert missing in open(os.path.join(td, "run.log")).read()
        missing = os.path.join(td, "missing.grid")
        r = _run([case.data, missing, "p%03d.prof", "v%03d.vtk", "run.log", "1", "--dim=2"], td)
        assert r.returncode == 1 and missing in r.stderr
        r = _run(["--mode=bogus"], td)
        assert r.returncode == 2 and "usage" in r.stderr
        assert not os.path.exists(os.path.join(td, "output.vtk"))  # nothing was written
