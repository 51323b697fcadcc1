"""Full-precision point files (sddd_write_point, the command line's -wd / -ws).

The reference writes only the high double of each result; a solve that
should continue from where another stopped (a warm start, a checkpoint)
needs the whole dd point.  sddd_write_point writes it as an initial-point
file (34 significant digits, the reader's layout); read back through
sddd_read_initial_point it must give the same point to dd accuracy, in the
dense and the sparse layout, and the command line's -ws file must equal the
C ABI's byte for byte (the solves are deterministic)."""
import ctypes
import importlib
import subprocess

import numpy as np
import pytest

from conftest import load_pkg

pytestmark = pytest.mark.gpu


def _dd(a):
    return a["hi"].astype(np.longdouble) + a["lo"].astype(np.longdouble)


@pytest.fixture(scope="module")
def files(tmp_path_factory):
    load_pkg()
    P = importlib.import_module("sdpa_dd_b200.problems")
    td = tmp_path_factory.mktemp("pointio")
    data = td / "maxcut.dat-s"
    data.write_text(P.maxcut(n=40, p=0.3, seed=3))
    param = P.write_param(str(td / "param.sdpa"), eps=1e-25)
    return data, param, td


def _final_point(sddd, data, par, dump=None, sparse=1):
    with sddd.Context(0) as c:
        c.read_problem(data)
        r = c.solve(par)
        assert r.phase == sddd.PHASES.index("pdOPT")
        if dump is not None:
            assert c.L.sddd_write_point(c.h, str(dump).encode(), sparse) == 0, c.L.sddd_last_error(c.h)
        return {w: c.get(w) for w in ("X", "Z", "y")}


@pytest.mark.parametrize("sparse", [0, 1])
def test_written_point_reads_back(files, sparse):
    sddd = load_pkg()
    data, param, td = files
    par = sddd.param(param)
    dump = td / f"final_{sparse}.txt"
    ref = _final_point(sddd, data, par, dump, sparse)
    first = dump.read_text().splitlines()[0]
    assert first.startswith("{") and first.count(",") == len(ref["y"]) - 1
    with sddd.Context(0) as c:
        c.read_problem(data)
        assert c.L.sddd_read_initial_point(c.h, str(dump).encode(), sparse, par.lambdaStar) == 0
        assert c.L.sddd_solver_start(c.h, ctypes.byref(par)) == 0  # loads the initial point
        for w in ("X", "Z", "y"):
            got, want = _dd(c.get(w)), _dd(ref[w])
            scale = max(float(np.max(np.abs(want))), 1e-300)
            err = float(np.max(np.abs(got - want)))
            # 34 digits and QD's reader: a few units of 2^-104 of the largest entry
            assert err <= 2.0 ** -100 * scale, (w, err, scale)


def test_command_line_point_file_equals_c_abi(files):
    sddd = load_pkg()
    data, param, td = files
    par = sddd.param(param)
    api = td / "api.txt"
    _final_point(sddd, data, par, api, 1)
    cli = td / "cli.txt"
    r = subprocess.run([str(sddd.BIN_PATH), "-ds", str(data), "-o", str(td / "cli.result"), "-p", param, "-ws", str(cli)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert cli.read_text() == api.read_text()
