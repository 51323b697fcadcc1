"""Problem dimensions read on the host (sddd_problem_info), no device needed.

A caller sizes its buffers (or a batch its block spaces) from a problem file
before any GPU work; the answer must be what a context reports after
sddd_read_problem, including the LP convention: each LP entry is a trailing
SDP block of order 1."""
import importlib

import pytest

from conftest import load_pkg


def _problems():
    load_pkg()
    return importlib.import_module("sdpa_dd_b200.problems")


def test_lp_entries_are_trailing_order_one_blocks(tmp_path):
    sddd = load_pkg()
    P = _problems()
    path = tmp_path / "lp.dat-s"
    path.write_text(P.with_lp(n=30, q=24, m=40, seed=7))
    m, sizes, space = sddd.problem_info(path)
    assert m == 40 and sizes == [30] + [1] * 24 and space == 30 * 30 + 24


def test_sdp_only_file(tmp_path):
    sddd = load_pkg()
    P = _problems()
    path = tmp_path / "mc.dat-s"
    path.write_text(P.maxcut(n=60, p=0.1, seed=2))
    assert sddd.problem_info(path) == (60, [60], 3600)


def test_several_blocks_and_lp_between_them(tmp_path):
    """LP blocks anywhere in the structure: the SDP blocks keep their order,
    the LP entries follow them in the file's LP order."""
    sddd = load_pkg()
    text = '"mixed"\n2 = mDIM\n4 = nBLOCK\n3 -2 2 -1 = bLOCKsTRUCT\n{1, 1}\n' \
           "0 1 1 1 1.0\n0 2 1 1 1.0\n0 2 2 2 1.0\n0 3 1 1 1.0\n0 4 1 1 1.0\n1 1 1 1 1.0\n2 3 2 2 1.0\n"
    path = tmp_path / "mixed.dat-s"
    path.write_text(text)
    assert sddd.problem_info(path) == (2, [3, 2, 1, 1, 1], 9 + 4 + 3)


def test_missing_file_is_an_error(tmp_path):
    sddd = load_pkg()
    with pytest.raises(sddd.SdddError, match="Cannot open"):
        sddd.problem_info(tmp_path / "nope.dat-s")
