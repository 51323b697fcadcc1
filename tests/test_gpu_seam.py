"""The MPLAPACK seam: the reference's own sdpa_dd with its Rgemm, Rpotrf and
Rtrsv replaced by sdpa-dd_b200/bindings/mplapack_sddd.cpp (forwarding to
sddd_Rgemm, sddd_Rpotrf and sddd_Rtrsv on the GPU), built by oracle/Makefile
as oracle/_ref/sdpa_dd_sddd, against the stock reference binary
(oracle/_ref/sdpa_dd) on the same files, one OpenMP thread each.

The kernels keep MPLAPACK's per-entry operation order, so the two runs must
print the same iterations, the same 32-digit objectives and the same result
file, line for line, apart from the timing lines.  Every dense Cholesky,
triangular solve and matrix product of these solves (the Schur matrix's
factor, the inverses of X and Z, the block products of Lal::multiply and
the ones inside the eigenvalue routines) runs on the GPU."""
import os
import re
import subprocess

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

SEAM_BIN = ROOT / "oracle" / "_ref" / "sdpa_dd_sddd"
REF_BIN = ROOT / "oracle" / "_ref" / "sdpa_dd"


def _cases():
    import importlib.util
    spec = importlib.util.spec_from_file_location("mk", ROOT / "tests" / "golden" / "make_golden.py")
    mk = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mk)
    return mk.CASES, mk.P


CASES, P = _cases()
# lines that differ between two runs of one binary: clocks, timings, the
# output file's name
TIMING = re.compile(r"(?i)(time|start at|end at|^out\s+is|=\s+[0-9.e+-]+,\s+[0-9.e+-]+\s*$)")


def _run(exe, data, param, out):
    r = subprocess.run([str(exe), "-ds", str(data), "-o", str(out), "-p", param], capture_output=True, text=True, timeout=900,
                       env=dict(os.environ, OMP_NUM_THREADS="1"))
    assert r.returncode == 0, (exe.name, r.returncode, r.stderr[-2000:])
    return r.stdout, out.read_text()


def _strip(text):
    return [ln for ln in text.splitlines() if not TIMING.search(ln) and ln.strip()]


@pytest.mark.parametrize("name", ["dense_n12_m20", "theta_nv24", "maxcut_n30", "control_9_6_m25"])
def test_reference_with_gpu_seam_matches_stock_reference(name, workdir):
    if not SEAM_BIN.exists() or not REF_BIN.exists():
        pytest.skip("oracle/_ref/sdpa_dd_sddd not built (make -C oracle ref)")
    make, eps = CASES[name]
    data = workdir / f"seam_{name}.dat-s"
    data.write_text(make())
    param = P.write_param(str(workdir / f"seam_{name}.param"), eps=eps)
    out_seam, res_seam = _run(SEAM_BIN, data, param, workdir / f"seam_{name}.gpu.result")
    out_ref, res_ref = _run(REF_BIN, data, param, workdir / f"seam_{name}.ref.result")
    for key in ("objValPrimal = ", "objValDual   = "):
        a = re.search(re.escape(key) + r"(\S+)", out_seam).group(1)
        b = re.search(re.escape(key) + r"(\S+)", out_ref).group(1)
        assert a == b, (key, a, b)
    ra, rb = _strip(res_seam), _strip(res_ref)
    assert len(ra) == len(rb), (len(ra), len(rb))
    diff = [(x, y) for x, y in zip(ra, rb) if x != y]
    assert not diff, diff[:5]
    assert "phase.value = " in res_seam
