"""Regenerate the LP-block fixture from the reference build.

    python tests/golden/make_lp_golden.py

For an SDP with an LP block (problems.with_lp: an SDP block of order 30 and
24 LP entries, m = 40, strictly feasible on both sides; epsilon 1e-20,
where the reference ends in pdOPT whatever the thread count, while at 1e-25
its LP slacks hit exact zeros first and the runs stop in pFEAS after a
thread-dependent number of iterations) it runs
oracle/_ref/sdpa_dd with 1 and 4 OpenMP threads and records the phase,
iteration count, the 32-digit objectives and the LP lists of the final xMat
and yMat (the result file's hi parts) in lp_block.json.  The GPU tests read
only that file.
"""
import importlib.util
import json
import os
import pathlib
import re
import subprocess
import sys
import tempfile

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parents[1]
spec = importlib.util.spec_from_file_location("problems", ROOT / "sdpa-dd_b200" / "problems.py")
P = importlib.util.module_from_spec(spec)
spec.loader.exec_module(P)
spec = importlib.util.spec_from_file_location("mk", HERE / "make_golden.py")
MK = importlib.util.module_from_spec(spec)
spec.loader.exec_module(MK)

N, Q, M, SEED, EPS = 30, 24, 40, 7, 1e-20


def lp_lists(result: str) -> dict:
    """The LP block's list in xMat and in yMat: the line after the SDP
    block that is a single {v,...} list of Q numbers."""
    out = {}
    for name in ("xMat", "yMat"):
        part = result.split(f"{name} = \n", 1)[1]
        lists = [ln for ln in part.splitlines() if re.fullmatch(r"\{[^{}]*\}", ln.strip()) and ln.count(",") == Q - 1]
        out[name] = [float(v) for v in lists[0].strip("{} ").split(",")]
    return out


def main():
    exe = ROOT / "oracle" / "_ref" / "sdpa_dd"
    if not exe.exists():
        sys.exit("build the reference first: make -C oracle ref")
    out = {"n": N, "q": Q, "m": M, "seed": SEED, "eps": EPS, "runs": []}
    with tempfile.TemporaryDirectory() as td:
        data = pathlib.Path(td) / "lp.dat-s"
        data.write_text(P.with_lp(n=N, q=Q, m=M, seed=SEED))
        param = P.write_param(str(pathlib.Path(td) / "param.sdpa"), eps=EPS)
        for threads in (1, 4):
            res = pathlib.Path(td) / "out.result"
            r = subprocess.run([str(exe), "-ds", str(data), "-o", str(res), "-p", param], capture_output=True, text=True,
                               env=dict(os.environ, OMP_NUM_THREADS=str(threads)), check=True)
            text = res.read_text()
            d = MK.parse(r.stdout, text)
            d["threads"] = threads
            d.update(lp_lists(text))
            out["runs"].append(d)
    (HERE / "lp_block.json").write_text(json.dumps(out, indent=1) + "\n")
    print(json.dumps({k: v for k, v in out["runs"][0].items() if k not in ("xMat", "yMat")}, indent=1))


if __name__ == "__main__":
    main()
