"""Fixtures of the reference build for problems with many blocks.

    python tests/golden/make_blocks_golden.py

Writes many_blocks.json: for each problem below (problems.blocks_with_lp:
an SDP block of order 30 with an LP block of 200 entries; 80 small dense
SDP blocks; 70 small SDP blocks with an LP block of 100 entries; all with m
<= 100, where the reference always takes its dense Schur path) the
reference's (oracle/_ref/sdpa_dd) phase, iteration count and 32-digit
objectives with 1 and 4 OpenMP threads, at epsilon 1e-20 (where both thread
counts end in pdOPT after the same number of iterations).  Each LP entry and
each small block is one more per-block result (inner products, step-length
eigenvalues), so these problems hold far more blocks than the solver's
fixed-size scratch of earlier versions covered.  The GPU tests read only the
JSON.
"""
import importlib.util
import json
import os
import pathlib
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

EPS = 1e-20


def _sizes(seed, count):
    import numpy as np
    return [int(n) for n in np.random.default_rng(seed).integers(2, 9, count)]


CASES = {
    "lp_q200": lambda: P.blocks_with_lp(sizes=(30,), q=200, m=40, seed=8),
    "blocks80": lambda: P.blocks_with_lp(sizes=_sizes(21, 80), q=0, m=60, seed=21),
    "blocks70_lp100": lambda: P.blocks_with_lp(sizes=_sizes(22, 70), q=100, m=60, seed=22),
}


def main():
    exe = ROOT / "oracle" / "_ref" / "sdpa_dd"
    if not exe.exists():
        sys.exit("build the reference first: make -C oracle ref")
    out = {"eps": EPS, "cases": {}}
    with tempfile.TemporaryDirectory() as td:
        param = P.write_param(str(pathlib.Path(td) / "param.sdpa"), eps=EPS)
        for name, make in CASES.items():
            data = pathlib.Path(td) / f"{name}.dat-s"
            data.write_text(make())
            runs = []
            for threads in (1, 4):
                res = pathlib.Path(td) / "out.result"
                r = subprocess.run([str(exe), "-ds", str(data), "-o", str(res), "-p", param], capture_output=True, text=True,
                                   env=dict(os.environ, OMP_NUM_THREADS=str(threads)), check=True)
                d = MK.parse(r.stdout, res.read_text())
                d["threads"] = threads
                runs.append(d)
            out["cases"][name] = runs
            print(name, [(d["phase"], d["iterations"]) for d in runs], file=sys.stderr)
    (HERE / "many_blocks.json").write_text(json.dumps(out, indent=1) + "\n")


if __name__ == "__main__":
    main()
