"""Fixtures of the reference build on its sparse Schur path.

    python tests/golden/make_sparse_golden.py

Writes sparse_schur.json: for each problem below (problems.chain_blocks:
SDP blocks in a chain, constraints numbered in a random order, optionally
with an LP block) the reference's (oracle/_ref/sdpa_dd) Schur form line,
phase, iteration count and 32-digit objectives with 1 and 4 OpenMP threads
at epsilon 1e-20.  Every problem has m > 100, more than 5 blocks and a
sparse aggregate pattern, so the reference takes its sparse Schur path
(Chordal::ordering_bMat, sdpa_chordal.cpp:348-438) with the oracle's
minimum-degree ordering in place of SPOOLES (oracle/spooles_shim.cpp).
The GPU tests read only the JSON.
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

CASES = {
    "chain40": lambda: P.chain_blocks(nblocks=40, n=10, per=4, overlap=2, q=0, seed=9),
    "chain40_lp30": lambda: P.chain_blocks(nblocks=40, n=10, per=4, overlap=2, q=30, seed=12),
    "chain150": lambda: P.chain_blocks(nblocks=150, n=8, per=6, overlap=3, q=0, seed=21),
    # the bench's sparse-Schur workload (m = 5990)
    "chain200_n20": lambda: P.chain_blocks(nblocks=200, n=20, per=20, overlap=10, q=0, seed=31),
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
                d["sparse"] = "SPARSE computation" in r.stdout
                runs.append(d)
            out["cases"][name] = runs
            print(name, [(d["phase"], d["iterations"], d["sparse"]) for d in runs], file=sys.stderr)
    (HERE / "sparse_schur.json").write_text(json.dumps(out, indent=1) + "\n")


if __name__ == "__main__":
    main()
