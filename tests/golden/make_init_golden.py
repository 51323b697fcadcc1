"""Regenerate the initial-point fixtures from the reference build.

    python tests/golden/make_init_golden.py

For a max-cut-shaped SDP (the shape on which the reference's runs agree
whatever the thread count) it writes a strictly feasible starting point,
x_i = ceil(lambda_max(L) / 4) + 1, X = diag(x) - L/4, Y = I (all dyadic, so
every reader parses the same dd values), as a dense init file (init_dense.txt,
for -id) and a sparse one (init_sparse.txt, for -is), runs oracle/_ref/sdpa_dd
on each with 1 and 4 OpenMP threads, and records the phase, iteration count
and the 32-digit objectives in init_point.json.  The GPU tests read only
these files.
"""
import importlib.util
import json
import os
import pathlib
import subprocess
import sys
import tempfile

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parents[1]
spec = importlib.util.spec_from_file_location("problems", ROOT / "sdpa-dd_b200" / "problems.py")
P = importlib.util.module_from_spec(spec)
spec.loader.exec_module(P)
spec = importlib.util.spec_from_file_location("mk", HERE / "make_golden.py")
MK = importlib.util.module_from_spec(spec)
spec.loader.exec_module(MK)

N, PROB, SEED, EPS = 40, 0.15, 21, 1e-25


def laplacian(n=N, p=PROB, seed=SEED):
    """The Laplacian P.maxcut draws for (n, p, seed)."""
    rng = np.random.default_rng(seed)
    A = np.triu(rng.random((n, n)) < p, 1)
    A = A | A.T
    return np.diag(A.sum(axis=1).astype(float)) - A.astype(float)


def init_point():
    L = laplacian()
    x = np.full(N, float(np.ceil(np.linalg.eigvalsh(L).max() / 4.0)) + 1.0)
    return x, np.diag(x) - L / 4.0, np.eye(N)


def fmt(v):
    return repr(float(v))


def write_init(path_dense, path_sparse):
    x, X, Y = init_point()
    head = "{" + ", ".join(fmt(v) for v in x) + "}\n"
    with open(path_dense, "w") as f:
        f.write(head)
        for M in (X, Y):
            for i in range(N):
                f.write(" ".join(fmt(v) for v in M[i]) + "\n")
    with open(path_sparse, "w") as f:
        f.write(head)
        for target, M in ((1, X), (2, Y)):
            for i in range(N):
                for j in range(i, N):
                    if M[i, j] != 0.0:
                        f.write(f"{target} 1 {i + 1} {j + 1} {fmt(M[i, j])}\n")


def main():
    exe = ROOT / "oracle" / "_ref" / "sdpa_dd"
    if not exe.exists():
        sys.exit("build the reference first: make -C oracle ref")
    dense, sparse = HERE / "init_dense.txt", HERE / "init_sparse.txt"
    write_init(dense, sparse)
    out = {"n": N, "p": PROB, "seed": SEED, "eps": EPS, "runs": {}}
    with tempfile.TemporaryDirectory() as td:
        data = pathlib.Path(td) / "maxcut.dat-s"
        data.write_text(P.maxcut(n=N, p=PROB, seed=SEED))
        param = P.write_param(str(pathlib.Path(td) / "param.sdpa"), eps=EPS)
        for flag, path in (("-id", dense), ("-is", sparse)):
            runs = []
            for threads in (1, 4):
                res = pathlib.Path(td) / "out.result"
                r = subprocess.run([str(exe), "-ds", str(data), flag, str(path), "-o", str(res), "-p", param], capture_output=True, text=True,
                                   env=dict(os.environ, OMP_NUM_THREADS=str(threads)), check=True)
                d = MK.parse(r.stdout, res.read_text())
                d["threads"] = threads
                runs.append(d)
            out["runs"][flag] = runs
    (HERE / "init_point.json").write_text(json.dumps(out, indent=1) + "\n")
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    main()
