"""Regenerate the end-to-end golden fixtures from the reference build.

    OMP_NUM_THREADS=1 python tests/golden/make_golden.py

Writes solves.json: for each seeded workload below, the reference's
(oracle/_ref/sdpa_dd, one OpenMP thread) phase, iteration count and the two
objective values as printed on stdout (32 digits, QD's dd output) and in
the result file (16 digits).  Needs oracle/_ref built from the reference
sources (make -C oracle ref); the GPU tests only read the JSON.
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

CASES = {
    "dense_n12_m20": (lambda: P.dense_random(n=12, m=20, seed=10), 1e-25),
    "maxcut_n30": (lambda: P.maxcut(n=30, p=0.2, seed=11), 1e-25),
    "theta_nv24": (lambda: P.theta(nv=24, p=0.5, seed=12), 1e-25),
    "control_9_6_m25": (lambda: P.control_like(sizes=(9, 6), m=25, seed=13), 1e-25),
    "dense_n50_m40": (lambda: P.dense_random(n=50, m=40, seed=14), 1e-25),
    "dense_n50_m100": (lambda: P.dense_random(n=50, m=100, seed=0), 1e-25),
    "maxcut_n60_eps20": (lambda: P.maxcut(n=60, p=0.1, seed=15), 1e-20),
    "dense_n8_m5_eps30": (lambda: P.dense_random(n=8, m=5, seed=16), 1e-30),
}


def parse(stdout: str, result: str) -> dict:
    d = {}
    d["phase"] = re.search(r"phase.value = (\w+)", result).group(1)
    d["iterations"] = int(re.search(r"Iteration = (\d+)", result).group(1))
    d["objValPrimal32"] = re.search(r"objValPrimal = (\S+)", stdout).group(1)
    d["objValDual32"] = re.search(r"objValDual   = (\S+)", stdout).group(1)
    d["objValPrimal16"] = re.search(r"objValPrimal = (\S+)", result).group(1)
    d["objValDual16"] = re.search(r"objValDual   = (\S+)", result).group(1)
    d["mu"] = re.search(r"\n\s+mu = (\S+)", result).group(1)
    d["relative_gap"] = re.search(r"relative gap = (\S+)", result).group(1)
    return d


def main():
    ref = ROOT / "oracle" / "_ref" / "sdpa_dd"
    env = dict(os.environ, OMP_NUM_THREADS="1")
    out = {}
    with tempfile.TemporaryDirectory() as td:
        td = pathlib.Path(td)
        for name, (make, eps) in CASES.items():
            data = td / f"{name}.dat-s"
            data.write_text(make())
            param = P.write_param(str(td / f"{name}.param"), eps=eps)
            res = td / f"{name}.result"
            r = subprocess.run([str(ref), "-ds", str(data), "-o", str(res), "-p", param], capture_output=True, text=True, env=env, check=True)
            out[name] = dict(parse(r.stdout, res.read_text()), eps=eps)
            print(name, out[name]["phase"], out[name]["iterations"], out[name]["objValPrimal32"], file=sys.stderr)
    (HERE / "solves.json").write_text(json.dumps(out, indent=1, sort_keys=True) + "\n")


if __name__ == "__main__":
    main()
