"""Regenerate the end-to-end golden fixtures from the reference build.

    python tests/golden/make_golden.py

Writes solves.json: for each seeded workload below, the reference's
(oracle/_ref/sdpa_dd, one OpenMP thread) phase, iteration count and the two
objective values as printed on stdout (32 digits, QD's dd output) and in
the result file (16 digits), and its mu after every pass of the main loop
(oracle/_ref/libsdpadd_ref.so stepped through ref_step).

The reference's dd reductions (Rdot, Rgemv, the inner products) combine
OpenMP partial sums in arrival order, so with more than one thread its
trajectory, final phase and iteration count vary from run to run once mu
nears the dd noise floor.  The same workloads are therefore also run with
VARIANT_THREADS threads, each VARIANT_REPEATS times: the fixture keeps each
run's phase, iteration count and objectives, and per pass the largest
relative distance of a run's mu from the one-thread mu ("mu_spread").

Needs oracle/_ref built from the reference sources (make -C oracle ref);
the GPU tests only read the JSON.
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


VARIANT_THREADS = (2, 3, 4, 8)
VARIANT_REPEATS = 2


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


def trajectory(name: str) -> list:
    """mu (hi, lo) after every pass of the reference's main loop, stepped in
    this process through oracle/_ref/libsdpadd_ref.so (ref_step returns 0
    while the loop goes on)."""
    import ctypes

    import numpy as np
    lib = ctypes.CDLL(str(ROOT / "oracle" / "_ref" / "libsdpadd_ref.so"))
    lib.ref_open.restype = ctypes.c_void_p
    make, eps = CASES[name]
    mus = []
    with tempfile.TemporaryDirectory() as td:
        data = pathlib.Path(td) / f"{name}.dat-s"
        data.write_text(make())
        param = P.write_param(str(pathlib.Path(td) / f"{name}.param"), eps=eps)
        h = ctypes.c_void_p(lib.ref_open(str(data).encode(), param.encode(), ctypes.c_double(1.2)))
        out = np.zeros(2, np.float64)
        try:
            while lib.ref_step(h) == 0:
                lib.ref_scalar(h, 0, out.ctypes.data_as(ctypes.c_void_p))
                mus.append([float(out[0]), float(out[1])])
        finally:
            lib.ref_close(h)
    return mus


def _run(name, data, param, res, threads):
    ref = ROOT / "oracle" / "_ref" / "sdpa_dd"
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    r = subprocess.run([str(ref), "-ds", str(data), "-o", str(res), "-p", param], capture_output=True, text=True, env=env, check=True)
    d = parse(r.stdout, res.read_text())
    t = subprocess.run([sys.executable, __file__, "--trajectory", name], capture_output=True, text=True, env=env, check=True)
    d["mu_trajectory"] = json.loads(t.stdout.strip().splitlines()[-1])  # the library prints a banner first
    return d


def _rel(a, b):
    from decimal import Decimal
    a, b = Decimal(a[0]) + Decimal(a[1]), Decimal(b[0]) + Decimal(b[1])
    return float(abs(a - b) / max(abs(b), Decimal("1e-300")))


def main():
    out = {}
    with tempfile.TemporaryDirectory() as td:
        td = pathlib.Path(td)
        for name, (make, eps) in CASES.items():
            data = td / f"{name}.dat-s"
            data.write_text(make())
            param = P.write_param(str(td / f"{name}.param"), eps=eps)
            res = td / f"{name}.result"
            one = _run(name, data, param, res, 1)
            variants = [dict(_run(name, data, param, res, t), threads=t) for t in VARIANT_THREADS for _ in range(VARIANT_REPEATS)]
            mu1 = one["mu_trajectory"]
            spread = []
            for k in range(min(len(mu1), *(len(v["mu_trajectory"]) for v in variants))):
                spread.append(max(_rel(v["mu_trajectory"][k], mu1[k]) for v in variants))
            keep = ("threads", "phase", "iterations", "objValPrimal32", "objValDual32")
            out[name] = dict(one, eps=eps, mu_spread=spread, variants=[{k: v[k] for k in keep} for v in variants])
            print(name, out[name]["phase"], out[name]["iterations"], sorted({(v["phase"], v["iterations"]) for v in variants}),
                  file=sys.stderr)
    (HERE / "solves.json").write_text(json.dumps(out, indent=1, sort_keys=True) + "\n")


if __name__ == "__main__":
    if len(sys.argv) == 3 and sys.argv[1] == "--trajectory":
        print(json.dumps(trajectory(sys.argv[2])))
    else:
        main()
