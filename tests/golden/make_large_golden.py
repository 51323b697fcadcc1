"""Golden fixtures of the reference build at the full-size workloads.

    python tests/golden/make_large_golden.py [NAME ...]

Writes large_solves.json: for each workload below (the max-cut n = 500, the
control-shaped blocks 100 + 50 with m = 1326 and a theta-shaped m = 3571
problem), the reference's (oracle/_ref/libsdpadd_ref.so, stepped through
ref_step as pinpal's main loop) mu after every pass, its final phase and
iteration count and the two objectives as printed (the reference's
REVERSE_PRIMAL_DUAL output: objValPrimal = -objValDual of its internal
problem), as dd pairs.  One run with one OpenMP thread is the parity
reference; VARIANTS further runs with more threads measure the reference's
own run-to-run spread (its OpenMP reductions add partial sums in arrival
order), as in make_golden.py.

The one-thread control-shaped run takes about 90 s per pass on one core, so
the whole file takes over an hour; the runs go in parallel.  Needs
oracle/_ref (make -C oracle ref); the GPU tests only read the JSON.
"""
import ctypes
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

CASES = {
    # max-cut shape, one dense block n = 500, m = 500, F3 (Hadamard) Schur
    "maxcut_n500": (lambda: P.maxcut(n=500, p=0.02, seed=1), 1e-25),
    # control shape, dense blocks 100 + 50, m = 1326, F1 Schur
    "control_100_50_m1326": (lambda: P.control_like(sizes=(100, 50), m=1326, seed=3), 1e-25),
    # theta shape, 120 vertices, p = 0.5: m = 3571, F3 + F2 Schur
    "theta_nv120": (lambda: P.theta(nv=120, p=0.5, seed=2), 1e-25),
}
# (threads) of the runs beside the one-thread run
# theta_nv120 ends where its mu stalls near 1.2e-25: the runs part in phase
# (pFEAS after a too-small step, or pdOPT) and iteration count, so it has
# more of them
VARIANTS = {"maxcut_n500": (2, 4, 3), "control_100_50_m1326": (2,), "theta_nv120": (2, 4, 3, 6, 8)}

PHASES = ["noINFO", "pFEAS", "dFEAS", "pdFEAS", "pdINF", "pFEAS_dINF", "pINF_dFEAS", "pdOPT", "pUNBD", "dUNBD"]
# Phase::reverse (sdpa_parts.cpp:956-990), applied before printing
REVERSED = {"pFEAS": "dFEAS", "dFEAS": "pFEAS", "pFEAS_dINF": "pINF_dFEAS", "pINF_dFEAS": "pFEAS_dINF", "pUNBD": "dUNBD", "dUNBD": "pUNBD"}


def run_one(name: str) -> dict:
    """One reference solve of `name` in this process (OMP_NUM_THREADS from
    the environment)."""
    import numpy as np
    lib = ctypes.CDLL(str(ROOT / "oracle" / "_ref" / "libsdpadd_ref.so"))
    lib.ref_open.restype = ctypes.c_void_p
    make, eps = CASES[name]
    out = np.zeros(2, np.float64)

    def scalar(h, what):
        lib.ref_scalar(h, what, out.ctypes.data_as(ctypes.c_void_p))
        return [float(out[0]), float(out[1])]

    with tempfile.TemporaryDirectory() as td:
        data = pathlib.Path(td) / f"{name}.dat-s"
        data.write_text(make())
        param = P.write_param(str(pathlib.Path(td) / f"{name}.param"), eps=eps)
        h = ctypes.c_void_p(lib.ref_open(str(data).encode(), param.encode(), ctypes.c_double(1.2)))
        lib.ref_set_capture(h, 0)
        mus = []
        try:
            while True:
                rc = lib.ref_step(h)
                if rc != 0:
                    break
                mus.append(scalar(h, 0))
            phase = PHASES[lib.ref_phase(h)]
            objP, objD = scalar(h, 7), scalar(h, 8)
            res = dict(stop=rc, phase=REVERSED.get(phase, phase), iterations=int(lib.ref_iteration(h)), mu_trajectory=mus,
                       objValPrimal=[-objD[0], -objD[1]], objValDual=[-objP[0], -objP[1]], threads=int(os.environ.get("OMP_NUM_THREADS", "1")))
        finally:
            lib.ref_close(h)
    return res


def _rel(a, b):
    from decimal import Decimal
    a, b = Decimal(a[0]) + Decimal(a[1]), Decimal(b[0]) + Decimal(b[1])
    return float(abs(a - b) / max(abs(b), Decimal("1e-300")))


def main(names):
    procs = []
    for name in names:
        for t in (1,) + VARIANTS[name]:
            env = dict(os.environ, OMP_NUM_THREADS=str(t))
            p = subprocess.Popen([sys.executable, __file__, "--run", name], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True, env=env)
            procs.append((name, t, p))
    runs = {}
    for name, t, p in procs:
        stdout, _ = p.communicate()
        if p.returncode != 0:
            raise RuntimeError(f"{name} with {t} threads failed")
        runs.setdefault(name, []).append(json.loads(stdout.strip().splitlines()[-1]))
    path = HERE / "large_solves.json"
    out = json.loads(path.read_text()) if path.exists() else {}
    for name in names:
        one = next(r for r in runs[name] if r["threads"] == 1)
        variants = [r for r in runs[name] if r is not one]
        mu1 = one["mu_trajectory"]
        spread = []
        for k in range(min([len(mu1)] + [len(v["mu_trajectory"]) for v in variants])):
            spread.append(max([_rel(v["mu_trajectory"][k], mu1[k]) for v in variants], default=0.0))
        keep = ("threads", "phase", "iterations", "objValPrimal", "objValDual")
        out[name] = dict(one, eps=CASES[name][1], mu_spread=spread, variants=[{k: v[k] for k in keep} for v in variants])
        print(name, one["phase"], one["iterations"], sorted({(v["phase"], v["iterations"]) for v in variants}), file=sys.stderr)
    path.write_text(json.dumps(out, indent=1, sort_keys=True) + "\n")


if __name__ == "__main__":
    if len(sys.argv) == 3 and sys.argv[1] == "--run":
        print(json.dumps(run_one(sys.argv[2])))
    else:
        main(sys.argv[1:] or list(CASES))
