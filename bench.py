#!/usr/bin/env python
"""Newton-iteration throughput of the dd interior-point method on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: the Lovasz-theta-shaped SDP with 200 vertices and edge probability
0.5 (seed 2: 9979 edges, m = 9980 constraints, one 200 x 200 block), the
configuration the headline target is quoted on.  A step is one full pass of
the reference's main loop (sdpa_main.cpp:294-376): predictor and corrector
Newton directions (Schur build, dd Cholesky of the 9980 x 9980 Schur matrix,
solves), step lengths, update and residuals.  The metric is dd-GFLOP/s of
the Schur build plus the Cholesky of B (the algorithmic counts of
sddd_work: m^3/3 for the Cholesky), over the whole step time.

The headline runs the tensor-core split form (--tc, default 16 slices: the
Cholesky trailing updates as INT8 slice products on tcgen05); the same
passes in the plain dd form (the reference's operation order, bit for bit)
are timed beside it ("plain_dd"), and both forms solve the problem from the
standard initial point to relative gap 1e-25 ("solve_to_gap", wall clock),
as do the max-cut (n = m = 500) and control-shaped (blocks 100 + 50, m =
1326) workloads ("solve_to_gap_other_configs"), each beside the reference
build's own solve of the same file.  The headline passes run with no
per-kernel instrumentation; the kernel breakdown and the roofline come from
a separate, profiled run of the same passes.

One JSON line on rank 0.  Multi-GPU runs are replicas (the single solve
does not shard): every rank solves its own copy, value sums the ranks' work
over the slowest rank's time.  --impl reference times the reference build's
stock main loop (oracle/_ref) on all host cores on the same m = 9980
workload: one pass after one untimed pass (about a minute each).
"""
from __future__ import annotations

import argparse
import ctypes
import datetime
import importlib.util
import json
import os
import pathlib
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = pathlib.Path(__file__).resolve().parent
WORKLOAD = dict(name="theta", nv=200, p=0.5, seed=2)
SMALL_THETA = dict(name="theta", nv=120, p=0.5, seed=2)  # m = 3571
# the other full-size shapes, solved to gap 1e-25 beside the headline
MAXCUT = dict(name="maxcut", n=500, p=0.02, seed=1)  # n = m = 500, F3 Schur
CONTROL = dict(name="control", sizes=(100, 50), m=1326, seed=3)  # F1 Schur
# 200 SDP blocks of order 20 in a chain (m = 5990): the reference's sparse
# Schur path (more than 5 blocks, a sparse aggregate pattern)
CHAIN = dict(name="chain", nblocks=200, n=20, per=20, overlap=10, seed=31)
EPS = 1e-25


def load_pkg():
    if "sdpa_dd_b200" in sys.modules:
        return sys.modules["sdpa_dd_b200"]
    pkg = ROOT / "sdpa-dd_b200"
    spec = importlib.util.spec_from_file_location("sdpa_dd_b200", pkg / "__init__.py", submodule_search_locations=[str(pkg)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["sdpa_dd_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def problems():
    load_pkg()
    import importlib
    return importlib.import_module("sdpa_dd_b200.problems")


def workload_label(w):
    if w["name"] == "theta":
        return f"theta-shaped SDP nv={w['nv']} p={w['p']} seed={w['seed']}"
    if w["name"] == "maxcut":
        return f"max-cut-shaped SDP n={w['n']} p={w['p']} seed={w['seed']}"
    if w["name"] == "chain":
        return (f"chain of {w['nblocks']} SDP blocks of order {w['n']} ({w['per']} own and {w['overlap']} shared constraints per block, "
                f"seed {w['seed']}; sparse Schur)")
    return f"control-shaped SDP blocks {w['sizes']} m={w['m']} seed={w['seed']}"


def write_workload(w, directory):
    P = problems()
    key = "_".join(f"{k}{v}" for k, v in sorted(w.items()) if k != "name").replace(" ", "").replace(",", "-")
    path = pathlib.Path(directory) / f"{w['name']}_{key}.dat-s"
    if not path.exists():
        if w["name"] == "theta":
            text = P.theta(nv=w["nv"], p=w["p"], seed=w["seed"])
        elif w["name"] == "maxcut":
            text = P.maxcut(n=w["n"], p=w["p"], seed=w["seed"])
        elif w["name"] == "chain":
            text = P.chain_blocks(nblocks=w["nblocks"], n=w["n"], per=w["per"], overlap=w["overlap"], seed=w["seed"])
        else:
            text = P.control_like(sizes=w["sizes"], m=w["m"], seed=w["seed"])
        tmp = str(path) + f".tmp{os.getpid()}"
        with open(tmp, "w") as f:
            f.write(text)
        os.replace(tmp, path)
    param = P.write_param(str(pathlib.Path(directory) / "bench.param"), eps=EPS)
    return path, param


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = max(mx, float(r[2]))
                for nm, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def trailing_flops(m, nb=64):
    """dd-flops of the Cholesky trailing updates (lower triangle incl. the
    diagonal, nb multiply-subtracts = 2 nb dd-flops per entry) and their
    launch count."""
    fl, launches = 0.0, 0
    for c0 in range(0, m, nb):
        M = m - c0 - min(nb, m - c0)
        if M > 0:
            fl += float(nb) * M * (M + 1)
            launches += 1
    return fl, launches


def cpu_reference(sample, warmup, steps, threads):
    """Time the reference build's stock main loop (oracle/_ref/sdpa_ref_iter)
    on the host: `warmup` untimed passes, then `steps` timed ones."""
    P = problems()
    exe = ROOT / "oracle" / "_ref" / "sdpa_ref_iter"
    if not exe.exists():
        return None, "oracle/_ref/sdpa_ref_iter is not built"
    workdir = pathlib.Path(tempfile.gettempdir()) / f"sddd_bench_ref_{os.getuid()}"
    workdir.mkdir(exist_ok=True)
    data, param = write_workload(sample, workdir)
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    r = subprocess.run([str(exe), str(data), param, str(warmup), str(steps)], capture_output=True, text=True, env=env)
    if r.returncode != 0:
        return None, f"reference run failed: {r.stderr.strip()[-200:]}"
    out = json.loads(r.stdout.strip().splitlines()[-1])
    secs = out["pass_s"]
    res = {"m": out["m"], "threads": out["threads"], "pass_s": secs, "schur_s": out.get("schur_s"), "chol_s": out.get("chol_s"),
           "setup_s": out.get("setup_s")}
    if sample["name"] == "theta":
        e = P.theta_edges(sample["nv"], sample["p"], sample["seed"])
        schur, chol = P.theta_work(sample["nv"], e)
        res["value"] = (schur + chol) * len(secs) / sum(secs) / 1e9
    return res, None


BATCH = {"count": 256, "seed": 4, "cpu_sample": 8}


def batch_measure(sddd, device, rank, world, args):
    """The batched workload: 256 dense random SDPs (n ~ U[10,80], m ~
    U[20,200], the dense_random construction), every one solved to relative
    gap 1e-25 with the gradient of its optimal value with respect to c, on
    one GPU through sddd_batch_*; beside it the reference build on a seeded
    sample of the same problems, one single-thread process per core."""
    P = problems()
    import importlib
    shard = importlib.import_module("sdpa_dd_b200.shard")
    probs = P.batch(BATCH["count"], seed=BATCH["seed"])
    workdir = pathlib.Path(tempfile.gettempdir()) / f"sddd_batch_{os.getuid()}_{device}"
    workdir.mkdir(exist_ok=True)
    paths = []
    for q, (n, m, text) in enumerate(probs):
        path = workdir / f"b{q}.dat-s"
        if not path.exists():
            path.write_text(text)
        paths.append((path, n, m))
    param_path = P.write_param(str(workdir / "param.sdpa"), eps=EPS, max_iter=200)
    par = sddd.param(param_path)
    # independent problems shard over ranks by work, no data-path exchange
    mine = shard.partition_by_work([shard.work_estimate(m, [n]) for _, n, m in paths], world)[rank]
    with sddd.Batch(device, args.batch_workers) as bt:
        if args.batch_core >= 0 and bt.L.sddd_batch_set_core(bt.h, args.batch_core) != 0:
            raise RuntimeError("sddd_batch_set_core failed")
        for q in mine:
            path, n, m = paths[q]
            bt.add_file(path, m, n * n)
        barrier(world)
        t = time.perf_counter()
        res = bt.solve(par, with_grad=True) if mine else []
        dt = allmax(world, time.perf_counter() - t)
    phases = [sddd.PHASES[r.phase] for r in res]
    n_opt = int(allsum(world, phases.count("pdOPT")))
    counts = {}
    for ph in phases:
        counts[ph] = counts.get(ph, 0) + 1
    out = {"workload": f"{BATCH['count']} dense random SDPs, n ~ U[10,80], m ~ U[20,200], seed {BATCH['seed']}, epsilon {EPS:g}, with d(c.x)/dc",
           "solves_per_s": len(paths) / dt,
           "solves_per_s_basis": "every problem run to the end of its main loop, whatever its final phase (phases below)",
           "pdopt_solves_per_s": n_opt / dt, "pdOPT": n_opt, "seconds": dt, "ranks": world, "workers": args.batch_workers or "default",
           "batched_core": {-1: "default (on)", 0: "off", 1: "on"}[args.batch_core],
           "phases_rank0": counts, "problems_rank0": len(mine),
           "mean_iterations_rank0": (sum(r.iterations for r in res) / len(res)) if res else None}
    exe = ROOT / "oracle" / "_ref" / "sdpa_dd"
    if rank == 0 and world == 1 and not args.no_cpu_baseline and exe.exists():
        import concurrent.futures as cf
        import random
        pick = random.Random(0).sample(range(len(paths)), BATCH["cpu_sample"])
        cores = os.cpu_count() or 1

        def run(q):
            path = paths[q][0]
            t0 = time.perf_counter()
            subprocess.run([str(exe), "-ds", str(path), "-o", str(path) + ".ref.out", "-p", param_path], capture_output=True,
                           env=dict(os.environ, OMP_NUM_THREADS="1"), check=False)
            dt_q = time.perf_counter() - t0
            import re
            mt = re.search(r"phase.value = (\w+)", pathlib.Path(str(path) + ".ref.out").read_text())
            return dt_q, mt.group(1) if mt else None

        with cf.ThreadPoolExecutor(max_workers=min(cores, len(pick))) as ex:
            runs = list(ex.map(run, pick))
        secs = [r[0] for r in runs]
        mean_s = sum(secs) / len(secs)
        ref_ph = [r[1] for r in runs]
        ours_ph = {}
        if world == 1:
            pos = {q: i for i, q in enumerate(mine)}
            ours_ph = {str(q): phases[pos[q]] for q in pick}
        out["cpu_reference"] = {"solves_per_s": cores / mean_s, "cores": cores, "kind": "reference",
                                "phases": {str(q): ph for q, ph in zip(pick, ref_ph)}, "phases_ours_same_problems": ours_ph,
                                "sample": f"oracle/_ref sdpa_dd on {len(pick)} of the problems (seeded pick), one thread each; "
                                          f"rate = cores / mean single-thread solve time ({mean_s:.2f} s), without gradients"}
    return out


def dist_init(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 and args.impl == "ours":
        import torch.distributed as dist
        import torch
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def allsum(world, v):
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(v)], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def allmax(world, v):
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# The reference arm's bounded sample of the headline workload: one main-loop
# pass at m = 9980 takes about a minute on 16 host cores, so it times
# REF_STEPS passes after REF_WARMUP untimed ones, whatever --steps/--warmup.
REF_WARMUP, REF_STEPS = 1, 1


def run_reference(args, world, rank):
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    res, why = cpu_reference(WORKLOAD, REF_WARMUP, REF_STEPS, threads)
    if res is None:
        print(json.dumps({"impl": "reference", "unavailable": why}))
        return 0
    sample = (f"{workload_label(WORKLOAD)} (m={res['m']}): {REF_STEPS} timed pass(es) of the stock main loop after {REF_WARMUP} untimed, "
              f"{res['threads']} OpenMP threads (bounded sample: ~1 min per pass)")
    line = {
        "impl": "reference",
        "metric": "Schur+Chol dd-GFLOP/s per Newton iteration",
        "value": res["value"], "unit": "dd-GFLOP/s", "higher_is_better": True,
        "n_gpus": world, "steps": REF_STEPS, "warmup": REF_WARMUP,
        "ms_per_step": 1e3 * sum(res["pass_s"]) / len(res["pass_s"]),
        "scaling": "weak", "vs_baseline": None, "dtype": "dd (f64 pairs)", "data": "synthetic",
        "config": {"workload": workload_label(WORKLOAD), "m": res["m"], "step": "one main-loop pass",
                   "reference": "oracle/_ref (SDPA-DD 7.1.3 built from its sources, OpenMP)"},
        "reference_timers_s_per_step": {"make_bMat": res["schur_s"], "cholesky_bMat": res["chol_s"]},
        "cpu_baseline": {"value": res["value"], "unit": "dd-GFLOP/s", "cores": res["threads"], "kind": "reference", "sample": sample},
        "e2e": {"value": res["value"], "unit": "dd-GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def _dd_dec(v):
    from decimal import Decimal, getcontext
    getcontext().prec = 60
    return Decimal(v.hi) + Decimal(v.lo)


KERNELS_ALL = ("schur_build", "schur_pairs_tc", "potrf_diag", "potrf_diag_pre", "potrf_panel", "potrf_trailing_update",
               "potrf_trailing_update_tc", "trsv", "trsv_diag_inverse", "sparse_factor", "sparse_solve", "min_eig")


def other_solves(sddd, args, local, world):
    """The max-cut (n = m = 500), control-shaped (blocks 100 + 50, m = 1326)
    and chain (200 blocks, m = 5990, sparse Schur) workloads solved to
    relative gap 1e-25 in each form, against the reference build's own
    solve of the same file (one OpenMP thread, tests/golden/*.json: phase,
    iterations, dd objectives) and its time to gap on the host cores
    (iterations x one timed pass of its stock main loop); beside them, one
    profiled solve's device time per iteration by phase."""
    import torch
    golden = {}
    gfile = ROOT / "tests" / "golden" / "large_solves.json"
    if gfile.exists():
        golden = json.loads(gfile.read_text())
    out = {}
    workdir = pathlib.Path(tempfile.gettempdir()) / f"sddd_bench_{os.getuid()}_{local}"
    workdir.mkdir(exist_ok=True)
    sfile = ROOT / "tests" / "golden" / "sparse_schur.json"
    if sfile.exists():
        for k, v in json.loads(sfile.read_text())["cases"].items():
            d = v[0]
            golden[k] = {"phase": d["phase"], "iterations": d["iterations"], "eps": 1e-20,
                         "objValPrimal": [d["objValPrimal32"], "0"], "objValDual": [d["objValDual32"], "0"]}
    forms = {"maxcut_n500": (("tc_split", args.tc, 0), ("plain", 0, 0)),
             "control_100_50_m1326": (("tc_split", args.tc, 0), ("plain", 0, 0)),
             "chain200_n20": (("sparse", 0, 0), ("dense_tc_split", args.tc, 1), ("dense_plain", 0, 1))}
    for key, w, gname in (("maxcut_n500", MAXCUT, "maxcut_n500"), ("control_100_50_m1326", CONTROL, "control_100_50_m1326"),
                          ("chain200_n20", CHAIN, "chain200_n20")):
        data, param_path = write_workload(w, workdir)
        g = golden.get(gname)
        if g and g.get("eps"):
            param_path = problems().write_param(str(workdir / f"bench_{key}.param"), eps=g["eps"])
        par = sddd.param(param_path)
        ent = {"workload": workload_label(w)}
        if g and g.get("eps"):
            ent["eps"] = g["eps"]
        with sddd.Context(local) as c:
            c.read_problem(data, sparse=True, kappa=1.2)
            ent["m"] = c.m
            for label, slices, mode in forms[key]:
                if slices == 0 and label.endswith("tc_split"):
                    continue
                if c.L.sddd_set_tc_split(c.h, slices) != 0:
                    raise RuntimeError(c.L.sddd_last_error(c.h).decode())
                c.set_schur_mode(mode)
                form = c.schur_form()[0]
                if form.sparse:
                    ent["schur_form"] = {"sparse": True, "nnz_factor": form.nnz, "tiles": form.ntiles, "aggregate": form.aggregate}
                barrier(world)
                torch.cuda.synchronize()
                t1 = time.perf_counter()
                r = c.solve(par)
                torch.cuda.synchronize()
                dt = allmax(world, (time.perf_counter() - t1) * 1e3) / 1e3
                e = {"seconds": dt, "iterations": r.iterations, "phase": sddd.PHASES[r.phase], "relative_gap": r.relative_gap.hi}
                if g:
                    from decimal import Decimal
                    for nm in ("objValPrimal", "objValDual"):
                        want = Decimal(g[nm][0]) + Decimal(g[nm][1])
                        e[f"{nm}_rel_diff_vs_reference"] = float(abs(_dd_dec(getattr(r, nm)) - want) / max(abs(want), Decimal(1)))
                ent[label] = e
            # one profiled solve of the first form: device ms per iteration by phase
            label, slices, mode = forms[key][0]
            c.L.sddd_set_tc_split(c.h, slices)
            c.set_schur_mode(mode)
            c.L.sddd_profile(c.h, 1)
            c.L.sddd_profile_reset(c.h)
            r = c.solve(par)
            ph = {}
            for name in KERNELS_ALL:
                t, n = ctypes.c_double(), ctypes.c_long()
                c.L.sddd_profile_read(c.h, name.encode(), ctypes.byref(t), ctypes.byref(n))
                if n.value:
                    ph[name] = round(t.value / max(1, r.iterations), 3)
            c.L.sddd_profile(c.h, 0)
            ent["phase_ms_per_iteration"] = {"form": label, **ph}
        if g:
            src = "tests/golden/sparse_schur.json" if key.startswith("chain") else "tests/golden/large_solves.json"
            ent["reference"] = {"phase": g["phase"], "iterations": g["iterations"], "source": f"{src} (one OpenMP thread)"}
        if local == 0 and not args.no_cpu_baseline and g:
            res, why = cpu_reference(w, 0, 1, os.cpu_count() or 1)
            if res is not None:
                ent["reference"].update({"pass_s": res["pass_s"][0], "cores": res["threads"],
                                         "time_to_gap_s": g["iterations"] * res["pass_s"][0],
                                         "time_to_gap_basis": "reference iterations x one timed pass of its stock main loop (setup excluded)"})
        out[key] = ent
    return out


KERNELS = ("potrf_trailing_update", "potrf_trailing_update_tc", "potrf_panel", "potrf_diag", "potrf_diag_pre", "trsv", "trsv_diag_inverse", "schur_build",
           "min_eig")


def run_ours(args, world, rank, local):
    sddd = load_pkg()
    L = sddd.lib()
    import torch
    torch.cuda.set_device(local)
    workdir = pathlib.Path(tempfile.gettempdir()) / f"sddd_bench_{os.getuid()}_{local}"
    workdir.mkdir(exist_ok=True)
    data, param_path = write_workload(WORKLOAD, workdir)
    ctx = sddd.Context(local)
    t0 = time.perf_counter()
    ctx.read_problem(data, sparse=True, kappa=1.2)
    setup_s = time.perf_counter() - t0
    schur = ctypes.c_double()
    chol = ctypes.c_double()
    L.sddd_work(ctx.h, ctypes.byref(schur), ctypes.byref(chol))
    step_flops = schur.value + chol.value
    par = sddd.param(param_path)
    stream = torch.cuda.ExternalStream(L.sddd_stream(ctx.h))

    def set_tc(slices):
        if L.sddd_set_tc_split(ctx.h, slices) != 0:
            raise RuntimeError(L.sddd_last_error(ctx.h).decode())

    def restart():
        ctx.call("sddd_solver_start", ctypes.byref(par))

    def iterate():
        rc = L.sddd_iterate(ctx.h)
        if rc < 0:
            raise RuntimeError(L.sddd_last_error(ctx.h).decode())
        if rc != 0:  # converged or stopped: continue from a fresh start
            restart()
            rc = L.sddd_iterate(ctx.h)
            if rc != 0:
                raise RuntimeError(f"solver stopped at its first iteration (rc={rc})")

    def timed_passes(steps, warmup, clocks=False, profile=False):
        """device time of `steps` main-loop passes (max over ranks) and the
        kernel launches inside the region; with profile, the per-kernel
        times (event pairs around every kernel group: a separate run, never
        the headline's)"""
        restart()
        for _ in range(warmup):
            iterate()
        barrier(world)
        torch.cuda.synchronize()
        clk = Clocks(local) if (clocks and rank == 0) else None
        L.sddd_profile(ctx.h, 1 if profile else 0)
        L.sddd_profile_reset(ctx.h)
        launches0 = L.sddd_launch_count()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(steps):
            iterate()
        ev1.record(stream)
        torch.cuda.synchronize()
        launches = L.sddd_launch_count() - launches0
        barrier(world)
        clk_res = clk.stop() if clk else None
        kern = {}
        if profile:
            for name in KERNELS:
                t = ctypes.c_double()
                n = ctypes.c_long()
                L.sddd_profile_read(ctx.h, name.encode(), ctypes.byref(t), ctypes.byref(n))
                kern[name] = (t.value, n.value)
            L.sddd_profile(ctx.h, 0)
        return allmax(world, ev0.elapsed_time(ev1)), kern, launches, clk_res

    # ---- headline: the tensor-core split form, device-resident, no profiling
    set_tc(args.tc)
    ms_max, _, launches, clk = timed_passes(args.steps, args.warmup, clocks=True)
    value = world * args.steps * step_flops / (ms_max * 1e-3) / 1e9
    # per-kernel breakdown of the same passes, in a separate profiled run
    prof_ms, kern, _, _ = timed_passes(args.steps, 1, profile=True)
    # ---- end to end through the C ABI with host buffers (same form), from
    # a fresh start so the timed passes stay inside one solve
    n_space = L.sddd_space_len(ctx.h)
    m = ctx.m
    X = torch.empty(2 * n_space, dtype=torch.float64).pin_memory()
    Z = torch.empty(2 * n_space, dtype=torch.float64).pin_memory()
    y = torch.empty(2 * m, dtype=torch.float64).pin_memory()
    px, pz, py = (ctypes.c_void_p(t.data_ptr()) for t in (X, Z, y))
    restart()
    for _ in range(args.warmup):
        iterate()
    L.sddd_get_point(ctx.h, px, py, pz)
    h2d = d2h = 16 * (2 * n_space + m)
    barrier(world)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        if L.sddd_set_point(ctx.h, px, py, pz) != 0:
            raise RuntimeError("set_point failed")
        if L.sddd_iterate(ctx.h) != 0:
            raise RuntimeError("the solve ended inside the timed end-to-end passes")
        L.sddd_get_point(ctx.h, px, py, pz)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    e2e_ms = allmax(world, e0.elapsed_time(e1))
    e2e_value = world * args.steps * step_flops / (e2e_ms * 1e-3) / 1e9
    # ---- the plain dd form (the reference's operation order) on the same passes
    plain = None
    if args.tc:
        set_tc(0)
        p_ms, _, _, _ = timed_passes(args.steps, 1)
        _, p_kern, _, _ = timed_passes(args.steps, 1, profile=True)
        plain = {"value": world * args.steps * step_flops / (p_ms * 1e-3) / 1e9, "ms_per_step": p_ms / args.steps,
                 "kernel_ms_per_step": {k: v[0] / args.steps for k, v in p_kern.items()}}
        set_tc(args.tc)
    # ---- time to relative gap 1e-25 from the standard initial point
    solves = None
    if not args.no_solve:
        solves = {}
        for label, slices in (("tc_split", args.tc), ("plain", 0)):
            if label == "tc_split" and not args.tc:
                continue
            set_tc(slices)
            barrier(world)
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            r = ctx.solve(par)
            torch.cuda.synchronize()
            dt = allmax(world, (time.perf_counter() - t1) * 1e3) / 1e3
            solves[label] = {"seconds": dt, "iterations": r.iterations, "phase": sddd.PHASES[r.phase],
                             "relative_gap": r.relative_gap.hi, "objValPrimal": r.objValPrimal.hi, "_obj": _dd_dec(r.objValPrimal)}
        set_tc(args.tc)
        if "tc_split" in solves:
            solves["speedup_tc_over_plain"] = solves["plain"]["seconds"] / solves["tc_split"]["seconds"]
        solves["objValPrimal_diff_tc_vs_plain"] = None
        if "tc_split" in solves:
            from decimal import Decimal
            a, b = solves["tc_split"].pop("_obj"), solves["plain"].pop("_obj")
            solves["objValPrimal_diff_tc_vs_plain"] = float(abs(a - b) / max(abs(b), Decimal(1)))
        else:
            solves["plain"].pop("_obj")
    # ---- roofline of the dominant kernel
    tr_fl, tr_launch = trailing_flops(m)
    fp64 = ctypes.c_double()
    L.sddd_fp64_peak(ctx.h, ctypes.byref(fp64))
    peak_dd = fp64.value / 20.0  # one dd multiply-subtract = 2 dd-flops = 20 FP64 instructions
    peaks = {}
    pfile = ROOT / "MEASURED_PEAKS.json"
    if pfile.exists():
        peaks = json.loads(pfile.read_text())
    if args.tc:
        t_ms, t_n = kern["potrf_trailing_update_tc"]
        pairs = args.tc * (args.tc + 1) // 2
        int8_ops = tr_fl * pairs  # entries x 64 (= tr_fl / 2) x pairs x 2 ops
        achieved = (int8_ops * args.steps) / (t_ms * 1e-3) / 1e12 if t_ms > 0 else None
        bf16 = peaks.get("bf16_tflops")
        peak = 2.0 * bf16 if bf16 else 2.0 * 1590.0
        traffic = None
        tfile = ROOT / "profiles" / "ozaki_syrk_traffic.json"
        if tfile.exists():
            bpe = json.loads(tfile.read_text()).get("bytes_per_entry")
            if bpe:
                traffic = bpe * (tr_fl / 128.0) / tr_launch
        roofline = {"kernel": "potrf_trailing_update_tc (ozaki_split + ozaki_syrk: INT8 slice products on tcgen05)", "bound": "tensor",
                    "achieved": achieved, "peak": peak, "unit": "TOPS (int8)", "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                    "peak_source": ("2 x measured dense bf16 burst (MEASURED_PEAKS.json bf16_tflops %.0f): the part's dense int8 rate is twice its bf16 rate"
                                    % bf16) if bf16 else "2 x fallback bf16 1590 TFLOP/s",
                    "slices": args.tc, "pairs": pairs, "launches_per_step": t_n / args.steps, "int8_ops_per_launch": int8_ops / tr_launch,
                    "dd_equivalent_gflops": (tr_fl * args.steps) / (t_ms * 1e-3) / 1e9 if t_ms > 0 else None,
                    "plain_fp64_ceiling_dd_gflops": peak_dd}
    else:
        t_ms, t_n = kern["potrf_trailing_update"]
        achieved = (tr_fl * args.steps) / (t_ms * 1e-3) / 1e9 if t_ms > 0 else None
        traffic = None
        tfile = ROOT / "profiles" / "potrf_trailing_update_traffic.json"
        if tfile.exists():
            traffic = json.loads(tfile.read_text()).get("bytes_per_launch")
        roofline = {"kernel": "potrf_trailing_update", "bound": "fp64", "achieved": achieved, "peak": peak_dd, "unit": "dd-GFLOP/s",
                    "frac": (achieved / peak_dd) if achieved and peak_dd else None, "traffic": traffic,
                    "peak_source": f"measured FP64 FMA rate {fp64.value:.0f} GFLOP/s / 20 FP64 instructions per dd multiply-add pair (2 dd-flops)",
                    "launches_per_step": t_n / args.steps, "ddflops_per_launch": tr_fl / tr_launch}
    batched = None if args.no_batch else batch_measure(sddd, local, rank, world, args)
    others = None if args.no_solve else other_solves(sddd, args, local, world)
    cpu = cpu_small = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        res, why = cpu_reference(WORKLOAD, 0, 1, threads)
        if res is not None:
            cpu = {"value": res["value"], "unit": "dd-GFLOP/s", "cores": res["threads"], "kind": "reference",
                   "sample": f"oracle/_ref stock main loop on the same workload ({workload_label(WORKLOAD)}, m={res['m']}): one pass, "
                             f"{res['threads']} OpenMP threads",
                   "pass_s": res["pass_s"][0], "make_bMat_s": res["schur_s"][0], "cholesky_bMat_s": res["chol_s"][0]}
            if solves and "tc_split" in solves:
                solves["reference_time_to_gap_s"] = solves["tc_split"]["iterations"] * res["pass_s"][0]
                solves["reference_time_to_gap_basis"] = "iterations of this solve x one timed pass of the reference's stock main loop"
        else:
            cpu = {"value": None, "unit": "dd-GFLOP/s", "cores": 0, "kind": "reference", "sample": why}
        res, why = cpu_reference(SMALL_THETA, 0, 1, threads)
        if res is not None:
            cpu_small = {"value": res["value"], "unit": "dd-GFLOP/s", "cores": res["threads"], "kind": "reference",
                         "sample": f"{workload_label(SMALL_THETA)} (m={res['m']}), one pass (a smaller config, for comparison only)"}
    if rank == 0:
        line = {
            "metric": "Schur+Chol dd-GFLOP/s per Newton iteration",
            "value": value, "unit": "dd-GFLOP/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "dd (f64 pairs); Cholesky trailing updates as int8 slice products" if args.tc else "dd (f64 pairs)", "data": "synthetic",
            "config": {"workload": f"theta-shaped SDP nv={WORKLOAD['nv']} p={WORKLOAD['p']} seed={WORKLOAD['seed']}", "m": m,
                       "block": ctx.sizes, "step": "one main-loop pass (predictor+corrector Newton, step length, update)",
                       "form": f"tensor-core split, {args.tc} slices" if args.tc else "plain dd",
                       "parallelism": f"replicas x{world}", "l2": "inputs larger than L2 (Schur matrix %.2f GB)" % (16.0 * m * m / 1e9),
                       "eps": EPS, "setup_s": setup_s},
            "step_ddflops": {"schur": schur.value, "cholesky": chol.value},
            "kernel_ms_per_step": {k: v[0] / args.steps for k, v in kern.items()},
            "kernel_breakdown_basis": f"a separate run of {args.steps} passes with per-kernel event pairs ({prof_ms / args.steps:.1f} ms per pass there)",
            "plain_dd": plain,
            "solve_to_gap": solves,
            "solve_to_gap_other_configs": others,
            "batched": batched,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "cpu_baseline_m3571": cpu_small,
            "e2e": {"value": e2e_value, "unit": "dd-GFLOP/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": int(launches),
            "clocks": clk,
        }
        print(json.dumps(line))
    ctx.close()
    return 0


def profile_case(args):
    """One dd Cholesky of an m x m SPD matrix through sddd_Rpotrf (the
    kernels of the bench's dominant phase, at a size an ncu capture can
    replay), then one solve with the factor (sddd_Rpotrs: the triangular
    solves); prints their times."""
    sddd = load_pkg()
    L = sddd.lib()
    import torch
    m = args.m
    g = torch.Generator(device="cuda").manual_seed(7)
    G = torch.randn(m, m, dtype=torch.float64, device="cuda", generator=g)
    A = G @ G.T / m + torch.eye(m, dtype=torch.float64, device="cuda")
    dd = torch.zeros(m * m, 2, dtype=torch.float64, device="cuda")
    dd[:, 0] = A.T.reshape(-1)  # column-major
    del G, A
    with sddd.Context(0) as ctx:
        if args.tc and L.sddd_set_tc_split(ctx.h, args.tc) != 0:
            raise RuntimeError(L.sddd_last_error(ctx.h).decode())
        torch.cuda.synchronize()
        t = time.perf_counter()
        info = L.sddd_Rpotrf(ctx.h, b"L", m, ctypes.c_void_p(dd.data_ptr()), m)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        rc = -1
        if info == 0:
            b = torch.zeros(m, 2, dtype=torch.float64, device="cuda")
            b[:, 0] = 1.0
            rc = L.sddd_Rpotrs(ctx.h, b"L", m, 1, ctypes.c_void_p(dd.data_ptr()), m, ctypes.c_void_p(b.data_ptr()), m)
            torch.cuda.synchronize()
        print(json.dumps({"case": "potrf", "m": m, "info": info, "s": t1 - t, "potrs_rc": rc, "potrs_s": time.perf_counter() - t1}))
    return 0 if info == 0 and rc == 0 else 1


def profile_case_sparse(args):
    """One sparse factorisation and solve (sddd_sparse_getCholesky /
    sddd_sparse_solveSystems) of the chain workload's Schur structure with
    random positive definite entries, for an ncu capture; prints its time."""
    sddd = load_pkg()
    L = sddd.lib()
    import numpy as np
    import torch
    workdir = pathlib.Path(tempfile.gettempdir()) / f"sddd_bench_{os.getuid()}_sp"
    workdir.mkdir(exist_ok=True)
    data, _ = write_workload(CHAIN, workdir)
    info, order, di, ci = sddd.plan_schur(data)
    m, nnz = info.m, info.nnz
    rng = np.random.default_rng(5)
    v = rng.standard_normal((nnz, 2)) * np.array([0.1, 1e-18])
    v[di[:-1], 0] = 4.0 + 10.0 * np.abs(rng.standard_normal(m))
    v[di[:-1], 1] = 0.0
    dv = torch.from_numpy(v.reshape(-1).copy()).cuda()
    dx = torch.from_numpy(np.stack([rng.standard_normal(m), np.zeros(m)], 1).reshape(-1).copy()).cuda()
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    with sddd.Context(0) as ctx:
        torch.cuda.synchronize()
        t = time.perf_counter()
        rc = L.sddd_sparse_getCholesky(ctx.h, m, p(di), p(ci), ctypes.c_void_p(dv.data_ptr()))
        rc2 = L.sddd_sparse_solveSystems(ctx.h, m, p(di), p(ci), ctypes.c_void_p(dv.data_ptr()), ctypes.c_void_p(dx.data_ptr()))
        torch.cuda.synchronize()
        print(json.dumps({"case": "sparse", "m": m, "nnz": nnz, "tiles": info.ntiles, "rc": [rc, rc2], "s": time.perf_counter() - t}))
    return 0 if rc == 0 and rc2 == 0 else 1


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-case", choices=["potrf", "sparse"], help="run one kernel-level case for an ncu capture and exit")
    ap.add_argument("--m", type=int, default=4096)
    ap.add_argument("--tc", type=int, default=16, help="slices of the tensor-core split Cholesky (8..16; 0 = plain dd only)")
    ap.add_argument("--no-solve", action="store_true", help="skip the two solves to relative gap 1e-25")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched workload (256 small SDPs)")
    ap.add_argument("--batch-workers", type=int, default=0, help="host workers of the batched workload (0: the library's default)")
    ap.add_argument("--batch-core", type=int, default=-1, choices=[-1, 0, 1], help="batched Newton core off (0) or on (1); -1: the library's default")
    ap.add_argument("--batch-only", action="store_true", help="run the batched workload alone and print its figures")
    args = ap.parse_args()
    if args.profile_case == "sparse":
        return profile_case_sparse(args)
    if args.profile_case:
        return profile_case(args)
    if args.warmup < 3:
        args.warmup = 3
    world, rank, local = dist_init(args)
    if args.batch_only:
        args.no_cpu_baseline = True
        print(json.dumps(batch_measure(load_pkg(), local, rank, world, args)))
        return 0
    try:
        if args.impl == "reference":
            return run_reference(args, world, rank)
        return run_ours(args, world, rank, local)
    finally:
        if world > 1 and args.impl == "ours":
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
