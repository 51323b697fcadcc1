"""Seeded synthetic SDP workloads in SDPA sparse format (.dat-s).

The reference reads problems from `.dat-s` text (sdpa_io.cpp:447-786), so
every workload here is produced as that text and both this library and the
reference parse the very same bytes.  Values are written with 17
significant digits; both readers turn each decimal string into the same dd
value (the QD 2.3.23 decimal reader, dd_real.cpp:1198).

SDPA conventions (sdpa_io.cpp:124-150, 692-694): the file lists the
objective vector c, then the entries `k block i j value` of F_0..F_m.  The
primal is  min c.x  s.t.  X = sum_k F_k x_k - F_0 >= 0, the dual
max F_0 . Y  s.t.  F_k . Y = c_k, Y >= 0.

Workloads (seed = workload index):
  0 dense_random   one block n=50, m=100, dense F_k ~ N(0,1)
  1 maxcut         n=m=500, F_k = e_k e_k^T, c = 1, F_0 = L/4 (Erdos-Renyi p=0.02)
  2 theta          200 vertices, edge prob 0.5 (m ~ 1 + 9950), F_1 = I, F_e = E_uv
  3 control_like   blocks 100 and 50, m = 1326, dense N(0,1)/sqrt(n)
  4 batch          256 dense random problems, n ~ U[10,80], m ~ U[20,200]

The maxcut and theta objective matrices follow the sign of the SDPLIB
files these shapes stand in for (mcp*.dat-s: F_0 = +L/4; theta*.dat-s:
F_0 = +J).
"""
from __future__ import annotations

import io
import os

import numpy as np

__all__ = [
    "dense_random",
    "maxcut",
    "theta",
    "with_lp",
    "blocks_with_lp",
    "control_like",
    "batch",
    "workload",
    "chain_blocks",
    "write_param",
    "WORKLOADS",
]


def _fmt(v: float) -> str:
    return repr(float(v)) if float(v) != int(v) or abs(v) >= 1e15 else str(int(v))


class _Writer:
    def __init__(self, m: int, blocks: list[int], c: np.ndarray, title: str):
        self.buf = io.StringIO()
        w = self.buf.write
        # the reference reads the title line into a 256-byte buffer
        # (sdpa_io.cpp:127, lengthOfString) and parses the rest of a longer
        # line as data
        if len(title) > 200:
            title = title[:197] + "..."
        w(f'"{title}"\n')
        w(f"{m} = mDIM\n{len(blocks)} = nBLOCK\n")
        w(" ".join(str(b) for b in blocks) + " = bLOCKsTRUCT\n")
        w("{" + ", ".join(_fmt(x) for x in c) + "}\n")

    def entries(self, k: int, blk: int, ii, jj, vv):
        lines = [f"{k} {blk} {i + 1} {j + 1} {_fmt(v)}\n" for i, j, v in zip(ii, jj, vv)]
        self.buf.write("".join(lines))

    def dense_upper(self, k: int, blk: int, M: np.ndarray):
        n = M.shape[0]
        iu, ju = np.triu_indices(n)
        vals = M[iu, ju]
        keep = vals != 0.0
        self.entries(k, blk, iu[keep], ju[keep], vals[keep])

    def text(self) -> str:
        return self.buf.getvalue()


def _dense_blocks(rng, m: int, sizes: list[int], scale_by_n: bool, with_x0: bool = False):
    """F_k per block ~ N(0,1) (or N(0,1)/sqrt(n)), symmetric; x0 ~ N(0,1);
    X0 = I + G G^T / n per block; F_0 = sum_k F_k x0_k - X0; c_k = tr F_k
    so that Y = I is dual feasible and x0 is primal feasible."""
    x0 = rng.standard_normal(m)
    Fs = []  # Fs[blk][k]
    F0 = []
    c = np.zeros(m)
    for n in sizes:
        s = 1.0 / np.sqrt(n) if scale_by_n else 1.0
        A = rng.standard_normal((m, n, n)) * s
        A = 0.5 * (A + A.transpose(0, 2, 1))
        G = rng.standard_normal((n, n))
        X0 = np.eye(n) + G @ G.T / n
        F0.append(np.tensordot(x0, A, axes=1) - X0)
        c += np.trace(A, axis1=1, axis2=2)
        Fs.append(A)
    if with_x0:
        return c, F0, Fs, x0
    return c, F0, Fs


def dense_random(n: int = 50, m: int = 100, seed: int = 0) -> str:
    rng = np.random.default_rng(seed)
    c, F0, Fs = _dense_blocks(rng, m, [n], scale_by_n=False)
    w = _Writer(m, [n], c, f"dense random SDP n={n} m={m} seed={seed}")
    w.dense_upper(0, 1, F0[0])
    for k in range(m):
        w.dense_upper(k + 1, 1, Fs[0][k])
    return w.text()


def control_like(sizes=(100, 50), m: int = 1326, seed: int = 3) -> str:
    rng = np.random.default_rng(seed)
    c, F0, Fs = _dense_blocks(rng, m, list(sizes), scale_by_n=True)
    w = _Writer(m, list(sizes), c, f"control-shaped SDP blocks={list(sizes)} m={m} seed={seed}")
    for b in range(len(sizes)):
        w.dense_upper(0, b + 1, F0[b])
    for k in range(m):
        for b in range(len(sizes)):
            w.dense_upper(k + 1, b + 1, Fs[b][k])
    return w.text()


def with_lp(n: int = 30, q: int = 24, m: int = 40, seed: int = 7) -> str:
    """An SDP block of order n and an LP block of q entries (block structure
    "n -q"), strictly feasible on both sides: F_k ~ N(0,1)/sqrt(n) on the
    SDP block, LP coefficients ~ N(0,1) on about half the entries; one x0 ~
    N(0,1) with slacks X0 = I + G G^T / n and s0 ~ 1 + U(0,1) sets F_0; c_k =
    tr F_k + the sum of its LP coefficients, so Y = I, y_lp = 1 is dual
    feasible."""
    rng = np.random.default_rng(seed)
    x0 = rng.standard_normal(m)
    A = rng.standard_normal((m, n, n)) / np.sqrt(n)
    A = 0.5 * (A + A.transpose(0, 2, 1))
    G = rng.standard_normal((n, n))
    F0 = np.tensordot(x0, A, axes=1) - (np.eye(n) + G @ G.T / n)
    a = rng.standard_normal((m, q)) * (rng.random((m, q)) < 0.5)
    f0 = x0 @ a - (1.0 + rng.random(q))
    c = np.trace(A, axis1=1, axis2=2) + a.sum(axis=1)
    w = _Writer(m, [n, -q], c, f"SDP block {n} + LP block {q}, m={m} seed={seed}")
    w.dense_upper(0, 1, F0)
    w.entries(0, 2, range(q), range(q), f0)
    for k in range(m):
        w.dense_upper(k + 1, 1, A[k])
        nz = np.nonzero(a[k])[0]
        w.entries(k + 1, 2, nz, nz, a[k, nz])
    return w.text()


def blocks_with_lp(sizes=(30,), q: int = 0, m: int = 40, seed: int = 8) -> str:
    """Dense SDP blocks of the given orders (the config-0 construction per
    block, entries N(0,1)/sqrt(n)) and, with q > 0, an LP block of q entries
    (coefficients N(0,1) on about half of them, slacks 1 + U(0,1) at x0):
    strictly feasible on both sides (Y = I, y_lp = 1 is dual feasible).
    Many small blocks exercise the per-block paths (inner products, step
    lengths) beyond a handful of blocks."""
    rng = np.random.default_rng(seed)
    sizes = [int(n) for n in sizes]
    c, F0, Fs, x0 = _dense_blocks(rng, m, sizes, scale_by_n=True, with_x0=True)
    blocks = list(sizes)
    if q > 0:
        a = rng.standard_normal((m, q)) * (rng.random((m, q)) < 0.5)
        f0 = x0 @ a - (1.0 + rng.random(q))
        c = c + a.sum(axis=1)
        blocks.append(-q)
    w = _Writer(m, blocks, c, f"{len(sizes)} SDP blocks + LP {q}, m={m} seed={seed}")
    for b in range(len(sizes)):
        w.dense_upper(0, b + 1, F0[b])
    if q > 0:
        w.entries(0, len(sizes) + 1, range(q), range(q), f0)
    for k in range(m):
        for b in range(len(sizes)):
            w.dense_upper(k + 1, b + 1, Fs[b][k])
        if q > 0:
            nz = np.nonzero(a[k])[0]
            w.entries(k + 1, len(sizes) + 1, nz, nz, a[k, nz])
    return w.text()


def chain_blocks(nblocks: int = 40, n: int = 10, per: int = 4, overlap: int = 2, q: int = 0, seed: int = 9) -> str:
    """SDP blocks in a chain: block b has `per` constraints of its own and
    shares `overlap` constraints with block b+1 (dense N(0,1)/sqrt(n) data on
    each block a constraint touches); with q > 0, q LP entries, entry t on
    the constraints of block t % nblocks.  The constraints are numbered in a
    random order, so the Schur matrix is a permuted band: more than 5 blocks,
    m > 100 and a sparse aggregate pattern put it on the reference's sparse
    Schur path.  Strictly feasible on both sides (x0 ~ N(0,1) primal, Y = I
    and y_lp = 1 dual) as the other generators."""
    rng = np.random.default_rng(seed)
    touch: list[list[int]] = []  # blocks of each constraint, natural order
    for b in range(nblocks):
        touch += [[b] for _ in range(per)]
        if b + 1 < nblocks:
            touch += [[b, b + 1] for _ in range(overlap)]
    m = len(touch)
    perm = rng.permutation(m)  # natural constraint t gets index perm[t]
    blocks_of = [None] * m
    for t in range(m):
        blocks_of[perm[t]] = touch[t]
    x0 = rng.standard_normal(m)
    c = np.zeros(m)
    Fk = [dict() for _ in range(m)]  # per constraint: block -> matrix
    F0 = []
    s = 1.0 / np.sqrt(n)
    for b in range(nblocks):
        X0 = np.eye(n)
        G = rng.standard_normal((n, n))
        X0 = X0 + G @ G.T / n
        acc = -X0
        for k in range(m):
            if b in blocks_of[k]:
                A = rng.standard_normal((n, n)) * s
                A = 0.5 * (A + A.T)
                Fk[k][b] = A
                acc = acc + x0[k] * A
                c[k] += np.trace(A)
        F0.append(acc)
    lp = []
    if q > 0:
        for t in range(q):
            b = t % nblocks
            ks = [k for k in range(m) if b in blocks_of[k]]
            a = {k: float(rng.standard_normal()) for k in ks if rng.random() < 0.5}
            f0 = sum(x0[k] * v for k, v in a.items()) - (1.0 + rng.random())
            for k, v in a.items():
                c[k] += v
            lp.append((a, f0))
    blocks = [n] * nblocks + ([-q] if q > 0 else [])
    w = _Writer(m, blocks, c, f"chain of {nblocks} SDP blocks n={n} per={per} overlap={overlap} LP {q} m={m} seed={seed}")
    for b in range(nblocks):
        w.dense_upper(0, b + 1, F0[b])
    if q > 0:
        w.entries(0, nblocks + 1, range(q), range(q), [f0 for _, f0 in lp])
    for k in range(m):
        for b in sorted(Fk[k]):
            w.dense_upper(k + 1, b + 1, Fk[k][b])
        if q > 0:
            ts = [t for t in range(q) if k in lp[t][0]]
            w.entries(k + 1, nblocks + 1, ts, ts, [lp[t][0][k] for t in ts])
    return w.text()


def maxcut(n: int = 500, p: float = 0.02, seed: int = 1) -> str:
    rng = np.random.default_rng(seed)
    A = np.triu(rng.random((n, n)) < p, 1)
    A = A | A.T
    deg = A.sum(axis=1)
    L = np.diag(deg.astype(float)) - A.astype(float)
    w = _Writer(n, [n], np.ones(n), f"maxcut-shaped SDP n={n} p={p} seed={seed}")
    w.dense_upper(0, 1, L / 4.0)
    for k in range(n):
        w.entries(k + 1, 1, [k], [k], [1.0])
    return w.text()


def theta(nv: int = 200, p: float = 0.5, seed: int = 2) -> str:
    rng = np.random.default_rng(seed)
    iu, ju = np.triu_indices(nv, 1)
    keep = rng.random(iu.shape[0]) < p
    eu, ev = iu[keep], ju[keep]
    m = 1 + eu.shape[0]
    c = np.zeros(m)
    c[0] = 1.0
    w = _Writer(m, [nv], c, f"theta-shaped SDP nv={nv} p={p} edges={eu.shape[0]} seed={seed}")
    w.dense_upper(0, 1, np.ones((nv, nv)))
    w.entries(1, 1, range(nv), range(nv), [1.0] * nv)
    for e in range(eu.shape[0]):
        w.entries(e + 2, 1, [eu[e]], [ev[e]], [1.0])
    return w.text()


def batch(count: int = 256, seed: int = 4):
    """List of (n, m, text) for the batched workload."""
    rng = np.random.default_rng(seed)
    out = []
    for b in range(count):
        n = int(rng.integers(10, 81))
        m = int(rng.integers(20, 201))
        out.append((n, m, dense_random(n, m, seed=int(rng.integers(1 << 31)))))
    return out


WORKLOADS = {
    0: ("dense_random", lambda: dense_random()),
    1: ("maxcut", lambda: maxcut()),
    2: ("theta", lambda: theta()),
    3: ("control_like", lambda: control_like()),
}


def workload(index: int, directory: str) -> str:
    """Write workload `index` as .dat-s under `directory` (cached by name)
    and return the path."""
    name, make = WORKLOADS[index]
    os.makedirs(directory, exist_ok=True)
    path = os.path.join(directory, f"w{index}_{name}.dat-s")
    if not os.path.exists(path):
        tmp = path + ".tmp%d" % os.getpid()
        with open(tmp, "w") as f:
            f.write(make())
        os.replace(tmp, path)
    return path


def write_param(path: str, eps: float = 1e-25, max_iter: int = 200, gamma: float = 0.9,
                lambda_star: float = 1e4, beta_star: float = 0.1, beta_bar: float = 0.3) -> str:
    """param.sdpa in the reference's 10-line layout (sdpa_parts.cpp:172-183)."""
    lines = [
        f"{max_iter}\tunsigned int maxIteration;",
        f"{eps:.1E}\tdouble 0.0 < epsilonStar;",
        f"{lambda_star:.1E}   double 0.0 < lambdaStar;",
        "2.0   \tdouble 1.0 < omegaStar;",
        "-1.0E5  double lowerBound;",
        "1.0E5   double upperBound;",
        f"{beta_star}     double 0.0 <= betaStar <  1.0;",
        f"{beta_bar}     double 0.0 <= betaBar  <  1.0, betaStar <= betaBar;",
        f"{gamma}     double 0.0 < gammaStar  <  1.0;",
        f"{eps:.1E}\tdouble 0.0 < epsilonDash;",
    ]
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
    return path


def theta_edges(nv: int = 200, p: float = 0.5, seed: int = 2) -> int:
    """Number of edges of the theta workload (same draw as theta())."""
    rng = np.random.default_rng(seed)
    iu, _ = np.triu_indices(nv, 1)
    return int((rng.random(iu.shape[0]) < p).sum())


def theta_work(nv: int, n_edges: int) -> tuple[float, float]:
    """Algorithmic dd-flops of one Schur build and one Cholesky of B for the
    theta workload, counted as the library counts them (sddd_work): the F2
    owner F_1 = I needs F = A Z^-1 (2 n per nonzero) and G = X F (2 n^3),
    then per partner 2 n + 2 per nonzero term; every edge owner (F3, two
    off-diagonal terms) costs 3 eff_i eff_j + 2 eff_j per partner."""
    n = float(nv)
    m = 1 + n_edges
    # sorted order: the E edges (effect 2) first, then F_1 (effect nv)
    schur = 8.0 * n_edges * (n_edges + 1)          # sum_q (3*2 + 2) * 2 (q + 1)
    schur += 2.0 * n * nv + 2.0 * n ** 3            # F and G of F_1
    schur += n_edges * (2.0 * n * 2 + 2.0 * 2)      # F_1 with each edge
    schur += 2.0 * n * nv + 2.0 * nv                # F_1 with itself
    return schur, float(m) ** 3 / 3.0
