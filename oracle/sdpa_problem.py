"""Python restatement of the reference's problem reader (test infrastructure).

Reads SDPA sparse `.dat-s` text the way sdpa_io.cpp does and builds, per
SDP block, the constraint list with each A_k block in the reference's
storage (sparse COO in input order, or dense after changeToDense), plus the
formula table.  Values go through the oracle's QD decimal reader, so they
equal the reference's parsed dd values bit for bit.

Only tests and the benchmark's CPU-baseline leg use this module.
"""
from __future__ import annotations

import ctypes
import re

import numpy as np

DD = np.dtype([("hi", "<f8"), ("lo", "<f8")])

# fscanf "%*[^0-9+-]%[^,} \t\n]": skip a non-empty run of characters that are
# not digits or signs, then take the token up to a separator.
_TOKEN = re.compile(r"[^0-9+\-]+([^,} \t\n]+)")


class _Stream:
    def __init__(self, text: str, pos: int = 0):
        self.t = text
        self.p = pos

    def token(self):
        m = _TOKEN.match(self.t, self.p)
        if not m:
            return None
        self.p = m.end()
        return m.group(1)

    def int_(self):
        tok = self.token()
        if tok is None:
            return None
        m = re.match(r"[+-]?\d+", tok)
        if not m:
            return None
        # %d stops at the first non-digit; the remainder stays in the stream
        self.p -= len(tok) - m.end()
        return int(m.group(0))


class Problem:
    """SDP-block data in the reference's layout (LP blocks not supported)."""

    def __init__(self, oracle_lib, text: str, kappa: float = 1.2):
        self.lib = oracle_lib
        lines = text.split("\n")
        # IO::read(fpData, fpout, m, str): comment lines start with * or "
        i = 0
        while lines[i][:1] in ("*", '"'):
            i += 1
        self.m = int(re.match(r"\s*([+-]?\d+)", lines[i]).group(1))
        rest = "\n".join(lines[i + 1:])
        s = _Stream(rest)
        # fscanf("%d") for nBlock: skips whitespace only
        mm = re.match(r"\s*([+-]?\d+)", rest)
        nblock = int(mm.group(1))
        s.p = mm.end()
        self.block_struct = [s.int_() for _ in range(nblock)]
        if any(b < 2 for b in self.block_struct):
            raise NotImplementedError("LP blocks are not handled by this reader")
        self.nblocks = nblock
        self.b = np.zeros(self.m, DD)
        for k in range(self.m):
            self.b[k] = self.read_dd(s.token())
        # entries: k l i j v (sdpa_io.cpp:653-700, sparse input)
        ent = {}  # (k, l) -> list of (i, j, value)
        order = {}  # k -> list of blocks in first-seen order (sorted later)
        while True:
            k = s.int_()
            if k is None:
                break
            l = s.int_()
            ii = s.int_()
            jj = s.int_()
            tok = s.token()
            if l is None or ii is None or jj is None or tok is None:
                break
            v = self.read_dd(tok)
            if k == 0:
                v = np.array((-v["hi"], -v["lo"]), DD)  # C = -F0
            ent.setdefault((k, l - 1), []).append((ii - 1, jj - 1, v))
        self.C = {}
        self.A = []  # A[k] = {block: mat}
        for k in range(self.m + 1):
            blocks = sorted(l for (kk, l) in ent if kk == k)
            mats = {l: self._mat(self.block_struct[l], ent[(k, l)]) for l in blocks}
            if k == 0:
                self.C = mats
            else:
                self.A.append(mats)
        # InputData::initialize_index_SDP: per block, constraints in order
        self.cons = [[k for k in range(self.m) if l in self.A[k]] for l in range(nblock)]
        self.kappa = kappa
        self.formula = self._formulas()

    def read_dd(self, tok):
        out = np.zeros(1, DD)
        rc = self.lib.o_dd_read(tok.encode(), out.ctypes.data_as(ctypes.c_void_p))
        if rc != 0:
            raise ValueError(tok)
        return out[0]

    @staticmethod
    def _mat(n, entries):
        rows = np.array([e[0] for e in entries], np.int32)
        cols = np.array([e[1] for e in entries], np.int32)
        vals = np.array([e[2] for e in entries], DD)
        nnz = len(entries)
        effect = int(sum(1 if r == c else 2 for r, c in zip(rows, cols)))
        if nnz >= n * n * 0.20:  # SparseMatrix::changeToDense (sdpa_struct.cpp:458)
            D = np.zeros((n, n), DD)  # [col][row] so that ravel() is column-major
            for r, c, v in zip(rows, cols, vals):
                D[c, r] = v
                D[r, c] = v
            return {"dense": 1, "nnz": n * n, "effect": n * n, "rows": rows, "cols": cols, "val": D.ravel().copy()}
        return {"dense": 0, "nnz": nnz, "effect": effect, "rows": rows, "cols": cols, "val": vals}

    def _formulas(self):
        out = []
        for l in range(self.nblocks):
            cons = self.cons[l]
            nc = len(cons)
            con = np.array(cons, np.int32)
            dense = np.array([self.A[k][l]["dense"] for k in cons], np.int32)
            eff = np.array([self.A[k][l]["effect"] for k in cons], np.int32)
            f = np.zeros(nc, np.int32)
            self.lib.o_formula(ctypes.c_long(self.block_struct[l]), nc, con.ctypes.data_as(ctypes.c_void_p),
                               dense.ctypes.data_as(ctypes.c_void_p), eff.ctypes.data_as(ctypes.c_void_p),
                               ctypes.c_double(self.kappa), f.ctypes.data_as(ctypes.c_void_p))
            out.append(f)
        return out


class OAmat(ctypes.Structure):
    _fields_ = [("con", ctypes.c_int), ("dense", ctypes.c_int), ("nnz", ctypes.c_int), ("effect", ctypes.c_int),
                ("formula", ctypes.c_int), ("row", ctypes.c_void_p), ("col", ctypes.c_void_p), ("val", ctypes.c_void_p)]


def schur(problem: Problem, X_blocks, invZ_blocks):
    """B from the oracle (o_schur_block over the blocks in order)."""
    m = problem.m
    B = np.zeros(m * m, DD)
    keep = []
    for l in range(problem.nblocks):
        n = problem.block_struct[l]
        cons = problem.cons[l]
        arr = (OAmat * len(cons))()
        for t, k in enumerate(cons):
            a = problem.A[k][l]
            keep.append(a)
            arr[t].con = k
            arr[t].dense = a["dense"]
            arr[t].nnz = a["nnz"]
            arr[t].effect = a["effect"]
            arr[t].formula = int(problem.formula[l][t])
            arr[t].row = a["rows"].ctypes.data
            arr[t].col = a["cols"].ctypes.data
            arr[t].val = a["val"].ctypes.data
        X = np.ascontiguousarray(X_blocks[l])
        Zi = np.ascontiguousarray(invZ_blocks[l])
        problem.lib.o_schur_block(ctypes.c_long(m), ctypes.c_long(n), len(cons), arr,
                                  X.ctypes.data_as(ctypes.c_void_p), Zi.ctypes.data_as(ctypes.c_void_p),
                                  B.ctypes.data_as(ctypes.c_void_p))
    return B
