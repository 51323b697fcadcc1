"""sdpa-dd_b200: the SDPA-DD double-double Newton hot path on NVIDIA B200.

The product is the C-ABI library `lib/libsddd.so` (include/sddd.h) and the
`bin/sdpa_dd_b200` command-line driver, built from csrc/ by build.py.  This
module binds the library with ctypes for tests and benchmarks; it has no
compute of its own and raises if the library is missing.
"""
from __future__ import annotations

import ctypes
import pathlib

import numpy as np

PKG = pathlib.Path(__file__).resolve().parent
LIB_PATH = PKG / "lib" / "libsddd.so"
BIN_PATH = PKG / "bin" / "sdpa_dd_b200"

DD = np.dtype([("hi", "<f8"), ("lo", "<f8")])


class SdddDD(ctypes.Structure):
    _fields_ = [("hi", ctypes.c_double), ("lo", ctypes.c_double)]


class SdddParam(ctypes.Structure):
    _fields_ = [("maxIteration", ctypes.c_int)] + [
        (n, ctypes.c_double)
        for n in ("epsilonStar", "lambdaStar", "omegaStar", "lowerBound", "upperBound", "betaStar", "betaBar", "gammaStar", "epsilonDash")
    ]


class SdddResult(ctypes.Structure):
    _fields_ = [("phase", ctypes.c_int), ("iterations", ctypes.c_int), ("stop_reason", ctypes.c_int),
                ("mu", SdddDD), ("relative_gap", SdddDD), ("gap", SdddDD), ("objValPrimal", SdddDD), ("objValDual", SdddDD),
                ("pfeas_error", SdddDD), ("dfeas_error", SdddDD),
                ("main_loop_seconds", ctypes.c_double), ("schur_seconds", ctypes.c_double), ("cholesky_seconds", ctypes.c_double)]


PHASES = ["noINFO", "pFEAS", "dFEAS", "pdFEAS", "pdINF", "pFEAS_dINF", "pINF_dFEAS", "pdOPT", "pUNBD", "dUNBD"]

_lib = None


class SdddSchurInfo(ctypes.Structure):
    """sddd_schur_info: the Schur form the reference's thresholds choose."""
    _fields_ = [("sparse", ctypes.c_int), ("m", ctypes.c_int), ("aggregate", ctypes.c_long), ("extended", ctypes.c_long),
                ("nnz", ctypes.c_long), ("ntiles", ctypes.c_long), ("reason", ctypes.c_char * 96)]


def lib() -> ctypes.CDLL:
    """The loaded libsddd.so (raises when it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: run `python sdpa-dd_b200/build.py`")
    L = ctypes.CDLL(str(LIB_PATH))
    vp, ci, cl, cd, cc = ctypes.c_void_p, ctypes.c_int, ctypes.c_long, ctypes.c_double, ctypes.c_char
    sig = {
        "sddd_version": (ctypes.c_char_p, []),
        "sddd_last_error": (ctypes.c_char_p, [vp]),
        "sddd_create": (ci, [ci, ctypes.POINTER(vp)]),
        "sddd_destroy": (ci, [vp]),
        "sddd_param_default": (ci, [ci, ctypes.POINTER(SdddParam)]),
        "sddd_param_read": (ci, [ctypes.c_char_p, ctypes.POINTER(SdddParam)]),
        "sddd_read_problem": (ci, [vp, ctypes.c_char_p, ci, cd]),
        "sddd_upload_problem": (ci, [vp, ci, ci, vp, vp, cl, vp, vp, vp, vp, vp, cd]),
        "sddd_dims": (ci, [vp, vp, vp, vp, vp, ci]),
        "sddd_space_len": (cl, [vp]),
        "sddd_formula": (ci, [vp, vp]),
        "sddd_init_point": (ci, [vp, SdddDD]),
        "sddd_set_point": (ci, [vp, vp, vp, vp]),
        "sddd_get_point": (ci, [vp, vp, vp, vp]),
        "sddd_compute_inverse": (ci, [vp]),
        "sddd_newton_rhs": (ci, [vp, ci, SdddDD, ci]),
        "sddd_schur_build": (ci, [vp]),
        "sddd_schur_factor": (ci, [vp]),
        "sddd_solve_dy": (ci, [vp]),
        "sddd_make_dz_dx": (ci, [vp, ci]),
        "sddd_min_eig": (ci, [vp, ci, ctypes.POINTER(SdddDD)]),
        "sddd_min_eig_noalloc": (ci, [vp, cl, vp, vp, vp]),
        "sddd_update": (ci, [vp, SdddDD, SdddDD]),
        "sddd_residuals": (ci, [vp, ctypes.POINTER(SdddDD), ctypes.POINTER(SdddDD)]),
        "sddd_inner": (ci, [vp, ci, ctypes.POINTER(SdddDD)]),
        "sddd_get": (cl, [vp, ci, vp]),
        "sddd_set": (ci, [vp, ci, vp]),
        "sddd_solve": (ci, [vp, ctypes.POINTER(SdddParam), ctypes.c_char_p, ci, ctypes.POINTER(SdddResult)]),
        "sddd_solver_start": (ci, [vp, ctypes.POINTER(SdddParam)]),
        "sddd_iterate": (ci, [vp]),
        "sddd_solver_result": (ci, [vp, ctypes.POINTER(SdddResult)]),
        "sddd_cli_main": (ci, [ci, vp]),
        "sddd_Rgemm": (ci, [vp, cc, cc, cl, cl, cl, SdddDD, vp, cl, vp, cl, SdddDD, vp, cl]),
        "sddd_Rpotrf": (ci, [vp, cc, cl, vp, cl]),
        "sddd_Rtrsv": (ci, [vp, cc, cc, cc, cl, vp, cl, vp, cl]),
        "sddd_Rpotrs": (ci, [vp, cc, cl, cl, vp, cl, vp, cl]),
        "sddd_set_tc_split": (ci, [vp, ci]),
        "sddd_set_wait_limit": (ci, [vp, cd]),
        "sddd_test_withhold_block": (ci, [vp, ci]),
        "sddd_get_tc_split": (ci, [vp]),
        "sddd_Rsyrk_tc": (ci, [vp, cl, cl, vp, cl, vp, cl, ci]),
        "sddd_Rdot_pairs_tc": (ci, [vp, cl, cl, vp, cl, vp, cl, vp, cl, ci]),
        "sddd_dd_op": (ci, [vp, ci, cl, vp, vp, vp]),
        "sddd_host_dd_op": (ci, [ci, cl, vp, vp, vp]),
        "sddd_host_dd_read": (ci, [ctypes.c_char_p, vp]),
        "sddd_host_dd_to_string": (ci, [SdddDD, ci, ctypes.c_char_p, ci]),
        "sddd_stream": (vp, [vp]),
        "sddd_launch_count": (ctypes.c_ulonglong, []),
        "sddd_profile": (ci, [vp, ci]),
        "sddd_profile_read": (ci, [vp, ctypes.c_char_p, ctypes.POINTER(cd), ctypes.POINTER(cl)]),
        "sddd_profile_reset": (ci, [vp]),
        "sddd_work": (ci, [vp, ctypes.POINTER(cd), ctypes.POINTER(cd)]),
        "sddd_fp64_peak": (ci, [vp, ctypes.POINTER(cd)]),
        "sddd_adjoint": (ci, [vp, vp, vp, vp, SdddDD, vp, vp]),
        "sddd_read_initial_point": (ci, [vp, ctypes.c_char_p, ci, cd]),
        "sddd_set_initial_point": (ci, [vp, vp, vp, vp]),
        "sddd_clear_initial_point": (ci, [vp]),
        "sddd_write_point": (ci, [vp, ctypes.c_char_p, ci]),
        "sddd_problem_info": (ci, [ctypes.c_char_p, ci, ctypes.POINTER(ci), ctypes.POINTER(ci), ctypes.POINTER(cl), vp, ci]),
        "sddd_dd_to_decimal": (ci, [SdddDD, ci, ctypes.c_char_p, ci]),
        "sddd_batch_create": (ci, [ci, ci, ctypes.POINTER(vp)]),
        "sddd_batch_destroy": (ci, [vp]),
        "sddd_batch_last_error": (ctypes.c_char_p, [vp]),
        "sddd_batch_add_file": (ci, [vp, ctypes.c_char_p, ci, cd]),
        "sddd_batch_add_problem": (ci, [vp, ci, ci, vp, vp, cl, vp, vp, vp, vp, vp, cd]),
        "sddd_batch_count": (ci, [vp]),
        "sddd_batch_solve": (ci, [vp, ctypes.POINTER(SdddParam), ci, vp]),
        "sddd_batch_status": (ci, [vp, ci]),
        "sddd_batch_get_point": (ci, [vp, ci, vp, vp, vp]),
        "sddd_batch_grad_c": (ci, [vp, ci, vp]),
        "sddd_adjoint_grad_F": (ci, [vp, ci, vp]),
        "sddd_batch_set_core": (ci, [vp, ci]),
        "sddd_batch_tuning": (ctypes.c_char_p, [vp]),
        "sddd_set_schur_mode": (ci, [vp, ci]),
        "sddd_schur_form": (ci, [vp, ctypes.POINTER(SdddSchurInfo), vp, vp, vp]),
        "sddd_plan_schur": (ci, [ctypes.c_char_p, ci, ci, ctypes.POINTER(SdddSchurInfo), vp, vp, vp]),
        "sddd_sparse_factor_values": (ci, [vp, vp]),
        "sddd_sparse_getCholesky": (ci, [vp, ci, vp, vp, vp]),
        "sddd_sparse_solveSystems": (ci, [vp, ci, vp, vp, vp, vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


class SdddError(RuntimeError):
    pass


class Context:
    """One device context (sddd_create) with its resident problem."""

    GET = {"X": 0, "Z": 1, "y": 2, "invCholX": 3, "invCholZ": 4, "invZ": 5, "B": 6, "g": 7, "Dx": 8, "Dy": 9, "Dz": 10,
           "dualMat": 11, "primalVec": 12, "adj_u": 13, "adj_R": 14}

    def __init__(self, device: int = 0):
        self.L = lib()
        h = ctypes.c_void_p()
        rc = self.L.sddd_create(device, ctypes.byref(h))
        if rc != 0:
            raise SdddError(f"sddd_create failed ({rc}): {self.L.sddd_last_error(None).decode()}")
        self.h = h

    def _check(self, rc, what):
        if rc < 0:
            raise SdddError(f"{what} failed ({rc}): {self.L.sddd_last_error(self.h).decode()}")
        return rc

    def close(self):
        if self.h:
            self.L.sddd_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def read_problem(self, path, sparse=True, kappa=1.2):
        self._check(self.L.sddd_read_problem(self.h, str(path).encode(), int(sparse), kappa), "read_problem")
        m, ns, nd = ctypes.c_int(), ctypes.c_int(), ctypes.c_long()
        sizes = np.zeros(4096, np.int32)
        self._check(self.L.sddd_dims(self.h, ctypes.byref(m), ctypes.byref(ns), ctypes.byref(nd), _ptr(sizes), 4096), "dims")
        self.m, self.nsdp, self.ndim = m.value, ns.value, nd.value
        self.sizes = [int(x) for x in sizes[: self.nsdp]]

    def _dims(self):
        m, ns, nd = ctypes.c_int(), ctypes.c_int(), ctypes.c_long()
        sizes = np.zeros(4096, np.int32)
        self._check(self.L.sddd_dims(self.h, ctypes.byref(m), ctypes.byref(ns), ctypes.byref(nd), _ptr(sizes), 4096), "dims")
        self.m, self.nsdp, self.ndim = m.value, ns.value, nd.value
        self.sizes = [int(x) for x in sizes[: self.nsdp]]

    def upload(self, m, block_struct, b, k, blk, i, j, val, kappa=1.2):
        """sddd_upload_problem: entries (k, blk, i, j, val) as in a .dat-s
        file (k = 0 is F_0; 1-based block, row, column); b and val are dd."""
        bs = np.ascontiguousarray(block_struct, np.int32)
        b = np.ascontiguousarray(b, DD)
        k, blk, i, j = (np.ascontiguousarray(a, np.int32) for a in (k, blk, i, j))
        val = np.ascontiguousarray(val, DD)
        self._check(self.L.sddd_upload_problem(self.h, int(m), len(bs), _ptr(bs), _ptr(b), len(val), _ptr(k), _ptr(blk), _ptr(i), _ptr(j),
                                               _ptr(val), kappa), "upload_problem")
        self._dims()

    def adjoint(self, g_x=None, g_Y=None, g_X=None, g_obj=(0.0, 0.0)):
        """sddd_adjoint at the current iterate; returns (grad_c, grad_F0)
        as dd arrays (grad_F0 a block space)."""
        keep = [None if a is None else np.ascontiguousarray(a, DD) for a in (g_x, g_Y, g_X)]
        gc = np.zeros(self.m, DD)
        gF0 = np.zeros(self.L.sddd_space_len(self.h), DD)
        self._check(self.L.sddd_adjoint(self.h, *[None if a is None else _ptr(a) for a in keep], SdddDD(*g_obj), _ptr(gc), _ptr(gF0)),
                    "adjoint")
        return gc, gF0

    def adjoint_grad_F(self, k):
        """Gradient with respect to F_k (k = 1..m) from the last adjoint."""
        out = np.zeros(self.L.sddd_space_len(self.h), DD)
        self._check(self.L.sddd_adjoint_grad_F(self.h, int(k), _ptr(out)), "adjoint_grad_F")
        return out

    def get(self, what):
        w = self.GET[what] if isinstance(what, str) else what
        n = self._check(self.L.sddd_get(self.h, w, None), "get")
        out = np.zeros(n, DD)
        self._check(self.L.sddd_get(self.h, w, _ptr(out)), "get")
        return out

    def set(self, what, arr):
        w = self.GET[what] if isinstance(what, str) else what
        arr = np.ascontiguousarray(arr, dtype=DD)
        self._check(self.L.sddd_set(self.h, w, _ptr(arr)), "set")

    def set_point(self, X, y, Z):
        X, y, Z = (np.ascontiguousarray(a, dtype=DD) for a in (X, y, Z))
        return self._check(self.L.sddd_set_point(self.h, _ptr(X), _ptr(y), _ptr(Z)), "set_point")

    def set_schur_mode(self, mode):
        """0 the reference's thresholds, 1 always dense, 2 always sparse."""
        self._check(self.L.sddd_set_schur_mode(self.h, mode), "sddd_set_schur_mode")

    def schur_form(self):
        """(info, order, diagonalIndex, column_index) of the attached problem."""
        info = SdddSchurInfo()
        self._check(self.L.sddd_schur_form(self.h, ctypes.byref(info), None, None, None), "sddd_schur_form")
        if not info.sparse:
            return info, None, None, None
        order = np.zeros(info.m, np.int32)
        di = np.zeros(info.m + 1, np.int32)
        ci_ = np.zeros(max(1, info.nnz), np.int32)
        self._check(self.L.sddd_schur_form(self.h, ctypes.byref(info), _ptr(order), _ptr(di), _ptr(ci_)), "sddd_schur_form")
        return info, order, di, ci_[:info.nnz]

    def sparse_factor_values(self, nnz):
        """The sparse factor of the last Schur factorisation (reference layout)."""
        out = np.zeros(nnz, DD)
        self._check(self.L.sddd_sparse_factor_values(self.h, _ptr(out)), "sddd_sparse_factor_values")
        return out

    def formula(self):
        out = np.zeros(self.m * self.nsdp, np.int32)
        self._check(self.L.sddd_formula(self.h, _ptr(out)), "formula")
        return out.reshape(self.m, self.nsdp)

    def call(self, name, *args):
        return self._check(getattr(self.L, name)(self.h, *args), name)

    def dd_scalar(self, name, *args):
        v = SdddDD()
        self._check(getattr(self.L, name)(self.h, *args, ctypes.byref(v)), name)
        return v.hi, v.lo

    def solve(self, param: SdddParam, result_path=None, print_=False):
        r = SdddResult()
        self._check(self.L.sddd_solve(self.h, ctypes.byref(param), None if result_path is None else str(result_path).encode(), int(print_),
                                      ctypes.byref(r)), "solve")
        return r


class Batch:
    """Independent problems solved together on one GPU (sddd_batch_*)."""

    def __init__(self, device: int = 0, workers: int = 0):
        self.L = lib()
        h = ctypes.c_void_p()
        rc = self.L.sddd_batch_create(device, workers, ctypes.byref(h))
        if rc != 0:
            raise SdddError(f"sddd_batch_create failed ({rc}): {self.L.sddd_last_error(None).decode()}")
        self.h = h
        self.dims = []  # (m, space length) per problem

    def close(self):
        if self.h:
            self.L.sddd_batch_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _added(self, rc, m, space_len):
        if rc < 0:
            raise SdddError(f"batch add failed ({rc}): {self.L.sddd_batch_last_error(self.h).decode()}")
        self.dims.append((m, space_len))
        return rc

    def add_file(self, path, m=None, space_len=None, sparse=True, kappa=1.2):
        """Adds a problem file; m and the block-space length default to
        the file's own (problem_info, read on the host)."""
        if m is None or space_len is None:
            m, _, space_len = problem_info(path, sparse)
        return self._added(self.L.sddd_batch_add_file(self.h, str(path).encode(), int(sparse), kappa), m, space_len)

    def add(self, m, block_struct, b, k, blk, i, j, val, kappa=1.2):
        bs = np.ascontiguousarray(block_struct, np.int32)
        b = np.ascontiguousarray(b, DD)
        k, blk, i, j = (np.ascontiguousarray(a, np.int32) for a in (k, blk, i, j))
        val = np.ascontiguousarray(val, DD)
        rc = self.L.sddd_batch_add_problem(self.h, int(m), len(bs), _ptr(bs), _ptr(b), len(val), _ptr(k), _ptr(blk), _ptr(i), _ptr(j), _ptr(val),
                                           kappa)
        return self._added(rc, int(m), int(sum(abs(int(x)) ** 2 for x in bs if x > 0)))

    def solve(self, param: SdddParam, with_grad=False):
        res = (SdddResult * len(self.dims))()
        rc = self.L.sddd_batch_solve(self.h, ctypes.byref(param), int(with_grad), ctypes.cast(res, ctypes.c_void_p))
        if rc < 0:
            raise SdddError(f"sddd_batch_solve failed ({rc}): {self.L.sddd_batch_last_error(self.h).decode()}")
        return list(res)

    def status(self, index):
        return self.L.sddd_batch_status(self.h, index)

    def point(self, index):
        m, L = self.dims[index]
        X, y, Z = np.zeros(L, DD), np.zeros(m, DD), np.zeros(L, DD)
        rc = self.L.sddd_batch_get_point(self.h, index, _ptr(X), _ptr(y), _ptr(Z))
        if rc != 0:
            raise SdddError(f"sddd_batch_get_point failed ({rc})")
        return X, y, Z

    def grad_c(self, index):
        out = np.zeros(self.dims[index][0], DD)
        rc = self.L.sddd_batch_grad_c(self.h, index, _ptr(out))
        if rc != 0:
            raise SdddError(f"sddd_batch_grad_c failed ({rc})")
        return out


def plan_schur(path, mode=0, sparse=True):
    """The Schur form of a problem file (host only): (info, order,
    diagonalIndex, column_index), the arrays None when B stays dense."""
    L = lib()
    info = SdddSchurInfo()
    rc = L.sddd_plan_schur(str(path).encode(), 1 if sparse else 0, mode, ctypes.byref(info), None, None, None)
    if rc != 0:
        raise SdddError(L.sddd_last_error(None).decode())
    if not info.sparse:
        return info, None, None, None
    order = np.zeros(info.m, np.int32)
    di = np.zeros(info.m + 1, np.int32)
    ci_ = np.zeros(max(1, info.nnz), np.int32)
    L.sddd_plan_schur(str(path).encode(), 1 if sparse else 0, mode, ctypes.byref(info), _ptr(order), _ptr(di), _ptr(ci_))
    return info, order, di, ci_[:info.nnz]


def problem_info(path, sparse=True):
    """(m, SDP block sizes, block-space length) of a problem file, read on
    the host only (sddd_problem_info: no device needed).  LP entries count
    as trailing blocks of order 1."""
    L = lib()
    m, ns, ln = ctypes.c_int(), ctypes.c_int(), ctypes.c_long()
    sizes = np.zeros(65536, np.int32)
    rc = L.sddd_problem_info(str(path).encode(), int(sparse), ctypes.byref(m), ctypes.byref(ns), ctypes.byref(ln), _ptr(sizes), len(sizes))
    if rc != 0:
        raise SdddError(f"sddd_problem_info failed ({rc}): {L.sddd_last_error(None).decode()}")
    return m.value, sizes[: min(ns.value, len(sizes))].tolist(), ln.value


def param(path=None, type_=0) -> SdddParam:
    p = SdddParam()
    L = lib()
    if path is None:
        rc = L.sddd_param_default(type_, ctypes.byref(p))
    else:
        rc = L.sddd_param_read(str(path).encode(), ctypes.byref(p))
    if rc != 0:
        raise SdddError(f"parameters: {rc}")
    return p
