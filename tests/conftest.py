"""Shared test plumbing: the gpu marker, the package loader and ctypes
handles on the oracle libraries (the CPU restatement in oracle/_build and
the reference build in oracle/_ref)."""
import ctypes
import importlib.util
import os
import pathlib
import subprocess
import sys

import numpy as np
import pytest

# The reference's Rdot combines OpenMP partial sums in arrival order
# (mplapack/Rdot_omp.cpp:97-111); one thread makes it deterministic.
os.environ.setdefault("OMP_NUM_THREADS", "1")
sys.path.insert(0, str(pathlib.Path(__file__).resolve().parents[1] / "oracle"))

ROOT = pathlib.Path(__file__).resolve().parents[1]
PKG_DIR = ROOT / "sdpa-dd_b200"
ORACLE_SO = ROOT / "oracle" / "_build" / "liboracle.so"
REF_SO = ROOT / "oracle" / "_ref" / "libsdpadd_ref.so"
REF_BIN = ROOT / "oracle" / "_ref" / "sdpa_dd"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def load_pkg():
    """Import the package directory `sdpa-dd_b200/` as `sdpa_dd_b200`."""
    if "sdpa_dd_b200" in sys.modules:
        return sys.modules["sdpa_dd_b200"]
    spec = importlib.util.spec_from_file_location(
        "sdpa_dd_b200", PKG_DIR / "__init__.py", submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["sdpa_dd_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


DD = np.dtype([("hi", "<f8"), ("lo", "<f8")])


def as_dd(a):
    """numpy array of dd values (structured hi/lo) from floats or pairs."""
    a = np.asarray(a)
    if a.dtype == DD:
        return np.ascontiguousarray(a)
    out = np.zeros(a.shape, dtype=DD)
    out["hi"] = a
    return out


def ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


@pytest.fixture(scope="session")
def oracle_lib():
    if not ORACLE_SO.exists():
        subprocess.run(["make", "-C", str(ROOT / "oracle"), "restated"], check=True, capture_output=True)
    lib = ctypes.CDLL(str(ORACLE_SO))
    return lib


@pytest.fixture(scope="session")
def ref_lib():
    if not REF_SO.exists():
        pytest.skip("reference build oracle/_ref not present")
    return ctypes.CDLL(str(REF_SO))


@pytest.fixture(scope="session")
def pkg():
    return load_pkg()


@pytest.fixture(scope="session")
def workdir(tmp_path_factory):
    return tmp_path_factory.mktemp("sddd")


class RefSolver:
    """ctypes wrapper over the reference's pinpal state (oracle/ref_capi.cpp)."""

    def __init__(self, lib, data, param=None, kappa=1.2):
        self.lib = lib
        lib.ref_open.restype = ctypes.c_void_p
        lib.ref_get.restype = ctypes.c_long
        self.h = lib.ref_open(str(data).encode(), None if param is None else str(param).encode(), ctypes.c_double(kappa))
        if not self.h:
            raise RuntimeError("ref_open failed")
        self.h = ctypes.c_void_p(self.h)
        dims = np.zeros(4096, np.int32)
        assert lib.ref_dims(self.h, ptr(dims), 4096) > 0
        self.m, self.nsdp, self.nlp, self.ndim = map(int, dims[:4])
        self.blocks = [int(x) for x in dims[4:4 + self.nsdp]]

    def get(self, what):
        n = self.lib.ref_get(self.h, what, None)
        out = np.zeros(n, DD)
        self.lib.ref_get(self.h, what, ptr(out))
        return out

    def blocks_of(self, flat):
        out, off = [], 0
        for n in self.blocks:
            out.append(flat[off:off + n * n].copy())
            off += n * n
        return out

    def scalar(self, what):
        out = np.zeros(1, DD)
        self.lib.ref_scalar(self.h, what, ptr(out))
        return out[0]

    def step(self):
        return self.lib.ref_step(self.h)

    def schur(self):
        out = np.zeros(self.m * self.m, DD)
        self.lib.ref_schur(self.h, ptr(out))
        return out

    def formula(self):
        out = np.zeros(self.m * self.nsdp, np.int32)
        self.lib.ref_formula(self.h, ptr(out))
        return out.reshape(self.m, self.nsdp)

    def close(self):
        if self.h:
            self.lib.ref_close(self.h)
            self.h = None
