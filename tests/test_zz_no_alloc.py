"""sddd_min_eig_noalloc, the allocation-free step-length eigenvalue, against
sddd_min_eig on the same block, on two calls in a row with different data.

The file name makes pytest collect it last, so it runs after every other
test has used the device; it also passes alone in a fresh process."""
import ctypes
import importlib

import numpy as np
import pytest

from conftest import DD, load_pkg

MAX_N = 4096  # SDDD_MIN_EIG_NOALLOC_MAX_N in include/sddd.h


def _dd(rng, hi):
    """dd values with a random low part below half an ulp of the high part."""
    out = np.zeros(hi.shape, DD)
    out["hi"] = hi
    out["lo"] = hi * rng.uniform(-1.0, 1.0, hi.shape) * 1e-17
    return out


def _block_pair(rng, n):
    """A lower-triangular L with a positive diagonal and a symmetric D,
    both n x n (row i, column j)."""
    Lh = np.tril(rng.normal(0.0, 0.3 / np.sqrt(n), (n, n)), -1) + np.diag(rng.uniform(0.5, 1.5, n))
    L = _dd(rng, Lh)
    L[np.triu_indices(n, 1)] = (0.0, 0.0)
    D = _dd(rng, rng.normal(0.0, 1.0, (n, n)))
    iu = np.triu_indices(n, 1)
    D[iu] = D.T[iu]
    return L, D


def _colmajor(a):
    return np.ascontiguousarray(a.ravel(order="F"))


@pytest.mark.gpu
@pytest.mark.parametrize("n", [12, 20, 21, 57, 200])
def test_noalloc_matches_min_eig_on_two_calls(n, tmp_path):
    import torch

    sddd = load_pkg()
    P = importlib.import_module("sdpa_dd_b200.problems")
    lib = sddd.lib()
    path = tmp_path / f"one_block_n{n}.dat-s"
    path.write_text(P.dense_random(n=n, m=3, seed=n))
    rng = np.random.default_rng(7000 + n)
    with sddd.Context(0) as ctx:
        ctx.read_problem(path)
        assert ctx.sizes == [n]
        stream = torch.cuda.current_stream()
        for call in range(2):
            L, D = _block_pair(rng, n)
            Lc, Dc = _colmajor(L), _colmajor(D)
            ctx.set("invCholX", Lc)
            ctx.set("Dx", Dc)
            want = ctx.dd_scalar("sddd_min_eig", 0)

            Ld = torch.from_numpy(Lc.view(np.float64).copy()).cuda()
            Dd = torch.from_numpy(Dc.view(np.float64).copy()).cuda()
            out = torch.full((2,), float("nan"), dtype=torch.float64, device="cuda")
            torch.cuda.synchronize()
            free_before = torch.cuda.mem_get_info()[0]
            rc = lib.sddd_min_eig_noalloc(ctypes.c_void_p(stream.cuda_stream), n, Ld.data_ptr(), Dd.data_ptr(), out.data_ptr())
            assert rc == 0, lib.sddd_last_error(None).decode()
            stream.synchronize()
            free_after = torch.cuda.mem_get_info()[0]
            got = out.cpu().numpy()
            # the same kernels in the same order as sddd_min_eig: identical bits
            assert (got[0], got[1]) == (want[0], want[1]), (n, call, tuple(got), want)
            if call == 1:
                # a warm call takes no device memory (the scratch array is
                # part of the loaded library image)
                assert free_after == free_before, (n, free_before, free_after)


def test_noalloc_rejects_orders_beyond_its_scratch():
    """The order check comes before any device work (no GPU needed)."""
    lib = load_pkg().lib()
    for n in (0, -3, MAX_N + 1, 1 << 40):
        rc = lib.sddd_min_eig_noalloc(None, n, None, None, None)
        assert rc == -1, n
        assert str(MAX_N).encode() in lib.sddd_last_error(None), n
