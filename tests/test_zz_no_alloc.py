"""rick_wstack_noalloc: gridding for callers that cannot allocate device memory
at run time (pipelines that reserve all GPU memory up front, or frameworks that
own the device memory pool).  Its scratch is a static device array, so two
calls in a row must each reproduce what the allocating plan entry point grids,
with nothing carried over from the earlier call.  Collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

import rick_b200 as R
from rick_b200 import synth
from _util import TOL_FP64, gpu_grid, gpu_rows, rel_l2

pytestmark = pytest.mark.gpu

NX = NY = 512
NW, SUP, KERNEL = 8, 7, "kaiser_bessel"


def _bind():
    L = R.lib()
    f = L.rick_wstack_noalloc
    f.argtypes = ([C.c_int, C.c_uint64, C.c_uint32, C.c_uint32] + [C.c_void_p] * 6 +
                  [C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p,
                   C.c_void_p])
    f.restype = C.c_int
    cap = L.rick_wstack_noalloc_capacity
    cap.argtypes = [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_uint64)]
    cap.restype = C.c_int
    return f, cap


def _call(f, rows, n, out):
    uu, vv, ww, wt, vr, vi = rows
    return f(NW, n, 8, 2, uu.data_ptr(), vv.data_ptr(), ww.data_ptr(), vr.data_ptr(),
             vi.data_ptr(), wt.data_ptr(), 1.0 / NX, 1.0 / NW, SUP, R.KERNELS[KERNEL], NX, NY,
             out.data_ptr(), None)


def test_noalloc_matches_plan_on_two_calls_in_a_row():
    import torch
    f, _ = _bind()
    out = torch.empty(2 * NW * NX * NY, dtype=torch.float64, device="cuda")
    for seed in (21, 22):
        obs = synth.make_observation("c1", seed=seed, time_fraction=0.05)
        n = R.rows_read(obs.meta)
        rows = gpu_rows(obs.uu[:n], obs.vv[:n], obs.ww[:n], obs.weights[: n * 2],
                        obs.vis_re[: n * 16], obs.vis_im[: n * 16])
        want, _ = gpu_grid(rows, n, NX, NY, NW, SUP, KERNEL, 8, 2, selection=R.ROWS_ALL)
        out.fill_(123.0)  # the entry point overwrites the cube
        assert _call(f, rows, n, out) == R.OK, R.last_error()
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert rel_l2(got, want) < TOL_FP64


def test_noalloc_rejects_jobs_beyond_its_scratch():
    """One row more than the stated capacity is refused before any work; the
    buffers passed are sized for that many rows all the same."""
    import torch
    f, cap = _bind()
    limit = C.c_uint64(0)
    assert cap(NW, NX, NY, C.byref(limit)) == R.OK and limit.value > 10_000
    n = limit.value + 1
    d = dict(dtype=torch.float64, device="cuda")
    s = dict(dtype=torch.float32, device="cuda")
    rows = (torch.full((n,), 0.5, **d), torch.full((n,), 0.5, **d), torch.full((n,), 0.5, **d),
            torch.ones(n * 2, **s), torch.zeros(n * 16, **s), torch.zeros(n * 16, **s))
    st = _call(f, rows, n, torch.zeros(2 * NW * NX * NY, **d))
    assert st == R.ERR_INVALID_ARG
    assert "scratch" in R.last_error()
    torch.cuda.synchronize()
