"""rick_wstack_noalloc: gridding for callers that cannot allocate device memory
at run time (pipelines that reserve all GPU memory up front, or frameworks that
own the device memory pool).  Its scratch is a static device array that keeps
the last call's contents, so a call must reproduce what the allocating plan
entry point grids whatever ran before it -- checked on a large job followed by
a smaller one with another geometry, kernel and support -- and a call must not
change the device's free memory.  Collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

import rick_b200 as R
from rick_b200 import synth
from _util import TOL_FP64, gpu_grid, gpu_rows, rel_l2

pytestmark = pytest.mark.gpu


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


def _call(f, rows, n, job, out):
    nx, nw, sup, kernel, nchan, npol = job
    uu, vv, ww, wt, vr, vi = rows
    return f(nw, n, nchan, npol, uu.data_ptr(), vv.data_ptr(), ww.data_ptr(), vr.data_ptr(),
             vi.data_ptr(), wt.data_ptr(), 1.0 / nx, 1.0 / nw, sup, R.KERNELS[kernel], nx, nx,
             out.data_ptr(), None)


def _job_rows(seed, fraction, nrows_max=None):
    obs = synth.make_observation("c1", seed=seed, time_fraction=fraction)
    n = R.rows_read(obs.meta)
    if nrows_max is not None:
        n = min(n, nrows_max)
    return gpu_rows(obs.uu[:n], obs.vv[:n], obs.ww[:n], obs.weights[: n * 2],
                    obs.vis_re[: n * 16], obs.vis_im[: n * 16]), n


def test_noalloc_matches_plan_on_two_calls_in_a_row():
    """A large job (1024^2 x 16 planes, Kaiser-Bessel 7, rows near the scratch
    limit) and then a small one (256^2 x 4 planes, Gaussian 9, few rows): the
    second call's bins, offsets and records sit in scratch the first call
    filled further, and its result must still equal the plan's."""
    import torch
    f, cap = _bind()
    big = (1024, 16, 7, "kaiser_bessel", 8, 2)
    small = (256, 4, 9, "gauss", 8, 2)
    limit = C.c_uint64(0)
    assert cap(big[1], big[0], big[0], C.byref(limit)) == R.OK
    rows_big, n_big = _job_rows(31, 1.0, nrows_max=int(limit.value))
    rows_small, n_small = _job_rows(32, 0.03)
    assert n_big > 10 * n_small
    for job, rows, n in ((big, rows_big, n_big), (small, rows_small, n_small)):
        nx, nw, sup, kernel, nchan, npol = job
        want, _ = gpu_grid(rows, n, nx, nx, nw, sup, kernel, nchan, npol, selection=R.ROWS_ALL)
        out = torch.full((2 * nw * nx * nx,), 123.0, dtype=torch.float64, device="cuda")
        assert _call(f, rows, n, job, out) == R.OK, R.last_error()   # overwrites the cube
        torch.cuda.synchronize()
        assert rel_l2(out.cpu().numpy(), want) < TOL_FP64


def test_noalloc_call_leaves_free_device_memory_unchanged():
    """After a first call (which sets the device up), a call changes the free
    device memory by nothing: it allocates nothing."""
    import torch
    f, _ = _bind()
    job = (512, 8, 7, "kaiser_bessel", 8, 2)
    rows, n = _job_rows(33, 0.05)
    out = torch.zeros(2 * 8 * 512 * 512, dtype=torch.float64, device="cuda")
    assert _call(f, rows, n, job, out) == R.OK, R.last_error()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    assert _call(f, rows, n, job, out) == R.OK, R.last_error()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_noalloc_rejects_jobs_beyond_its_scratch():
    """One row more than the stated capacity is refused before any work; the
    buffers passed are sized for that many rows all the same."""
    import torch
    f, cap = _bind()
    nx, nw = 512, 8
    limit = C.c_uint64(0)
    assert cap(nw, nx, nx, C.byref(limit)) == R.OK and limit.value > 10_000
    n = limit.value + 1
    d = dict(dtype=torch.float64, device="cuda")
    s = dict(dtype=torch.float32, device="cuda")
    rows = (torch.full((n,), 0.5, **d), torch.full((n,), 0.5, **d), torch.full((n,), 0.5, **d),
            torch.ones(n * 2, **s), torch.zeros(n * 16, **s), torch.zeros(n * 16, **s))
    st = _call(f, rows, n, (nx, nw, 7, "kaiser_bessel", 8, 2),
               torch.zeros(2 * nw * nx * nx, **d))
    assert st == R.ERR_INVALID_ARG
    assert "scratch" in R.last_error()
    torch.cuda.synchronize()
