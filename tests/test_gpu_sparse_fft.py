"""The sparse-aware FFT path of rick_plan_image (power-of-two grids: touched-row
FFT, column FFT fused with the w-correction) against the oracle and against the
dense path (full cube, cuFFT, separate w-correction; RICK_DENSE_FFT=1)."""
import os

import numpy as np
import pytest

import oracle as O
import rick_b200 as R
from _util import TOL_FP64, TOL_MIXED, gpu_image, gpu_rows, rel_l2

pytestmark = pytest.mark.gpu


def _rows(seed, n, nchan, npol, spread=0.15, wmax=0.999):
    rng = np.random.default_rng(seed)
    uu = np.clip(0.5 + spread * rng.standard_normal(n), 0, 1)
    vv = np.clip(0.5 + spread * rng.standard_normal(n), 0, 0.9999)
    ww = rng.random(n) * wmax
    wt = rng.uniform(0.5, 1.5, n * npol).astype(np.float32)
    vr = rng.standard_normal(n * nchan * npol).astype(np.float32)
    vi = rng.standard_normal(n * nchan * npol).astype(np.float32)
    return uu, vv, ww, wt, vr, vi


def _dense_image(*args, **kw):
    os.environ["RICK_DENSE_FFT"] = "1"
    try:
        return gpu_image(*args, **kw)
    finally:
        del os.environ["RICK_DENSE_FFT"]


def _oracle_image(host, nx, ny, nw, kernel, sup, nchan, npol, res, wmin, wmax, phase_on=True):
    uu, vv, ww, wt, vr, vi = host
    grid, _ = O.wstack(kernel, nw, nchan, npol, uu, vv, ww, vr, vi, wt, 1 / nx, 1 / nw, sup, nx, ny)
    gss = O.fft_planes(grid, nw, nx, ny)
    return O.phase_correction(gss, nx, ny, nw, res, wmin, wmax, phase_on)


@pytest.mark.parametrize("nx,ny,nw,kernel,sup", [
    (256, 256, 8, "kaiser_bessel", 7),
    (256, 128, 4, "gauss", 7),      # non-square
    (128, 512, 3, "gauss_hi", 9),
    (64, 64, 2, "kaiser_bessel", 3),  # smallest supported axis
    (1024, 1024, 1, "gauss", 7),    # single plane: plain sum
    (256, 4096, 12, "kaiser_bessel", 7),  # 4096-point columns (64 x 64), anchors + steps
    (4096, 128, 3, "gauss", 7),     # 4096-point rows
    (128, 8192, 10, "kaiser_bessel", 7),  # 8192-point columns, phase at every plane
])
def test_sparse_path_vs_oracle(nx, ny, nw, kernel, sup):
    n, nchan, npol = 6000, 2, 2
    host = _rows(nx + ny + nw, n, nchan, npol)
    rows = gpu_rows(*host)
    res, wmin, wmax = 1.0 / (2.4 * max(nx, ny)), -120.0, 95.0
    want_re, want_im = _oracle_image(host, nx, ny, nw, kernel, sup, nchan, npol, res, wmin, wmax)
    re, im, st = gpu_image(rows, n, nx, ny, nw, sup, kernel, nchan, npol, res, wmin, wmax,
                           selection=R.ROWS_ALL)
    assert rel_l2(re, want_re) < TOL_FP64 and rel_l2(im, want_im) < TOL_FP64
    re2, im2, _ = gpu_image(rows, n, nx, ny, nw, sup, kernel, nchan, npol, res, wmin, wmax,
                            selection=R.ROWS_ALL, precision="mixed")
    err = rel_l2(np.concatenate([re2, im2]), np.concatenate([want_re, want_im]))
    assert err < TOL_MIXED


def test_sparse_path_phase_off():
    nx = ny = 256
    nw, n = 6, 5000
    host = _rows(3, n, 1, 2)
    rows = gpu_rows(*host)
    want_re, want_im = _oracle_image(host, nx, ny, nw, "gauss", 7, 1, 2, 1e-3, -50.0, 60.0,
                                     phase_on=False)
    re, im, _ = gpu_image(rows, n, nx, ny, nw, 7, "gauss", 1, 2, 1e-3, -50.0, 60.0,
                          selection=R.ROWS_ALL, phase_on=False)
    assert rel_l2(re, want_re) < TOL_FP64 and rel_l2(im, want_im) < TOL_FP64


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_sparse_matches_dense_at_8192(precision):
    """The largest supported axis (8192) with a thin track, against the dense
    cuFFT path on the same plan geometry."""
    nx = ny = 8192
    nw, n, nchan, npol = 2, 20000, 1, 2
    host = _rows(9, n, nchan, npol, spread=0.05)
    rows = gpu_rows(*host)
    args = (rows, n, nx, ny, nw, 9, "gauss_hi", nchan, npol, 2e-5, -900.0, 800.0)
    re, im, _ = gpu_image(*args, precision=precision, selection=R.ROWS_ALL)
    re_d, im_d, _ = _dense_image(*args, precision=precision, selection=R.ROWS_ALL)
    tol = TOL_FP64 if precision == "fp64" else TOL_MIXED
    assert rel_l2(re, re_d) < tol and rel_l2(im, im_d) < tol


def test_sparse_path_empty_planes_and_rows():
    """Planes with no rows at all, and a single row: exact zeros stay exact."""
    nx = ny = 512
    nw = 16
    uu = np.array([0.5]); vv = np.array([0.25]); ww = np.array([0.40])  # plane 6 only
    host = (uu, vv, ww, np.ones(1, np.float32), np.ones(1, np.float32), np.zeros(1, np.float32))
    rows = gpu_rows(*host)
    want_re, want_im = _oracle_image(host, nx, ny, nw, "kaiser_bessel", 7, 1, 1, 1e-3, -10.0, 10.0)
    re, im, _ = gpu_image(rows, 1, nx, ny, nw, 7, "kaiser_bessel", 1, 1, 1e-3, -10.0, 10.0,
                          selection=R.ROWS_ALL)
    assert rel_l2(re, want_re) < TOL_FP64 and rel_l2(im, want_im) < TOL_FP64


def test_fused_image_refuses_export():
    import torch
    nx = 256
    host = _rows(4, 100, 1, 1)
    rows = gpu_rows(*host)
    with R.Plan(R.Geometry(nx, nx, 2, 7, "gauss"), 100, 1, 1, device=0) as plan:
        img = torch.empty(2 * nx * nx, dtype=torch.float64, device="cuda")
        plan.image(100, rows, 1e-3, -1.0, 1.0, img[: nx * nx], img[nx * nx:], R.ROWS_ALL)
        with pytest.raises(R.RickError) as e:
            plan.export_cube(torch.empty(2 * 2 * nx * nx, dtype=torch.float64, device="cuda"),
                             dst_is_host=False)
        assert e.value.status == R.ERR_INVALID_ARG
        # the stage path still produces the full cube
        plan.grid(100, rows, R.ROWS_ALL)
        plan.export_cube(torch.empty(2 * 2 * nx * nx, dtype=torch.float64, device="cuda"),
                         dst_is_host=False)


def test_mixed_phase_recurrence_skips_empty_planes():
    """Rows only on planes 1, 2, 5, 13, 14 of 16 (gaps of 1, 3, 8, 1 planes): the
    mixed form's plane-to-plane phase advance must span the skipped planes."""
    nx = ny = 512
    nw, n = 16, 4000
    rng = np.random.default_rng(17)
    planes = np.array([1, 2, 5, 13, 14])
    ww = (planes[rng.integers(0, len(planes), n)] + rng.uniform(0.1, 0.9, n)) / nw
    uu = np.clip(0.5 + 0.2 * rng.standard_normal(n), 0, 1)
    vv = np.clip(0.5 + 0.2 * rng.standard_normal(n), 0, 0.9999)
    host = (uu, vv, ww, np.ones(n, np.float32), rng.standard_normal(n).astype(np.float32),
            rng.standard_normal(n).astype(np.float32))
    rows = gpu_rows(*host)
    res, wmin, wmax = 1.0 / 1300.0, -2500.0, 2200.0
    want_re, want_im = _oracle_image(host, nx, ny, nw, "kaiser_bessel", 7, 1, 1, res, wmin, wmax)
    for precision, tol in (("fp64", TOL_FP64), ("mixed", TOL_MIXED)):
        re, im, _ = gpu_image(rows, n, nx, ny, nw, 7, "kaiser_bessel", 1, 1, res, wmin, wmax,
                              selection=R.ROWS_ALL, precision=precision)
        err = rel_l2(np.concatenate([re, im]), np.concatenate([want_re, want_im]))
        assert err < tol, (precision, err)


def _pair_case_rows(seed, n, nw, planes=None):
    rng = np.random.default_rng(seed)
    if planes is None:
        ww = rng.random(n) * 0.999
    else:
        planes = np.asarray(planes)
        ww = (planes[rng.integers(0, len(planes), n)] + rng.uniform(0.1, 0.9, n)) / nw
    uu = np.clip(0.5 + 0.2 * rng.standard_normal(n), 0, 1)
    vv = np.clip(0.5 + 0.2 * rng.standard_normal(n), 0, 0.9999)
    return (uu, vv, ww, rng.uniform(0.5, 1.5, 2 * n).astype(np.float32),
            rng.standard_normal(2 * n).astype(np.float32),
            rng.standard_normal(2 * n).astype(np.float32))


@pytest.mark.parametrize("nx,ny,nw,phase_on,planes", [
    (128, 2048, 5, True, None),                 # 2048-point columns (radix-4 last pass)
    (64, 1024, 6, False, None),                 # 1024-point columns (radix-2), phase off
    (256, 1024, 16, True, [1, 2, 5, 13, 14]),   # planes without rows between planes with rows
    (64, 4096, 7, True, [0, 6]),                # the first and last planes only
    (64, 8192, 6, True, [0, 3, 5]),             # 8192 points: FP64 split in halves, FP32 pairs
    (128, 8192, 3, False, None),                # 8192 points, PHASE_ON off
])
def test_two_column_pass_vs_oracle(nx, ny, nw, phase_on, planes):
    """Column lengths 1024..8192 run two transforms per block, one pass apart
    (at 8192 FP64, the even and odd rows of one column): each form against the
    oracle, including plane gaps and PHASE_ON off."""
    n = 5000
    host = _pair_case_rows(nx + ny + nw, n, nw, planes)
    rows = gpu_rows(*host)
    res, wmin, wmax = 1.0 / (2.3 * max(nx, ny)), -700.0, 650.0
    want_re, want_im = _oracle_image(host, nx, ny, nw, "kaiser_bessel", 7, 1, 2, res, wmin, wmax,
                                     phase_on=phase_on)
    want = np.concatenate([want_re, want_im])
    for precision, tol in (("fp64", TOL_FP64), ("mixed", TOL_MIXED)):
        re, im, _ = gpu_image(rows, n, nx, ny, nw, 7, "kaiser_bessel", 1, 2, res, wmin, wmax,
                              selection=R.ROWS_ALL, precision=precision, phase_on=phase_on)
        err = rel_l2(np.concatenate([re, im]), want)
        assert err < tol, (precision, err)


def test_image_rows_at_an_odd_address():
    """Image arrays that do not start on a 16-byte boundary (one double past
    it): the column pass writes them element by element, with the same values."""
    import torch
    nx, ny, nw, n = 128, 4096, 4, 4000
    host = _pair_case_rows(5, n, nw)
    rows = gpu_rows(*host)
    res, wmin, wmax = 1.0 / 9000.0, -300.0, 280.0
    want_re, want_im = _oracle_image(host, nx, ny, nw, "kaiser_bessel", 7, 1, 2, res, wmin, wmax)
    geom = R.Geometry(nx, ny, nw, 7, "kaiser_bessel", "fp64")
    with R.Plan(geom, n, 1, 2, device=0) as plan:
        buf = torch.full((2 * nx * ny + 1,), float("nan"), dtype=torch.float64, device="cuda")
        plan.image(n, rows, res, wmin, wmax, buf[1: 1 + nx * ny], buf[1 + nx * ny:], R.ROWS_ALL)
        torch.cuda.synchronize()
        got = buf.cpu().numpy()
    assert np.isnan(got[0])
    assert rel_l2(got[1:], np.concatenate([want_re, want_im])) < TOL_FP64
