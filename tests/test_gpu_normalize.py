"""NORMALIZE_UVW on the device (rick_normalize_uvw; rick_plan_desc.normalize_uvw)
against the oracle, bit for bit."""
import numpy as np
import pytest

import oracle as O
import rick_b200 as R
from _util import TOL_FP64, gpu_rows, rel_l2, to_dev
from test_oracle import _uvw_cases

pytestmark = pytest.mark.gpu


def test_device_normalize_is_bit_exact():
    import torch
    for u, v, w in _uvw_cases():
        du, dv, dw = to_dev(u), to_dev(v), to_dev(w)
        scratch = torch.zeros(16, dtype=torch.float64, device="cuda")
        R.normalize_uvw(len(u), du, dv, dw, scratch)
        torch.cuda.synchronize()
        eu, ev, ew, ext = O.normalize_uvw(u, v, w)
        assert np.array_equal(du.cpu().numpy(), eu)
        assert np.array_equal(dv.cpu().numpy(), ev)
        assert np.array_equal(dw.cpu().numpy(), ew)
        assert np.array_equal(scratch[:7].cpu().numpy(), ext)


def test_plan_normalizes_before_gridding():
    import torch
    rng = np.random.default_rng(8)
    n, nchan, npol, nx, nw = 4000, 2, 2, 256, 4
    u = rng.normal(0, 900, n); v = rng.normal(0, 700, n); w = rng.normal(0, 40, n)
    wt = np.ones(n * npol, np.float32)
    vr = rng.standard_normal(n * nchan * npol).astype(np.float32)
    vi = rng.standard_normal(n * nchan * npol).astype(np.float32)
    rows = gpu_rows(u, v, w, wt, vr, vi)
    geom = R.Geometry(nx, nx, nw, 7, "gauss", "fp64")
    res, wmin, wmax = 1.0 / 2000.0, -60.0, 60.0
    with R.Plan(geom, n, nchan, npol, device=0, normalize_uvw=True) as plan:
        img = torch.empty(2 * nx * nx, dtype=torch.float64, device="cuda")
        plan.image(n, rows, res, wmin, wmax, img[: nx * nx], img[nx * nx:], R.ROWS_ALL)
        torch.cuda.synchronize()
        got = img.cpu().numpy()
        # the rows were rewritten in place, like the reference's data arrays
        eu, ev, ew, _ = O.normalize_uvw(u, v, w)
        assert np.array_equal(rows[0].cpu().numpy(), eu)
    grid, _ = O.wstack("gauss", nw, nchan, npol, eu, ev, ew, vr, vi, wt, 1 / nx, 1 / nw, 7, nx, nx)
    re, im = O.phase_correction(O.fft_planes(grid, nw, nx, nx), nx, nx, nw, res, wmin, wmax, True)
    assert rel_l2(got, np.concatenate([re, im])) < TOL_FP64
