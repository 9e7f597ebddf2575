"""Batched imaging (rick_batch_*): every job of a batch against the oracle and
against the same job imaged alone by a plan; graph replays, explicit and
autotuned schedules, argument checks."""
import numpy as np
import pytest

import oracle as O
import rick_b200 as R
from _util import TOL_FP64, TOL_MIXED, gpu_image, gpu_rows, rel_l2

pytestmark = pytest.mark.gpu

# (nx, ny, nw, kernel, support, nchan, npol, rows, selection)
JOBS = [
    (64, 64, 2, "gauss", 3, 1, 1, 900, R.ROWS_ALL),
    (256, 256, 8, "kaiser_bessel", 7, 2, 2, 5000, R.ROWS_ALL),
    (128, 512, 3, "gauss_hi", 9, 1, 2, 3000, R.ROWS_SECTOR0),
    (512, 512, 4, "kaiser_bessel", 7, 4, 2, 8000, R.ROWS_ALL),
    (1024, 1024, 1, "gauss", 7, 3, 2, 4000, R.ROWS_ALL),
    (256, 128, 5, "gauss", 5, 2, 1, 0, R.ROWS_ALL),  # no rows: an all-zero image
    (256, 4096, 10, "kaiser_bessel", 7, 2, 2, 6000, R.ROWS_ALL),  # 4096-point columns
]


def _host_rows(seed, n, nchan, npol):
    rng = np.random.default_rng(seed)
    uu = np.clip(0.5 + 0.15 * rng.standard_normal(n), 0, 1)
    vv = np.clip(0.5 + 0.15 * rng.standard_normal(n), 0, 1.0)
    ww = rng.random(n) * 0.999
    wt = rng.uniform(0.5, 1.5, n * npol).astype(np.float32)
    vr = rng.standard_normal(n * nchan * npol).astype(np.float32)
    vi = rng.standard_normal(n * nchan * npol).astype(np.float32)
    return uu, vv, ww, wt, vr, vi


def _params(i, nx, ny):
    return 1.0 / (2.3 * max(nx, ny)), -80.0 - 10 * i, 70.0 + 5 * i


def _make(precision):
    import torch
    jobs, host = [], []
    for i, (nx, ny, nw, kernel, sup, nchan, npol, n, sel) in enumerate(JOBS):
        h = _host_rows(100 + i, n, nchan, npol)
        rows = gpu_rows(*h) if n else tuple(torch.empty(1, device="cuda") for _ in range(6))
        img = torch.full((2 * nx * ny,), float("nan"), dtype=torch.float64, device="cuda")
        res, wmin, wmax = _params(i, nx, ny)
        geom = R.Geometry(nx, ny, nw, sup, kernel, precision)
        jobs.append(R.Job(geom, n, nchan, npol, rows, res, wmin, wmax, img[: nx * ny],
                          img[nx * ny:], sel))
        host.append((h, img))
    return jobs, host


def _oracle(i, h):
    nx, ny, nw, kernel, sup, nchan, npol, n, sel = JOBS[i]
    res, wmin, wmax = _params(i, nx, ny)
    uu, vv, ww, wt, vr, vi = h
    if sel == R.ROWS_SECTOR0:
        keep = O.sector0_rows(vv, n + 1000, nx, ny, sup).astype(np.int64)
        nv = nchan * npol
        uu, vv, ww = uu[keep], vv[keep], ww[keep]
        wt = wt.reshape(n, npol)[keep].ravel()
        vr = vr.reshape(n, nv)[keep].ravel()
        vi = vi.reshape(n, nv)[keep].ravel()
    grid, _ = O.wstack(kernel, nw, nchan, npol, uu, vv, ww, vr, vi, wt, 1 / nx, 1 / nw, sup, nx, ny)
    gss = O.fft_planes(grid, nw, nx, ny)
    return O.phase_correction(gss, nx, ny, nw, res, wmin, wmax, True)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_matches_oracle(precision):
    import torch
    jobs, host = _make(precision)
    tol = TOL_FP64 if precision == "fp64" else TOL_MIXED
    with R.Batch(jobs, precision, device=0) as b:
        b.run()
        torch.cuda.synchronize()
        first = [img.cpu().numpy().copy() for _, img in host]
        for i, (h, img) in enumerate(host):
            nx, ny = JOBS[i][0], JOBS[i][1]
            re, im = first[i][: nx * ny], first[i][nx * ny:]
            if JOBS[i][7] == 0:
                assert not np.any(re) and not np.any(im)
                continue
            want_re, want_im = _oracle(i, h)
            err = rel_l2(np.concatenate([re, im]), np.concatenate([want_re, want_im]))
            assert err < tol, (i, err)
        # a graph replay recomputes the same images (split tiles add in any
        # order: FP64 sums agree to rounding, FP32 sums to FP32 rounding)
        for _, img in host:
            img.fill_(float("nan"))
        b.run()
        torch.cuda.synchronize()
        for i, (_, img) in enumerate(host):
            again = img.cpu().numpy()
            assert rel_l2(again, first[i]) < (1e-13 if precision == "fp64" else 1e-6)
        st = b.stats()
        assert st["rows_in"] == sum(j[7] for j in JOBS)
        assert st["rows_gridded"] + st["rows_dropped"] == st["rows_in"]
        t = b.tuning()
        assert t["max_chunk"] >= 64 and t["grid_blocks_per_sm"] >= 1
        assert t["planes_in_flight"] in (0, 1, 2)   # 0: column-pass state in tensor memory


def test_batch_equals_plans_alone():
    """Each job in the batch gives the image the plan API gives for it alone."""
    import torch
    jobs, host = _make("fp64")
    tune = {"max_chunk": 1024, "grid_blocks_per_sm": 4, "planes_in_flight": 1}
    with R.Batch(jobs, "fp64", device=0, tuning=tune) as b:
        assert b.tuning() == tune
        b.run()
        torch.cuda.synchronize()
        for i, (h, img) in enumerate(host):
            nx, ny, nw, kernel, sup, nchan, npol, n, sel = JOBS[i]
            if n == 0:
                continue
            res, wmin, wmax = _params(i, nx, ny)
            re, im, _ = gpu_image(gpu_rows(*h), n, nx, ny, nw, sup, kernel, nchan, npol, res,
                                  wmin, wmax, selection=sel)
            got = img.cpu().numpy()
            assert rel_l2(got, np.concatenate([re, im])) < 1e-13, i


def test_batch_footprint_and_rejections():
    import torch
    jobs, _ = _make("mixed")
    assert R.Batch.footprint(jobs, "mixed") < R.Batch.footprint(jobs, "fp64")
    bad = list(jobs)
    j = bad[1]
    g = R.Geometry(384, 384, 2, 7, "gauss", "mixed")   # not a power of two
    bad[1] = R.Job(g, j.nrows, j.freq_per_chan, j.polarizations, j.rows, j.resolution, j.wmin,
                   j.wmax, j.image_re, j.image_im)
    with pytest.raises(R.RickError) as e:
        R.Batch(bad, "mixed", device=0)
    assert e.value.status == R.ERR_INVALID_ARG
    g = R.Geometry(8192, 8192, 1, 7, "gauss", "mixed")  # above the batch limit
    bad[1] = R.Job(g, j.nrows, j.freq_per_chan, j.polarizations, j.rows, j.resolution, j.wmin,
                   j.wmax, j.image_re, j.image_im)
    with pytest.raises(R.RickError):
        R.Batch(bad, "mixed", device=0)
    with pytest.raises(R.RickError):
        R.Batch([], "mixed", device=0)
    torch.cuda.synchronize()
