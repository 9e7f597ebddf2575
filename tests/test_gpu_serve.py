"""Served imaging (rick_server_*): jobs arriving while others run are admitted
by HBM footprint and batched; each job's image is the same alone and in the
mix, within the stated tolerance."""
import threading
import time

import numpy as np
import pytest

import rick_b200 as R
from _util import TOL_MIXED, gpu_image, gpu_rows, rel_l2
from test_gpu_batch import JOBS, _host_rows, _oracle, _params

pytestmark = pytest.mark.gpu


def _served_jobs(copies):
    import torch
    out = []
    for c in range(copies):
        for i, (nx, ny, nw, kernel, sup, nchan, npol, n, sel) in enumerate(JOBS):
            if n == 0:
                continue
            h = _host_rows(100 + i, n, nchan, npol)
            img = torch.full((2 * nx * ny,), float("nan"), dtype=torch.float64, device="cuda")
            res, wmin, wmax = _params(i, nx, ny)
            job = R.Job(R.Geometry(nx, ny, nw, sup, kernel, "mixed"), n, nchan, npol,
                        gpu_rows(*h), res, wmin, wmax, img[: nx * ny], img[nx * ny:], sel)
            out.append((i, h, img, job))
    return out


def test_served_results_equal_alone():
    import torch
    items = _served_jobs(3)
    rng = np.random.default_rng(5)
    tickets = [None] * len(items)
    with R.Server("mixed", device=0, hbm_budget=6 * 10**9, max_batch_jobs=4, streams=2) as srv:
        def producer():
            for k, (_, _, _, job) in enumerate(items):
                tickets[k] = srv.submit(job)
                time.sleep(float(rng.exponential(0.002)))   # Poisson arrivals, ~500 jobs/s
        th = threading.Thread(target=producer)
        th.start()
        th.join()
        results = [srv.wait(t, timeout_ms=60_000) for t in tickets]
        st = srv.stats()
    torch.cuda.synchronize()
    assert st["jobs_done"] == len(items) and st["jobs_waiting"] == 0
    assert st["batches"] >= 2 and st["peak_bytes"] <= 6 * 10**9
    assert all(r["status"] == 0 and r["latency_ms"] >= r["queue_ms"] >= 0 for r in results)
    alone = {}
    for (i, h, img, _), r in zip(items, results):
        nx, ny, nw, kernel, sup, nchan, npol, n, sel = JOBS[i]
        if i not in alone:
            res, wmin, wmax = _params(i, nx, ny)
            re, im, _ = gpu_image(gpu_rows(*h), n, nx, ny, nw, sup, kernel, nchan, npol, res,
                                  wmin, wmax, precision="mixed", selection=sel)
            alone[i] = np.concatenate([re, im])
            want_re, want_im = _oracle(i, h)
            assert rel_l2(alone[i], np.concatenate([want_re, want_im])) < TOL_MIXED
        got = img.cpu().numpy()
        # FP32 tile sums of split tiles add in any order: equal to FP32 rounding
        assert rel_l2(got, alone[i]) < 1e-6, (i, r)


def test_server_rejects_job_over_budget():
    items = _served_jobs(1)
    with R.Server("mixed", device=0, hbm_budget=10**4, max_batch_jobs=4, streams=1) as srv:
        with pytest.raises(R.RickError) as e:
            srv.submit(items[0][3])
        assert e.value.status == R.ERR_BUDGET


def _big_job(seed, img):
    """A 4096^2 x 32-plane mixed job with uniform random rows on every plane:
    some milliseconds on the device, long enough to hold later jobs waiting."""
    import torch
    g = torch.Generator(device="cuda").manual_seed(seed)
    n, nchan, npol, nx, nw = 400_000, 16, 4, 4096, 32
    d = dict(device="cuda", generator=g)
    rows = (0.05 + 0.9 * torch.rand(n, dtype=torch.float64, **d),
            0.05 + 0.9 * torch.rand(n, dtype=torch.float64, **d),
            0.999 * torch.rand(n, dtype=torch.float64, **d),
            torch.ones(n * npol, dtype=torch.float32, device="cuda"),
            torch.randn(n * nchan * npol, dtype=torch.float32, **d),
            torch.randn(n * nchan * npol, dtype=torch.float32, **d))
    return R.Job(R.Geometry(nx, nx, nw, 7, "kaiser_bessel", "mixed"), n, nchan, npol, rows,
                 1e-5, -50.0, 60.0, img[: nx * nx], img[nx * nx:], R.ROWS_ALL)


def _wait_launched(srv, batches, limit_s=20.0):
    t0 = time.time()
    while srv.stats()["batches"] < batches:
        assert time.time() - t0 < limit_s, srv.stats()
        time.sleep(0.0002)


def test_shutdown_mid_stream_cancels_waiting_jobs():
    """A server shut down (drain=False) while one job runs and two wait: the
    running job completes with the image it has alone, the waiting ones come
    back RICK_ERR_CANCELLED, and later submissions are refused the same way.
    The failure is made on the host: no kernel is interrupted."""
    import torch
    imgs = [torch.full((2 * 4096 * 4096,), float("nan"), dtype=torch.float64, device="cuda")
            for _ in range(3)]
    jobs = [_big_job(40 + k, imgs[k]) for k in range(3)]
    need = R.Batch.footprint([jobs[0]], "mixed")
    with R.Server("mixed", device=0, hbm_budget=int(need * 1.5), max_batch_jobs=4,
                  streams=1) as srv:
        tickets = [srv.submit(j) for j in jobs]
        _wait_launched(srv, 1)
        srv.shutdown(drain=False)
        assert srv.wait(tickets[0], timeout_ms=60_000)["status"] == R.OK
        for t in tickets[1:]:
            with pytest.raises(R.RickError) as e:
                srv.wait(t, timeout_ms=60_000)
            assert e.value.status == R.ERR_CANCELLED
        with pytest.raises(R.RickError) as e:
            srv.submit(jobs[1])
        assert e.value.status == R.ERR_CANCELLED
        st = srv.stats()
    torch.cuda.synchronize()
    assert st["jobs_done"] == 1 and st["batches"] == 1
    j = jobs[0]
    re, im, _ = gpu_image(j.rows, j.nrows, 4096, 4096, 32, 7, "kaiser_bessel", 16, 4,
                          j.resolution, j.wmin, j.wmax, precision="mixed", selection=R.ROWS_ALL)
    assert rel_l2(imgs[0].cpu().numpy(), np.concatenate([re, im])) < 1e-6
    assert torch.isnan(imgs[1]).all() and torch.isnan(imgs[2]).all()   # never launched


def test_cancel_a_waiting_job():
    """cancel() takes a job out of the queue before it is launched; a job
    already launched cannot be cancelled and completes."""
    import torch
    imgs = [torch.full((2 * 4096 * 4096,), float("nan"), dtype=torch.float64, device="cuda")
            for _ in range(2)]
    jobs = [_big_job(50 + k, imgs[k]) for k in range(2)]
    need = R.Batch.footprint([jobs[0]], "mixed")
    with R.Server("mixed", device=0, hbm_budget=int(need * 1.5), max_batch_jobs=4,
                  streams=1) as srv:
        a, b = srv.submit(jobs[0]), srv.submit(jobs[1])
        _wait_launched(srv, 1)
        assert srv.cancel(b) is True
        assert srv.cancel(a) is False
        assert srv.wait(a, timeout_ms=60_000)["status"] == R.OK
        with pytest.raises(R.RickError) as e:
            srv.wait(b, timeout_ms=60_000)
        assert e.value.status == R.ERR_CANCELLED
    torch.cuda.synchronize()
    assert not torch.isnan(imgs[0]).any() and torch.isnan(imgs[1]).all()
