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
