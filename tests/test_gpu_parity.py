"""Parity of the CUDA path (through the C ABI) with the reference and the oracle.

Plain form (FP64): relative L2 <= 1e-12 on the grid and the image.
Mixed form (FP32 grid/FFT): relative L2 <= 1e-5 on the image.
"""
import numpy as np
import pytest

import oracle as O
import rick_b200 as R
from conftest import golden_cases
from _util import TOL_FP64, TOL_MIXED, gpu_grid, gpu_image, gpu_rows, rel_l2

pytestmark = pytest.mark.gpu
CASES = golden_cases()


def _read_rows(g):
    n = g["nfile"] - 1000  # init.c:337-339
    nv = g["nchan"] * g["npol"]
    return n, gpu_rows(g["uu"][:n], g["vv"][:n], g["ww"][:n], g["weights"][: n * g["npol"]],
                       g["vis_re"][: n * nv], g["vis_im"][: n * nv])


def _packed_host(g):
    r = g["rows"].astype(np.int64)
    nv = g["nchan"] * g["npol"]
    return (np.ascontiguousarray(g["uu"][r]), np.ascontiguousarray(g["vv"][r]),
            np.ascontiguousarray(g["ww"][r]),
            np.ascontiguousarray(g["weights"].reshape(-1, g["npol"])[r].ravel()),
            np.ascontiguousarray(g["vis_re"].reshape(-1, nv)[r].ravel()),
            np.ascontiguousarray(g["vis_im"].reshape(-1, nv)[r].ravel()))


@pytest.mark.parametrize("case", CASES)
def test_grid_matches_reference(case, golden):
    g = golden(case)
    n, rows = _read_rows(g)
    grid, st = gpu_grid(rows, n, g["nx"], g["ny"], g["nw"], g["support"], g["kernel"], g["nchan"],
                        g["npol"])
    assert rel_l2(grid, g["grid"]) < TOL_FP64
    # sector-0 rows reach the grid, minus the rows of plane index Nw
    assert st["rows_gridded"] == len(g["rows"]) - g["w_edge_removed"]
    assert st["rows_dropped"] == n - st["rows_gridded"]
    # cells the reference leaves at zero stay exactly zero
    assert np.array_equal(grid == 0, g["grid"] == 0)


@pytest.mark.parametrize("case", CASES)
def test_image_matches_reference(case, golden):
    g = golden(case)
    n, rows = _read_rows(g)
    re, im, _ = gpu_image(rows, n, g["nx"], g["ny"], g["nw"], g["support"], g["kernel"],
                          g["nchan"], g["npol"], g["resolution"], g["wmin"], g["wmax"])
    assert rel_l2(re, g["image_re"]) < TOL_FP64
    assert rel_l2(im, g["image_im"]) < TOL_FP64


@pytest.mark.parametrize("case", CASES)
def test_mixed_image_within_1e5(case, golden):
    g = golden(case)
    n, rows = _read_rows(g)
    re, im, _ = gpu_image(rows, n, g["nx"], g["ny"], g["nw"], g["support"], g["kernel"],
                          g["nchan"], g["npol"], g["resolution"], g["wmin"], g["wmax"],
                          precision="mixed")
    err = rel_l2(np.concatenate([re, im]), np.concatenate([g["image_re"], g["image_im"]]))
    assert err < TOL_MIXED


@pytest.mark.parametrize("case", CASES)
def test_dropin_wstack_accumulates(case, golden):
    """w-stacking.h:39-57 through the C ABI: host arrays, grid += ..."""
    g = golden(case)
    R.set_kernel(g["kernel"])
    uu, vv, ww, wt, vr, vi = _packed_host(g)
    grid = np.zeros(2 * g["nw"] * g["nx"] * g["ny"])
    R.wstack(g["nw"], len(uu), g["nchan"], g["npol"], uu, vv, ww, vr, vi, wt, 1.0 / g["nx"],
             1.0 / g["nw"], g["support"], g["nx"], g["ny"], grid)
    assert rel_l2(grid, g["grid"]) < TOL_FP64
    R.wstack(g["nw"], len(uu), g["nchan"], g["npol"], uu, vv, ww, vr, vi, wt, 1.0 / g["nx"],
             1.0 / g["nw"], g["support"], g["nx"], g["ny"], grid)
    assert rel_l2(grid, 2 * g["grid"]) < TOL_FP64


@pytest.mark.parametrize("case", CASES)
def test_dropin_fft_and_phase(case, golden):
    """rick_fft_planes + phase_correction (w-stacking.h:70-83) on host buffers."""
    g = golden(case)
    nx, ny, nw = g["nx"], g["ny"], g["nw"]
    gridss = R.fft_planes(g["grid"], nw, nx, ny)
    assert rel_l2(gridss, O.fft_planes(g["grid"], nw, nx, ny)) < TOL_FP64
    re, im = np.zeros(nx * ny), np.zeros(nx * ny)
    R.set_phase_on(True)
    R.phase_correction(gridss, re, im, nx, ny, nw, nx, ny, g["resolution"], g["wmin"], g["wmax"])
    assert rel_l2(re, g["image_re"]) < TOL_FP64 and rel_l2(im, g["image_im"]) < TOL_FP64
    R.phase_correction(gridss, re, im, nx, ny, nw, nx, ny, g["resolution"], g["wmin"], g["wmax"])
    assert rel_l2(re, 2 * g["image_re"]) < TOL_FP64


@pytest.fixture(scope="module")
def c1_small():
    from rick_b200 import synth
    return synth.make_observation("c1", seed=11, time_fraction=0.25)


@pytest.mark.parametrize("kernel", ["gauss", "gauss_hi", "kaiser_bessel"])
def test_synthetic_c1_image_vs_oracle(kernel, c1_small):
    """Config-1 geometry (512^2 x 8 planes, sky model + noise), a quarter of the
    track, against the oracle pipeline (restated CPU path + FP64 FFT)."""
    obs = c1_small
    nx = ny = 512
    nw = 8
    sup = 9 if kernel == "gauss_hi" else 7
    ref = O.image(obs, nx, ny, nw, kernel, sup, threads=0)
    n = R.rows_read(obs.meta)
    rows = gpu_rows(obs.uu[:n], obs.vv[:n], obs.ww[:n], obs.weights[: n * 2],
                    obs.vis_re[: n * 16], obs.vis_im[: n * 16])
    res = R.resolution_of(obs.meta)
    re, im, st = gpu_image(rows, n, nx, ny, nw, sup, kernel, 8, 2, res, obs.meta["wmin"],
                           obs.meta["wmax"])
    assert st["rows_gridded"] == ref["rows"] - ref["dropped"]
    assert rel_l2(re, ref["image_re"]) < TOL_FP64 and rel_l2(im, ref["image_im"]) < TOL_FP64
    re2, im2, _ = gpu_image(rows, n, nx, ny, nw, sup, kernel, 8, 2, res, obs.meta["wmin"],
                            obs.meta["wmax"], precision="mixed")
    err = rel_l2(np.concatenate([re2, im2]), np.concatenate([ref["image_re"], ref["image_im"]]))
    assert err < TOL_MIXED


def test_non_square_grid_and_single_plane():
    rng = np.random.default_rng(5)
    n, nx, ny, nw, nchan, npol = 4000, 96, 40, 1, 3, 1
    uu = rng.random(n); vv = rng.random(n) * 0.9; ww = rng.random(n) * 0.999
    wt = rng.random(n * npol).astype(np.float32)
    vr = rng.standard_normal(n * nchan * npol).astype(np.float32)
    vi = rng.standard_normal(n * nchan * npol).astype(np.float32)
    want, dropped = O.wstack("kaiser_bessel", nw, nchan, npol, uu, vv, ww, vr, vi, wt, 1 / nx,
                             1 / nw, 7, nx, ny)
    grid, st = gpu_grid(gpu_rows(uu, vv, ww, wt, vr, vi), n, nx, ny, nw, 7, "kaiser_bessel",
                        nchan, npol, selection=R.ROWS_ALL)
    assert rel_l2(grid, want) < TOL_FP64
    assert st["rows_dropped"] == dropped


def test_empty_and_all_dropped():
    rng = np.random.default_rng(6)
    nx = ny = 64
    rows = gpu_rows(np.zeros(1), np.zeros(1), np.zeros(1), np.zeros(1, np.float32),
                    np.zeros(1, np.float32), np.zeros(1, np.float32))
    grid, st = gpu_grid(rows, 0, nx, ny, 4, 7, "gauss", 1, 1)
    assert not grid.any() and st["rows_gridded"] == 0
    n = 500   # every row on plane index Nw (w == 1.0): all dropped
    rows = gpu_rows(rng.random(n), rng.random(n) * 0.9, np.ones(n), np.ones(n, np.float32),
                    np.ones(n, np.float32), np.ones(n, np.float32))
    grid, st = gpu_grid(rows, n, nx, ny, 4, 7, "gauss", 1, 1)
    assert not grid.any() and st["rows_dropped"] == n
    re, im, st = gpu_image(rows, n, nx, ny, 4, 7, "gauss", 1, 1, 1e-3, -10.0, 10.0)
    assert not re.any() and not im.any()


def test_dense_tile_split_over_work_items():
    """Many rows in one tile: the tile is split into several work items whose
    partial tiles are combined with atomics; the sum must not change."""
    rng = np.random.default_rng(8)
    n, nx, nw = 200_000, 256, 2
    uu = 0.5 + 0.01 * rng.standard_normal(n); vv = 0.5 + 0.01 * rng.standard_normal(n)
    ww = rng.random(n) * 0.999
    wt = np.ones(n, np.float32)
    vr = rng.standard_normal(n).astype(np.float32); vi = rng.standard_normal(n).astype(np.float32)
    want, _ = O.wstack("kaiser_bessel", nw, 1, 1, uu, vv, ww, vr, vi, wt, 1 / nx, 1 / nw, 7, nx, nx)
    grid, st = gpu_grid(gpu_rows(uu, vv, ww, wt, vr, vi), n, nx, nx, nw, 7, "kaiser_bessel", 1, 1,
                        selection=R.ROWS_ALL)
    assert st["work_items"] > (nx // 32) ** 2 // 4   # dense tiles were split
    assert rel_l2(grid, want) < TOL_FP64


def test_plan_reuse_is_repeatable(c1_small):
    import torch
    obs = c1_small
    n = R.rows_read(obs.meta)
    rows = gpu_rows(obs.uu[:n], obs.vv[:n], obs.ww[:n], obs.weights[: n * 2],
                    obs.vis_re[: n * 16], obs.vis_im[: n * 16])
    geom = R.Geometry(512, 512, 8, 7, "kaiser_bessel", "fp64")
    with R.Plan(geom, n, 8, 2, device=0) as plan:
        imgs = []
        for _ in range(3):
            img = torch.empty(2 * 512 * 512, dtype=torch.float64, device="cuda")
            plan.image(n, rows, R.resolution_of(obs.meta), obs.meta["wmin"], obs.meta["wmax"],
                       img[: 512 * 512], img[512 * 512:])
            imgs.append(img.cpu().numpy())
    assert rel_l2(imgs[1], imgs[0]) < 1e-14 and rel_l2(imgs[2], imgs[0]) < 1e-14


def test_host_entry_point_matches_device(c1_small):
    obs = c1_small
    n = R.rows_read(obs.meta)
    nx = 512
    geom = R.Geometry(nx, nx, 8, 7, "kaiser_bessel", "fp64")
    res = R.resolution_of(obs.meta)
    with R.Plan(geom, n, 8, 2, device=0) as plan:
        re, im = np.zeros(nx * nx), np.zeros(nx * nx)
        host = (np.ascontiguousarray(obs.uu[:n]), np.ascontiguousarray(obs.vv[:n]),
                np.ascontiguousarray(obs.ww[:n]), np.ascontiguousarray(obs.weights[: n * 2]),
                np.ascontiguousarray(obs.vis_re[: n * 16]),
                np.ascontiguousarray(obs.vis_im[: n * 16]))
        plan.image_host(n, host, res, obs.meta["wmin"], obs.meta["wmax"], re, im)
    ref = O.image(obs, nx, nx, 8, "kaiser_bessel", 7)
    assert rel_l2(re, ref["image_re"]) < TOL_FP64 and rel_l2(im, ref["image_im"]) < TOL_FP64


def test_launch_count_advances():
    before = R.launch_count()
    rows = gpu_rows(np.array([0.5]), np.array([0.5]), np.array([0.5]), np.ones(1, np.float32),
                    np.ones(1, np.float32), np.ones(1, np.float32))
    gpu_image(rows, 1, 64, 64, 2, 7, "gauss", 1, 1, 1e-3, -1.0, 1.0)
    assert R.launch_count() - before >= 5


@pytest.mark.parametrize("slice_rows", [1000, 7919, 1 << 20])
def test_streaming_ingest_matches_host_call(c1_small, slice_rows):
    """rick_plan_ingest_*: samples in slices of rows give the image of the
    one-call host path (which the oracle pins)."""
    obs = c1_small
    n = R.rows_read(obs.meta)
    nx = 512
    geom = R.Geometry(nx, nx, 8, 7, "kaiser_bessel", "fp64")
    res = R.resolution_of(obs.meta)
    host = (np.ascontiguousarray(obs.uu[:n]), np.ascontiguousarray(obs.vv[:n]),
            np.ascontiguousarray(obs.ww[:n]), np.ascontiguousarray(obs.weights[: n * 2]),
            np.ascontiguousarray(obs.vis_re[: n * 16]), np.ascontiguousarray(obs.vis_im[: n * 16]))
    with R.Plan(geom, n, 8, 2, device=0) as plan:
        re0, im0 = np.zeros(nx * nx), np.zeros(nx * nx)
        plan.image_host(n, host, res, obs.meta["wmin"], obs.meta["wmax"], re0, im0, R.ROWS_SECTOR0)
        re, im = np.zeros(nx * nx), np.zeros(nx * nx)
        plan.ingest(n, host, res, obs.meta["wmin"], obs.meta["wmax"], re, im, R.ROWS_SECTOR0,
                    slice_rows=slice_rows)
    assert rel_l2(re, re0) < 1e-13 and rel_l2(im, im0) < 1e-13


def test_streaming_ingest_checks_the_row_order(c1_small):
    obs = c1_small
    n = 5000
    geom = R.Geometry(256, 256, 4, 7, "gauss", "fp64")
    host = (np.ascontiguousarray(obs.uu[:n]), np.ascontiguousarray(obs.vv[:n]),
            np.ascontiguousarray(obs.ww[:n]), np.ascontiguousarray(obs.weights[: n * 2]),
            np.ascontiguousarray(obs.vis_re[: n * 16]), np.ascontiguousarray(obs.vis_im[: n * 16]))
    L = R.lib()
    with R.Plan(geom, n, 8, 2, device=0) as plan:
        h = plan._h
        p = [R._ptr(x) for x in host]
        R.check(L.rick_plan_ingest_begin(h, n, p[0], p[1], p[2], p[3], R.ROWS_ALL), "begin")
        assert L.rick_plan_ingest_samples(h, 100, 10, p[4], p[5]) == R.ERR_INVALID_ARG  # skips rows
        R.check(L.rick_plan_ingest_samples(h, 0, 10, p[4], p[5]), "samples")
        out = np.zeros(256 * 256)
        assert L.rick_plan_ingest_end(h, 1e-3, -1.0, 1.0, R._ptr(out), R._ptr(out)) == \
            R.ERR_INVALID_ARG  # rows 10.. have no samples


@pytest.mark.parametrize("nchan,npol", [(64, 4), (5, 4), (33, 1)])
def test_wide_rows_match_oracle(nchan, npol):
    """Rows of many samples (64 x 4 is the LOFAR-like workload's row: the sample
    pass spreads it over 32 lanes with vector loads; 5 x 4 and 33 x 1 take the
    16- and 32-lane forms without them), a few NaN samples skipped as the
    reference skips them (w-stacking.cu:191-192)."""
    rng = np.random.default_rng(40 + nchan + npol)
    n, nx, nw = 2500, 256, 6
    uu = np.clip(0.5 + 0.18 * rng.standard_normal(n), 0, 1)
    vv = np.clip(0.5 + 0.18 * rng.standard_normal(n), 0, 0.9999)
    ww = rng.random(n) * 0.999
    wt = rng.uniform(0.5, 1.5, n * npol).astype(np.float32)
    vr = rng.standard_normal(n * nchan * npol).astype(np.float32)
    vi = rng.standard_normal(n * nchan * npol).astype(np.float32)
    vr[rng.random(vr.size) < 0.01] = np.nan
    want, dropped = O.wstack("kaiser_bessel", nw, nchan, npol, uu, vv, ww, vr, vi, wt, 1 / nx,
                             1 / nw, 7, nx, nx)
    rows = gpu_rows(uu, vv, ww, wt, vr, vi)
    grid, st = gpu_grid(rows, n, nx, nx, nw, 7, "kaiser_bessel", nchan, npol,
                        selection=R.ROWS_ALL)
    assert rel_l2(grid, want) < TOL_FP64
    assert st["rows_dropped"] == dropped
    res, wmin, wmax = 1.0 / (2.4 * nx), -140.0, 120.0
    gss = O.fft_planes(want, nw, nx, nx)
    want_re, want_im = O.phase_correction(gss, nx, nx, nw, res, wmin, wmax, True)
    re, im, _ = gpu_image(rows, n, nx, nx, nw, 7, "kaiser_bessel", nchan, npol, res, wmin, wmax,
                          selection=R.ROWS_ALL)
    assert rel_l2(re, want_re) < TOL_FP64 and rel_l2(im, want_im) < TOL_FP64
    re2, im2, _ = gpu_image(rows, n, nx, nx, nw, 7, "kaiser_bessel", nchan, npol, res, wmin,
                            wmax, selection=R.ROWS_ALL, precision="mixed")
    err = rel_l2(np.concatenate([re2, im2]), np.concatenate([want_re, want_im]))
    assert err < TOL_MIXED


def test_grid_and_plane_edges_match_oracle():
    """Rows on the edges: u, v at 0 and 1 and a few cells inside and outside
    them (footprints clipped by the grid or entirely off it; below -half a
    support the reference's unsigned bounds would wrap, so those rows are
    dropped), w on plane boundaries, at 0, just below 0 (truncation toward zero
    keeps it on plane 0), just below 1 and at 1 (dropped: plane Nw)
    (w-stacking.cu:143-149)."""
    nx, nw = 128, 5
    dx, dw = 1.0 / nx, 1.0 / nw
    edges = np.array([-4.5 * dx, -2.5 * dx, 0.0, 1e-12, 0.5 * dx, dx, 2.5 * dx, 0.5,
                      1 - 2.5 * dx, 1 - dx, 1 - 1e-12, 1.0, 1 + 2 * dx, 1 + 5 * dx])
    wvals = np.array([-1e-12, 0.0, dw, 2 * dw, 0.5, 4 * dw, 1 - 1e-12, 1.0])
    uu, vv, ww = [a.ravel() for a in np.meshgrid(edges, edges, wvals, indexing="ij")]
    n = len(uu)
    rng = np.random.default_rng(77)
    wt = rng.uniform(0.5, 1.5, n).astype(np.float32)
    vr = rng.standard_normal(n * 2).astype(np.float32)
    vi = rng.standard_normal(n * 2).astype(np.float32)
    for kernel, sup in (("kaiser_bessel", 7), ("gauss_hi", 9)):
        want, dropped = O.wstack(kernel, nw, 2, 1, uu, vv, ww, vr, vi, wt, dx, dw, sup, nx, nx)
        grid, st = gpu_grid(gpu_rows(uu, vv, ww, wt, vr, vi), n, nx, nx, nw, sup, kernel, 2, 1,
                            selection=R.ROWS_ALL)
        assert rel_l2(grid, want) < TOL_FP64, kernel
        assert st["rows_dropped"] == dropped > 0, kernel


def test_dropin_sequence_reuses_one_plan(golden):
    """The reference's call sequence through the drop-ins -- wstack
    (gridding_cpu.c:187-204), rick_fft_planes, phase_correction
    (fourier_transform.c:209-216) -- twice on the same cube: the image equals
    the reference's each time, and the second round creates no plan and
    allocates no row buffer (one cached plan serves all three calls)."""
    g = golden(CASES[0])
    nx, ny, nw = g["nx"], g["ny"], g["nw"]
    R.set_kernel(g["kernel"])
    R.set_phase_on(True)
    uu, vv, ww, wt, vr, vi = _packed_host(g)

    def one_round():
        grid = np.zeros(2 * nw * nx * ny)
        R.wstack(nw, len(uu), g["nchan"], g["npol"], uu, vv, ww, vr, vi, wt, 1.0 / nx, 1.0 / nw,
                 g["support"], nx, ny, grid)
        gridss = R.fft_planes(grid, nw, nx, ny)
        re, im = np.zeros(nx * ny), np.zeros(nx * ny)
        R.phase_correction(gridss, re, im, nx, ny, nw, nx, ny, g["resolution"], g["wmin"],
                           g["wmax"])
        assert rel_l2(re, g["image_re"]) < TOL_FP64 and rel_l2(im, g["image_im"]) < TOL_FP64

    one_round()
    before = R.dropin_counters()
    one_round()
    assert R.dropin_counters() == before


def test_dropins_on_large_pageable_buffers():
    """Buffers above the staging chunk (64 MiB) go through the pinned ring and
    the host thread pool: a 1024^2 x 8 cube (134 MB) through rick_fft_planes
    and phase_correction, and rows whose sample arrays are 77 MB through
    wstack, all on pageable numpy memory, against the oracle."""
    from rick_b200 import synth
    nx = ny = 1024
    nw = 8
    rng = np.random.default_rng(3)
    grid = rng.standard_normal(2 * nw * nx * ny)
    got = R.fft_planes(grid, nw, nx, ny)
    assert rel_l2(got, O.fft_planes(grid, nw, nx, ny)) < TOL_FP64
    re, im = np.zeros(nx * ny), np.zeros(nx * ny)
    R.set_phase_on(True)
    R.phase_correction(got, re, im, nx, ny, nw, nx, ny, 1.0 / 3000.0, -200.0, 180.0)
    want_re, want_im = O.phase_correction(got, nx, ny, nw, 1.0 / 3000.0, -200.0, 180.0)
    assert rel_l2(re, want_re) < TOL_FP64 and rel_l2(im, want_im) < TOL_FP64
    n, nchan, npol = 300_000, 64, 1
    uu = 0.25 + 0.5 * rng.random(n)
    vv = 0.25 + 0.5 * rng.random(n)
    ww = 0.999 * rng.random(n)
    wt = np.ones(n * npol, dtype=np.float32)
    vr = rng.standard_normal(n * nchan * npol).astype(np.float32)
    vi = rng.standard_normal(n * nchan * npol).astype(np.float32)
    R.set_kernel("kaiser_bessel")
    g = np.zeros(2 * nw * nx * ny)
    R.wstack(nw, n, nchan, npol, uu, vv, ww, vr, vi, wt, 1.0 / nx, 1.0 / nw, 7, nx, ny, g)
    want, _ = O.wstack("kaiser_bessel", nw, nchan, npol, uu, vv, ww, vr, vi, wt, 1.0 / nx,
                       1.0 / nw, 7, nx, ny)
    assert rel_l2(g, want) < TOL_FP64
