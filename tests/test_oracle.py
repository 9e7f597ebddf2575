"""The oracle, pinned: against the golden fixtures (made by the reference's own
compiled code, tests/golden/make_golden.py) and, where the reference build is
present, against the reference bit for bit.  CPU only."""
import os

import numpy as np
import pytest

import oracle as O
from conftest import golden_cases
from _util import rel_l2

CASES = golden_cases()


def _packed(g):
    r = g["rows"].astype(np.int64)
    nv = g["nchan"] * g["npol"]
    return (g["uu"][r], g["vv"][r], g["ww"][r], g["weights"].reshape(-1, g["npol"])[r].ravel(),
            g["vis_re"].reshape(-1, nv)[r].ravel(), g["vis_im"].reshape(-1, nv)[r].ravel())


@pytest.mark.parametrize("case", CASES)
def test_rows_match_golden(case, golden):
    g = golden(case)
    rows = O.sector0_rows(g["vv"], g["nfile"], g["nx"], g["ny"], g["support"])
    assert np.array_equal(rows, g["rows"])


@pytest.mark.parametrize("case", CASES)
def test_wstack_bitexact_vs_golden(case, golden):
    g = golden(case)
    uu, vv, ww, wt, vr, vi = _packed(g)
    grid, dropped = O.wstack(g["kernel"], g["nw"], g["nchan"], g["npol"], uu, vv, ww, vr, vi, wt,
                             1.0 / g["nx"], 1.0 / g["nw"], g["support"], g["nx"], g["ny"],
                             threads=1)
    assert dropped == g["w_edge_removed"]
    assert np.array_equal(grid, g["grid"])


@pytest.mark.parametrize("case", CASES)
def test_phase_bitexact_vs_golden(case, golden):
    g = golden(case)
    gridss = O.fft_planes(g["grid"], g["nw"], g["nx"], g["ny"])
    re, im = O.phase_correction(gridss, g["nx"], g["ny"], g["nw"], g["resolution"], g["wmin"],
                                g["wmax"], threads=1)
    # same FFT implementation as the fixture generator: identical bits
    assert rel_l2(re, g["image_re"]) < 1e-15 and rel_l2(im, g["image_im"]) < 1e-15


def test_tables_symmetric_and_peaked():
    for kern in ("gauss", "kaiser_bessel"):
        for sup in (7, 9):
            t = O.table(kern, sup)
            n = 5 * sup
            assert np.allclose(t[: n // 2], t[::-1][: n // 2])   # w-stacking.cu:48,87
            assert np.argmax(t) == n // 2 and t[n // 2] > 0


def test_known_answer_single_visibility():
    """One visibility at a cell centre: footprint of C x C cells, table indices
    (int)(5*|u_dist + K|) with u_dist = j + 0.5 - pos_u (w-stacking.cu:162-176)."""
    nx = ny = 32
    nw, sup, K = 2, 7, 3
    pos = 10.5
    uu = np.array([pos / nx]); vv = np.array([pos / nx]); ww = np.array([0.75])
    vr = np.array([2.0, 0.0], np.float32); vi = np.array([-1.0, 0.0], np.float32)
    wt = np.array([0.5], np.float32)
    grid, dropped = O.wstack("gauss", nw, 2, 1, uu, vv, ww, vr, vi, wt, 1 / nx, 1 / nw, sup, nx,
                             ny, threads=1)
    assert dropped == 0
    cube = grid.view(np.complex128).reshape(nw, ny, nx)
    assert np.count_nonzero(cube[0]) == 0
    nz = np.argwhere(cube[1] != 0)
    assert nz[:, 0].min() == 10 - K and nz[:, 0].max() == 10 + K
    assert nz[:, 1].min() == 10 - K and nz[:, 1].max() == 10 + K
    tab = O.table("gauss", sup)
    for k in range(10 - K, 10 + K + 1):
        for j in range(10 - K, 10 + K + 1):
            jk = int(5 * abs(j + 0.5 - pos + K))
            kk = int(5 * abs(k + 0.5 - pos + K))
            want = (0.5 * 2.0) * (tab[jk] * tab[kk]) + 1j * (0.5 * -1.0) * (tab[jk] * tab[kk])
            assert cube[1, k, j] == want


def test_nan_sample_skipped():
    """A sample whose real part is NaN contributes nothing (w-stacking.cu:191-192)."""
    nx = ny = 16
    uu = np.array([0.5, 0.5]); vv = np.array([0.5, 0.5]); ww = np.array([0.1, 0.1])
    vr = np.array([1.0, np.nan], np.float32); vi = np.array([1.0, 5.0], np.float32)
    wt = np.array([1.0, 1.0], np.float32)
    g2, _ = O.wstack("kaiser_bessel", 1, 1, 1, uu, vv, ww, vr, vi, wt, 1 / nx, 1.0, 7, nx, ny)
    g1, _ = O.wstack("kaiser_bessel", 1, 1, 1, uu[:1], vv[:1], ww[:1], vr[:1], vi[:1], wt[:1],
                     1 / nx, 1.0, 7, nx, ny)
    assert np.array_equal(g1, g2)


def test_single_plane_is_plain_sum():
    """num_w_planes == 1: no phase screen (phase_correction.cu:202, :236-241)."""
    rng = np.random.default_rng(0)
    gridss = rng.standard_normal(2 * 8 * 8)
    re, im = O.phase_correction(gridss, 8, 8, 1, 1e-3, -10.0, 10.0)
    z = gridss.view(np.complex128)
    assert np.array_equal(re, z.real) and np.array_equal(im, z.imag)


@pytest.mark.skipif(not O.ref_available(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("kernel", ["gauss", "gauss_hi", "kaiser_bessel"])
def test_restatement_bitexact_vs_reference(kernel):
    """The restatement equals the reference's compiled wstack/phase_correction
    bit for bit on fresh random rows (single-threaded)."""
    rng = np.random.default_rng(7)
    n, nx, ny, nw, sup, nchan, npol = 3000, 96, 64, 5, 9 if kernel == "gauss_hi" else 7, 4, 2
    uu = rng.random(n); vv = rng.random(n); ww = rng.random(n) * 0.999
    wt = rng.random(n * npol).astype(np.float32)
    vr = rng.standard_normal(n * nchan * npol).astype(np.float32)
    vi = rng.standard_normal(n * nchan * npol).astype(np.float32)
    g1, _ = O.wstack(kernel, nw, nchan, npol, uu, vv, ww, vr, vi, wt, 1 / nx, 1 / nw, sup, nx, ny,
                     threads=1)
    g2 = np.zeros_like(g1)
    O.ref_lib(kernel).wstack(nw, n, nchan, npol, uu, vv, ww, vr, vi, wt, 1 / nx, 1 / nw, sup, nx,
                             ny, g2, 1, 0)
    assert np.array_equal(g1, g2)
    gss = O.fft_planes(g1, nw, nx, ny)
    r1, i1 = O.phase_correction(gss, nx, ny, nw, 3e-4, -300.0, 250.0, threads=1)
    r2, i2 = np.zeros(nx * ny), np.zeros(nx * ny)
    O.ref_lib(kernel).phase_correction(gss, r2, i2, nx, ny, nw, nx, ny, 3e-4, -300.0, 250.0, 1, 0)
    assert np.array_equal(r1, r2) and np.array_equal(i1, i2)


@pytest.mark.skipif(not O.ref_available(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("grid,sup", [(64, 7), (100, 9), (48, 3)])
def test_row_selection_vs_reference(grid, sup):
    rng = np.random.default_rng(grid)
    vv = rng.random(4000)
    vv[[3, 17]] = 1.0
    vv[25] = 1.0 + 0.5 / grid
    a = O.sector0_rows(vv, 5000, grid, grid, sup)
    b = O.ref_sector0_rows(vv, 4000, grid, grid, sup)
    assert np.array_equal(a, b)


def _uvw_cases():
    rng = np.random.default_rng(3)
    n = 5000
    for case in range(4):
        u = rng.normal(0, 3000, n); v = rng.normal(-100, 2000, n); w = rng.normal(5, 50, n)
        if case == 1:
            w = -np.abs(w) - 1            # every w negative: max w stays at its start value 0
        if case == 2:
            u, v = np.abs(u) + 10, np.abs(v) + 5
        if case == 3:
            u, v = -np.abs(u), -np.abs(v)
        yield u, v, w


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(O.__file__), "_ref",
                                                    "libref_norm.so")),
                    reason="reference build (oracle/_ref) not present")
def test_normalize_uvw_matches_reference_bit_for_bit():
    """gridding.c:21-83 through the reference's own gridding() (NORMALIZE_UVW,
    one rank) against the oracle's restatement."""
    for u, v, w in _uvw_cases():
        a = O.normalize_uvw(u, v, w)
        b = O.ref_normalize_uvw(u, v, w)
        for x, y in zip(a[:3], b):
            assert np.array_equal(x, y)


@pytest.mark.parametrize("kernel,nw,grid", [("gauss", 8, 256), ("kaiser_bessel", 5, 192),
                                            ("gauss_hi", 6, 128)])
def test_plane_chunked_oracle_is_bitexact(kernel, nw, grid):
    """The plane-at-a-time oracle (for cubes that do not fit in memory or pass
    the reference's 32-bit indices) equals the whole-cube oracle bit for bit,
    single-threaded: same rows, same drops, same image."""
    from rick_b200 import synth
    obs = synth.make_observation("c1", seed=11, time_fraction=0.08)
    sup = 9 if kernel == "gauss_hi" else 7
    a = O.image(obs, grid, grid, nw, kernel, sup, threads=1)
    b = O.image_chunked(obs, grid, grid, nw, kernel, sup, threads=1)
    assert (a["rows"], a["dropped"]) == (b["rows"], b["dropped"])
    assert np.array_equal(a["image_re"], b["image_re"])
    assert np.array_equal(a["image_im"], b["image_im"])
    assert np.abs(a["image_re"]).max() > 0
