"""Generate the golden fixtures in tests/golden/ from the reference itself.

Run in a container that has the reference sources (oracle/Makefile `ref`
target builds oracle/_ref from them):

    make -C oracle ref && python tests/golden/make_golden.py

Every output here is computed by the reference's own compiled CPU code:
  * rows   : gridding.c:139-197 initialize_array (one rank), reversed as
             gridding_cpu.c:118 packs them, after init.c:337-339's 1000-row drop;
  * grid   : w-stacking.cu wstack, CPU branch, one OpenMP thread, per kernel macro;
  * image  : phase_correction.cu phase_correction, CPU branch, PHASE_ON, applied to
             numpy.fft.ifft2 of the grid (the FFTW_BACKWARD/(Nx*Ny) step of
             fourier_transform.c:34-76; FFTW is absent, pocketfft stands in).
Rows whose w-plane index equals Nw (w == 1.0) are removed before the reference
wstack is called, because it would write them past the end of the cube
(w-stacking.cu:168); the fixtures record how many were removed.

The inputs are seeded random rows (not a sky model): u, v concentrated toward
the uv centre like a real coverage plus a uniform part, w uniform, and rows
placed exactly on the edges u = 1, v = 1, w = 1 and on cell boundaries.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402

CASES = [
    # name, kernel, nx, ny, nw, support, nfile_rows, nchan, npol, nan_frac
    ("gauss_40x40x4_s7_c3p2_nan", "gauss", 40, 40, 4, 7, 1800, 3, 2, 0.02),
    ("kb_48x48x4_s7_c2p4", "kaiser_bessel", 48, 48, 4, 7, 1900, 2, 4, 0.0),
    ("gausshi_40x40x3_s9_c1p1", "gauss_hi", 40, 40, 3, 9, 1800, 1, 1, 0.0),
]


def make_rows(seed, nfile, nx, nchan, npol, nan_frac):
    rng = np.random.default_rng(seed)
    n_c = nfile // 2
    # centre-concentrated part + uniform part, in [0, 1]
    uu = np.concatenate([np.clip(0.5 + 0.08 * rng.standard_normal(n_c), 0, 1),
                         rng.random(nfile - n_c)])
    vv = np.concatenate([np.clip(0.5 + 0.08 * rng.standard_normal(n_c), 0, 1),
                         rng.random(nfile - n_c)])
    ww = rng.random(nfile)
    # edge rows (inside the rows that are read: before the last 1000)
    uu[5], vv[6], ww[7] = 1.0, 1.0, 1.0
    uu[8], vv[8] = 0.0, 0.0
    uu[9] = 17.0 / nx          # exactly on a cell boundary
    vv[9] = 0.5
    uu[11], vv[11] = 1.0, 1.0
    weights = rng.uniform(0.5, 1.5, nfile * npol).astype(np.float32)
    vr = rng.standard_normal(nfile * nchan * npol).astype(np.float32)
    vi = rng.standard_normal(nfile * nchan * npol).astype(np.float32)
    if nan_frac:
        vr[rng.random(vr.size) < nan_frac] = np.nan
    return uu, vv, ww, weights, vr, vi


def main():
    for k, (name, kernel, nx, ny, nw, sup, nfile, nchan, npol, nan_frac) in enumerate(CASES):
        uu, vv, ww, wt, vr, vi = make_rows(100 + k, nfile, nx, nchan, npol, nan_frac)
        nread = nfile - 1000                                  # init.c:337-339
        rows = O.ref_sector0_rows(vv[:nread], nread, nx, ny, sup)
        r = rows.astype(np.int64)
        dx, dw = 1.0 / nx, 1.0 / nw                           # init.c:11-12
        keep = (ww[r] / dw).astype(np.int64) < nw             # the reference would write these past the cube
        r_in = r[keep]
        nv = nchan * npol
        grid = np.zeros(2 * nw * nx * ny)
        R = O.ref_lib(kernel)
        R.wstack(nw, len(r_in), nchan, npol, np.ascontiguousarray(uu[r_in]),
                 np.ascontiguousarray(vv[r_in]), np.ascontiguousarray(ww[r_in]),
                 np.ascontiguousarray(vr.reshape(-1, nv)[r_in].ravel()),
                 np.ascontiguousarray(vi.reshape(-1, nv)[r_in].ravel()),
                 np.ascontiguousarray(wt.reshape(-1, npol)[r_in].ravel()), dx, dw, sup, nx, ny,
                 grid, 1, 0)
        gridss = O.fft_planes(grid, nw, nx, ny)
        uvmax = 2000.0 + 100 * k
        resolution = 1.0 / uvmax                              # gridding_cpu.c:78
        wmin, wmax = -150.0 - 10 * k, 140.0 + 5 * k
        img_re, img_im = np.zeros(nx * ny), np.zeros(nx * ny)
        R.phase_correction(np.ascontiguousarray(gridss), img_re, img_im, nx, ny, nw, nx, ny,
                           resolution, wmin, wmax, 1, 0)
        out = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(out, kernel=kernel, nx=nx, ny=ny, nw=nw, support=sup, nchan=nchan,
                            npol=npol, nfile=nfile, uu=uu, vv=vv, ww=ww, weights=wt, vis_re=vr,
                            vis_im=vi, rows=rows, w_edge_removed=int((~keep).sum()), grid=grid,
                            resolution=resolution, wmin=wmin, wmax=wmax, uvmin=-uvmax,
                            uvmax=uvmax, image_re=img_re, image_im=img_im)
        print(f"{out}: {len(rows)} rows ({int((~keep).sum())} w-edge removed), "
              f"{os.path.getsize(out)} bytes")


if __name__ == "__main__":
    main()
