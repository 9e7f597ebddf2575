"""Shared helpers for the parity tests (GPU runs go through the C ABI)."""
from __future__ import annotations

import numpy as np

import rick_b200 as R

# Tolerances (relative L2 on the image / grid against the oracle).
TOL_FP64 = 1e-12   # plain form: FP64 grid and FFT
TOL_MIXED = 1e-5   # mixed form: FP32 grid and FFT


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))


def to_dev(a, dtype=None):
    import torch
    a = np.ascontiguousarray(a if dtype is None else np.asarray(a, dtype=dtype))
    return torch.from_numpy(a).cuda()


def gpu_rows(uu, vv, ww, weights, vis_re, vis_im):
    return (to_dev(uu, np.float64), to_dev(vv, np.float64), to_dev(ww, np.float64),
            to_dev(weights, np.float32), to_dev(vis_re, np.float32), to_dev(vis_im, np.float32))


def gpu_grid(rows, n, nx, ny, nw, support, kernel, nchan, npol, precision="fp64",
             selection=R.ROWS_SECTOR0):
    """Grid device rows with a plan; return the cube as FP64 numpy (wstack layout)."""
    import torch
    geom = R.Geometry(nx, ny, nw, support, kernel, precision)
    with R.Plan(geom, max(n, 1), nchan, npol, device=0) as plan:
        plan.grid(n, rows, selection)
        out = torch.empty(2 * nw * nx * ny, dtype=torch.float64, device="cuda")
        plan.export_cube(out, dst_is_host=False)
        torch.cuda.synchronize()
        stats = plan.stats()
        return out.cpu().numpy(), stats


def gpu_image(rows, n, nx, ny, nw, support, kernel, nchan, npol, resolution, wmin, wmax,
              precision="fp64", selection=R.ROWS_SECTOR0, phase_on=True):
    import torch
    geom = R.Geometry(nx, ny, nw, support, kernel, precision, phase_on)
    with R.Plan(geom, max(n, 1), nchan, npol, device=0) as plan:
        img = torch.empty(2 * nx * ny, dtype=torch.float64, device="cuda")
        plan.image(n, rows, resolution, wmin, wmax, img[: nx * ny], img[nx * ny:], selection)
        torch.cuda.synchronize()
        stats = plan.stats()
        im = img.cpu().numpy()
        return im[: nx * ny], im[nx * ny:], stats
