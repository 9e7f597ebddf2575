"""Both forms of the CUDA path against the FP64 oracle on the three single-image
workloads at their full sizes (every row of the track, the full grid and plane
count):

  c1  512^2 x 8 planes, Gaussian 7, 279,800 rows x 8 chan x 2 pol
  c2  4096^2 x 32 planes, Kaiser-Bessel 7, 5,096,600 rows x 64 chan x 4 pol
      (1.305e9 visibilities) -- the whole-cube oracle (``oracle.image``)
  c3  8192^2 x 64 planes, high-precision Gaussian 9, 3,789,800 rows x 16 x 2
      -- the plane-chunked oracle (``oracle.image_chunked``): the FP64 cube is
      68.7 GB and its indices pass 2^32

Tolerances (relative L2 over the real and imaginary image planes): plain form
<= 1e-12, mixed form <= 1e-5.  The max-abs error relative to the image peak is
printed beside each.  The oracle runs on every host core (OpenMP) with
scipy's multi-threaded FFT; its row order within a plane is the reference's,
and its atomic FP64 adds make its own last bits thread-order dependent (far
below the tolerances)."""
import os

import numpy as np
import pytest

import oracle as O
import rick_b200 as R
from rick_b200 import synth
from _util import TOL_FP64, TOL_MIXED, rel_l2

pytestmark = pytest.mark.gpu


def _threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def _gpu_images(obs, cfg, forms):
    import torch
    n = R.rows_read(obs.meta)
    nv = cfg.nchan * cfg.npol
    rows = (obs.uu[:n].contiguous(), obs.vv[:n].contiguous(), obs.ww[:n].contiguous(),
            obs.weights[: n * cfg.npol].contiguous(), obs.vis_re[: n * nv].contiguous(),
            obs.vis_im[: n * nv].contiguous())
    g = cfg.grid
    out = {}
    for precision in forms:
        torch.cuda.empty_cache()
        img = torch.empty(2 * g * g, dtype=torch.float64, device="cuda")
        geom = R.Geometry(g, g, cfg.w_planes, cfg.w_support, cfg.kernel, precision)
        with R.Plan(geom, n, cfg.nchan, cfg.npol, device=0) as plan:
            plan.image(n, rows, R.resolution_of(obs.meta), obs.meta["wmin"], obs.meta["wmax"],
                       img[: g * g], img[g * g:], R.ROWS_SECTOR0)
            torch.cuda.synchronize()
            st = plan.stats()
        out[precision] = (img.cpu().numpy(), st)
        del img
    return out


def _check(name, got, ref):
    want = np.concatenate([ref["image_re"], ref["image_im"]])
    out = {}
    for precision, (img, stats) in got.items():
        err = rel_l2(img, want)
        mx = float(np.abs(img - want).max() / np.abs(want).max())
        print(f"{name} {precision}: rel L2 {err:.3e}, max-abs / peak {mx:.3e}, "
              f"rows gridded {stats['rows_gridded']} (oracle {ref['rows'] - ref['dropped']})")
        assert stats["rows_gridded"] == ref["rows"] - ref["dropped"]
        out[precision] = err
    assert out["fp64"] < TOL_FP64, out
    assert out["mixed"] < TOL_MIXED, out


def _run(name, chunked):
    import torch
    cfg = synth.CONFIGS[name]
    obs = synth.make_observation(cfg, seed=2024, device="cuda")
    got = _gpu_images(obs, cfg, ("fp64", "mixed"))
    host = synth.to_numpy(obs)
    del obs
    torch.cuda.empty_cache()
    oracle = O.image_chunked if chunked else O.image
    ref = oracle(host, cfg.grid, cfg.grid, cfg.w_planes, cfg.kernel, cfg.w_support,
                 threads=_threads(), fft_workers=_threads())
    _check(name, got, ref)


def test_c1_full_track_both_forms_vs_oracle():
    _run("c1", chunked=False)


def test_c2_lofar_like_both_forms_vs_oracle():
    _run("c2", chunked=False)


def test_c3_wide_field_both_forms_vs_plane_chunked_oracle():
    _run("c3", chunked=True)
