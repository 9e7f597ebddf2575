"""Parity oracle for RICK's imaging hot path (TEST INFRASTRUCTURE ONLY).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU legs import this
module, and only as the checker or as the timed CPU baseline.  The product
library never routes through it.

* ``liboracle.so`` (built from oracle/rick_oracle.c) restates the reference's
  CPU ``wstack`` (w-stacking.cu:211-536), ``phase_correction``
  (phase_correction.cu:97-250) and one-rank row selection (init.c:335-340,
  gridding.c:139-188, gridding_cpu.c:118-138) with 64-bit indices.
* The FFT between them is ``numpy.fft.ifft2`` in FP64 on each (Ny, Nx) plane,
  which equals fourier_transform.c:34-76 (FFTW_BACKWARD, then x 1/(Nx*Ny)).
  FFTW itself is third-party and absent here; pocketfft stands in.
* ``oracle/_ref/libref_*.so`` are the reference's own sources compiled
  unmodified (oracle/Makefile); ``ref_*`` functions call them.  They pin the
  restatement bit-for-bit in single-threaded runs.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
KERNELS = {"gauss": 0, "gauss_hi": 1, "kaiser_bessel": 2}
REF_LIBS = {"gauss": "libref_gauss.so", "gauss_hi": "libref_gauss_hi.so",
            "kaiser_bessel": "libref_kb.so"}

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_fp = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")

_lib = None
_ref = {}


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError(f"oracle library missing: {path} (run `make -C oracle`)")
        L = C.CDLL(path)
        L.oracle_wstack.argtypes = [C.c_int, C.c_int, C.c_uint64, C.c_uint32, C.c_uint32,
                                    _dp, _dp, _dp, _fp, _fp, _fp, C.c_double, C.c_double,
                                    C.c_int, C.c_int, C.c_int, _dp, C.c_int,
                                    C.POINTER(C.c_uint64)]
        L.oracle_wstack.restype = C.c_int
        L.oracle_phase_correction.argtypes = [_dp, _dp, _dp, C.c_int, C.c_int, C.c_int, C.c_int,
                                              C.c_int, C.c_double, C.c_double, C.c_double,
                                              C.c_int, C.c_int]
        L.oracle_phase_correction.restype = C.c_int
        L.oracle_phase_correction_planes.argtypes = [_dp, _dp, _dp, C.c_int, C.c_int, C.c_int,
                                                     C.c_int, C.c_int, C.c_int, C.c_int,
                                                     C.c_double, C.c_double, C.c_double,
                                                     C.c_int, C.c_int]
        L.oracle_phase_correction_planes.restype = C.c_int
        L.oracle_sector0_rows.argtypes = [_dp, C.c_uint64, C.c_int, C.c_int, C.c_int, _u64p]
        L.oracle_sector0_rows.restype = C.c_uint64
        L.oracle_normalize_uvw.argtypes = [C.c_uint64, _dp, _dp, _dp, _dp]
        L.oracle_normalize_uvw.restype = None
        L.oracle_make_gauss_table.argtypes = [_dp, C.c_int]
        L.oracle_make_kb_table.argtypes = [_dp, C.c_int]
        _lib = L
    return _lib


def ref_available(kernel: str = "kaiser_bessel") -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", REF_LIBS[kernel]))


def ref_lib(kernel: str):
    """The reference's own CPU wstack/phase_correction for one kernel macro."""
    if kernel not in _ref:
        path = os.path.join(HERE, "_ref", REF_LIBS[kernel])
        if not os.path.exists(path):
            raise RuntimeError(f"reference build missing: {path} (run `make -C oracle ref`)")
        L = C.CDLL(path, mode=C.RTLD_LOCAL)
        # w-stacking.h:39-57 (C prototype) and w-stacking.h:70-83
        L.wstack.argtypes = [C.c_int, C.c_uint, C.c_uint, C.c_uint, _dp, _dp, _dp, _fp, _fp, _fp,
                             C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, _dp, C.c_int,
                             C.c_int]
        L.wstack.restype = None
        L.phase_correction.argtypes = [_dp, _dp, _dp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                       C.c_double, C.c_double, C.c_double, C.c_int, C.c_int]
        L.phase_correction.restype = None
        _ref[kernel] = L
    return _ref[kernel]


def table(kernel: str, w_support: int) -> np.ndarray:
    t = np.zeros(5 * w_support)
    if kernel == "gauss":
        lib().oracle_make_gauss_table(t, w_support)
    elif kernel == "kaiser_bessel":
        lib().oracle_make_kb_table(t, w_support)
    return t


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def wstack(kernel, nw, nchan, npol, uu, vv, ww, vis_re, vis_im, weights, dx, dw, w_support,
           nx, ny, grid=None, threads=0):
    """Restated CPU wstack; accumulates into ``grid`` (2*nw*ny*nx doubles)."""
    n = len(uu)
    if grid is None:
        grid = np.zeros(2 * nw * nx * ny)
    dropped = C.c_uint64(0)
    rc = lib().oracle_wstack(KERNELS[kernel], nw, n, nchan, npol, _c(uu, np.float64),
                             _c(vv, np.float64), _c(ww, np.float64), _c(vis_re, np.float32),
                             _c(vis_im, np.float32), _c(weights, np.float32), dx, dw, w_support,
                             nx, ny, grid, threads, C.byref(dropped))
    assert rc == 0
    return grid, int(dropped.value)


def fft_planes(grid, nw, nx, ny, workers=None):
    """fourier_transform.c:34-76: per plane FFTW_BACKWARD x 1/(Nx*Ny)."""
    z = grid.view(np.complex128).reshape(nw, ny, nx)
    if workers:
        import scipy.fft as sfft
        out = sfft.ifft2(z, axes=(-2, -1), workers=workers)
    else:
        out = np.fft.ifft2(z, axes=(-2, -1))
    return np.ascontiguousarray(out).view(np.float64).reshape(-1)


def phase_correction(gridss, nx, ny, nw, resolution, wmin, wmax, phase_on=True, threads=0,
                     image_re=None, image_im=None):
    if image_re is None:
        image_re = np.zeros(nx * ny)
        image_im = np.zeros(nx * ny)
    rc = lib().oracle_phase_correction(_c(gridss, np.float64), image_re, image_im, nx, ny, nw, nx,
                                       ny, resolution, wmin, wmax, int(phase_on), threads)
    assert rc == 0
    return image_re, image_im


def phase_correction_planes(gridss, nx, ny, nw, w_first, w_count, resolution, wmin, wmax,
                            image_re, image_im, phase_on=True, threads=0):
    """phase_correction.cu:185-250 over planes w_first..w_first+w_count-1 of an
    nw-plane cube (``gridss`` holds only those planes), accumulating into the
    image; consecutive ranges give the bits of one whole-cube call."""
    rc = lib().oracle_phase_correction_planes(_c(gridss, np.float64), image_re, image_im, nx, ny,
                                              nw, w_first, w_count, nx, ny, resolution, wmin,
                                              wmax, int(phase_on), threads)
    assert rc == 0
    return image_re, image_im


def plane_of(ww, nw):
    """w-stacking.cu:466-469: grid_w = (int)(ww / dw), dw = 1/Nw (init.c:12):
    FP64 division, truncation toward zero."""
    dw = 1.0 / nw
    return np.trunc(np.asarray(ww, dtype=np.float64) / dw).astype(np.int64)


def sector0_rows(vv, nmeasures_file, nx, ny, w_support):
    out = np.zeros(max(int(nmeasures_file), 1), dtype=np.uint64)
    n = lib().oracle_sector0_rows(_c(vv, np.float64), nmeasures_file, nx, ny, w_support, out)
    return out[:n]


def resolution_of(meta) -> float:
    """gridding_cpu.c:78: 1 / max(|uvmin|, |uvmax|)."""
    return 1.0 / max(abs(meta["uvmin"]), abs(meta["uvmax"]))


def pack(obs, rows):
    npol, nchan = obs.meta["polarisations"], obs.meta["freq_per_chan"]
    r = rows.astype(np.int64)
    w = obs.weights.reshape(-1, npol)[r].reshape(-1)
    vr = obs.vis_re.reshape(-1, nchan * npol)[r].reshape(-1)
    vi = obs.vis_im.reshape(-1, nchan * npol)[r].reshape(-1)
    return obs.uu[r], obs.vv[r], obs.ww[r], w, vr, vi


def image(obs, nx, ny, nw, kernel, w_support, phase_on=True, threads=0, return_grid=False,
          fft_workers=None):
    """The whole one-rank pipeline: init.c:335-340 row drop, sector-0 packing,
    wstack, per-plane FFT, phase_correction.  Inputs are the rows of the file
    (``obs`` holds ``Nmeasures`` rows as written by the binMS creator)."""
    rows = sector0_rows(obs.vv, obs.meta["Nmeasures"], nx, ny, w_support)
    uu, vv, ww, w, vr, vi = pack(obs, rows)
    dx, dw = 1.0 / nx, 1.0 / nw                                  # init.c:11-12
    grid, dropped = wstack(kernel, nw, obs.meta["freq_per_chan"], obs.meta["polarisations"], uu,
                           vv, ww, vr, vi, w, dx, dw, w_support, nx, ny, threads=threads)
    gridss = fft_planes(grid, nw, nx, ny, workers=fft_workers)
    img_re, img_im = phase_correction(gridss, nx, ny, nw, resolution_of(obs.meta),
                                      obs.meta["wmin"], obs.meta["wmax"], phase_on, threads)
    out = dict(image_re=img_re, image_im=img_im, rows=len(rows), dropped=dropped)
    if return_grid:
        out["grid"] = grid
        out["gridss"] = gridss
    return out


def image_chunked(obs, nx, ny, nw, kernel, w_support, phase_on=True, threads=0,
                  fft_workers=None, progress=None):
    """The one-rank pipeline of ``image`` one w-plane at a time, with 64-bit
    indices throughout, for cubes too large to hold (8192^2 x 64 FP64 is 68.7 GB)
    and past the reference's 32-bit cube indices (w-stacking.cu:168,
    phase_correction.cu:198).  Per plane iw: the packed rows whose plane is iw by
    the reference's expression (``plane_of``), in their packing order, are
    gridded with Nw' = 1 and w' = 0 (w enters wstack only through grid_w,
    w-stacking.cu:466-469, so the plane's cells receive the same additions in
    the same order), the plane is transformed, and phase_correction over that
    plane alone (global iw, the whole cube's dw and dwnorm) accumulates into the
    image.  Single-threaded, the image has the bits of ``image``."""
    rows = sector0_rows(obs.vv, obs.meta["Nmeasures"], nx, ny, w_support)
    uu, vv, ww, w, vr, vi = pack(obs, rows)
    nchan, npol = obs.meta["freq_per_chan"], obs.meta["polarisations"]
    nv = nchan * npol
    dx, dw = 1.0 / nx, 1.0 / nw
    gw = plane_of(ww, nw)
    order = np.argsort(gw, kind="stable")
    bounds = np.searchsorted(gw[order], np.arange(nw + 1))
    dropped = int(len(gw) - (bounds[nw] - bounds[0]))      # grid_w outside [0, Nw)
    w2, vr2, vi2 = w.reshape(-1, npol), vr.reshape(-1, nv), vi.reshape(-1, nv)
    res = resolution_of(obs.meta)
    img_re, img_im = np.zeros(nx * ny), np.zeros(nx * ny)
    for iw in range(nw):
        sel = order[bounds[iw]:bounds[iw + 1]]
        plane = np.zeros(2 * nx * ny)
        if len(sel):
            _, d = wstack(kernel, 1, nchan, npol, uu[sel], vv[sel], np.zeros(len(sel)),
                          vr2[sel].ravel(), vi2[sel].ravel(), w2[sel].ravel(), dx, dw, w_support,
                          nx, ny, grid=plane, threads=threads)
            dropped += d
        gss = fft_planes(plane, 1, nx, ny, workers=fft_workers)
        del plane
        phase_correction_planes(gss, nx, ny, nw, iw, 1, res, obs.meta["wmin"], obs.meta["wmax"],
                                img_re, img_im, phase_on, threads)
        if progress:
            progress(iw)
    return dict(image_re=img_re, image_im=img_im, rows=len(rows), dropped=dropped)


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))


def ref_sector0_rows(vv, nmeasures_read, nx, ny, w_support):
    """The reference's own gridding.c:139-197 initialize_array (oracle/_ref/
    libref_rows.so) for one rank, then gridding_cpu.c:118's reverse packing
    order.  ``nmeasures_read`` is the row count after init.c:337-339."""
    path = os.path.join(HERE, "_ref", "libref_rows.so")
    if not os.path.exists(path):
        raise RuntimeError(f"reference build missing: {path} (run `make -C oracle ref`)")
    L = C.CDLL(path, mode=C.RTLD_LOCAL)
    vv = np.ascontiguousarray(vv, dtype=np.float64)

    class FileData(C.Structure):  # allvars.h:150-158
        _fields_ = [("uu", C.c_void_p), ("vv", C.c_void_p), ("ww", C.c_void_p),
                    ("weights", C.c_void_p), ("visreal", C.c_void_p), ("visimg", C.c_void_p)]
    data = FileData.in_dll(L, "data")
    data.vv = vv.ctypes.data
    C.c_uint.in_dll(L, "metaData").value = int(nmeasures_read)  # meta.Nmeasures is the first field
    C.c_uint.in_dll(L, "nsectors").value = 1                      # init.c:20 with one rank
    C.c_int.in_dll(L, "yaxis").value = ny                          # init.c:22
    dx = 1.0 / nx                                                   # init.c:11
    C.c_double.in_dll(L, "dx").value = dx
    C.c_double.in_dll(L, "w_supporth").value = (double_half := float((w_support - 1) // 2)) * dx
    L.initialize_array.argtypes = []
    L.initialize_array.restype = None
    L.initialize_array()
    histo = C.POINTER(C.c_uint).in_dll(L, "histo_send")
    sectors = C.POINTER(C.POINTER(C.c_uint)).in_dll(L, "sectorarray")
    n = histo[0]
    rows = np.array([sectors[0][i] for i in range(n)], dtype=np.uint64)
    del double_half
    return rows[::-1].copy()


def normalize_uvw(uu, vv, ww):
    """gridding.c:21-83 (NORMALIZE_UVW) restated: normalised copies of u, v, w
    and the extrema (min u, v, w, max u, v, w, maxg)."""
    u, v, w = (np.array(x, dtype=np.float64, copy=True) for x in (uu, vv, ww))
    ext = np.zeros(7)
    lib().oracle_normalize_uvw(len(u), u, v, w, ext)
    return u, v, w, ext


def ref_normalize_uvw(uu, vv, ww, nx=64, ny=64, w_support=7):
    """The reference's own gridding() built with NORMALIZE_UVW (oracle/_ref/
    libref_norm.so), one rank, one thread: the rows it normalises in place
    (the sector gridding it calls afterwards is stubbed out)."""
    path = os.path.join(HERE, "_ref", "libref_norm.so")
    if not os.path.exists(path):
        raise RuntimeError(f"reference build missing: {path} (run `make -C oracle ref`)")
    L = C.CDLL(path, mode=C.RTLD_LOCAL)
    u, v, w = (np.array(x, dtype=np.float64, copy=True) for x in (uu, vv, ww))

    class FileData(C.Structure):  # allvars.h:150-158
        _fields_ = [("uu", C.c_void_p), ("vv", C.c_void_p), ("ww", C.c_void_p),
                    ("weights", C.c_void_p), ("visreal", C.c_void_p), ("visimg", C.c_void_p)]
    data = FileData.in_dll(L, "data")
    data.uu, data.vv, data.ww = u.ctypes.data, v.ctypes.data, w.ctypes.data
    C.c_int.in_dll(L, "param").value = 1                  # param.num_threads (first field)
    C.c_uint.in_dll(L, "metaData").value = len(u)         # meta.Nmeasures (first field)
    C.c_uint.in_dll(L, "nsectors").value = 1
    C.c_int.in_dll(L, "yaxis").value = ny
    dx = 1.0 / nx
    C.c_double.in_dll(L, "dx").value = dx
    C.c_double.in_dll(L, "w_supporth").value = float((w_support - 1) // 2) * dx
    L.gridding.argtypes = []
    L.gridding.restype = None
    L.gridding()
    return u, v, w
