"""The C ABI boundary and host-side logic, without a GPU: the library loads,
exports every symbol include/rick_b200.h declares, and reports errors as
statuses; binMS / paramfile I/O; the host driver's argument handling."""
import os
import re
import subprocess

import numpy as np
import pytest

import rick_b200 as R
from rick_b200 import binms, synth

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "rick_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"\b([a-z_][a-z0-9_]*)\s*\(", src)
    keywords = {"if", "sizeof", "return"}
    return sorted({n for n in names if n not in keywords})


def test_header_declares_the_dropins():
    names = declared_functions()
    for n in ("wstack", "phase_correction", "rick_fft_planes", "rick_plan_create",
              "rick_plan_image", "rick_plan_image_host"):
        assert n in names


def test_library_exports_every_declared_symbol():
    lib = R.lib()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_kernel_names_listed():
    names = R.kernel_names()
    assert "k_grid_tiles" in names and "k_phase_sum" in names and "k_bin_scatter" in names


def test_status_strings():
    assert R.status_string(0) == "ok"
    assert R.status_string(255) == "no accelerators found"
    assert R.status_string(21) == "HBM budget exceeded"


def test_invalid_plan_description_is_rejected_before_any_device_call():
    with pytest.raises(R.RickError) as e:
        R.Plan(R.Geometry(64, 64, 4, w_support=8), 10, 1, 1)   # even support
    assert e.value.status == R.ERR_INVALID_ARG
    with pytest.raises(R.RickError) as e:
        R.Plan(R.Geometry(0, 64, 4), 10, 1, 1)
    assert e.value.status == R.ERR_INVALID_ARG


def test_footprint_accounts_for_cube():
    g = R.Geometry(4096, 4096, 32, 7, "kaiser_bessel", "fp64")
    b64 = R.Plan.footprint(g, 5_096_600, 64, 4)
    g.precision = "mixed"
    b32 = R.Plan.footprint(g, 5_096_600, 64, 4)
    assert b64 > 2 * 32 * 4096 * 4096 * 8 and b32 < b64


@pytest.mark.skipif(__import__("torch").cuda.is_available(), reason="needs a machine without GPU")
def test_no_gpu_reports_status_255():
    with pytest.raises(R.RickError) as e:
        R.Plan(R.Geometry(64, 64, 4), 10, 1, 1)
    assert e.value.status == R.ERR_NO_ACCELERATORS_FOUND
    grid = np.zeros(2 * 4 * 16 * 16)
    with pytest.raises(R.RickError) as e:
        R.wstack(4, 1, 1, 1, [0.5], [0.5], [0.5], [1.0], [0.0], [1.0], 1 / 16, 0.25, 7, 16, 16,
                 grid)
    assert e.value.status == R.ERR_NO_ACCELERATORS_FOUND


def test_binms_roundtrip(tmp_path):
    obs = synth.make_observation("c1", seed=3, time_fraction=0.02)
    d = binms.write_binms(obs, str(tmp_path / "c1.binMS"))
    meta, arr = binms.read_binms(d)
    n = obs.meta["Nmeasures"] - 1000
    assert meta["Nmeasures"] == obs.meta["Nmeasures"] and meta["polarisations"] == 2
    assert meta["uvmax"] == obs.meta["uvmax"] and meta["wmin"] == obs.meta["wmin"]
    assert np.array_equal(arr["uu"], obs.uu[:n]) and np.array_equal(arr["vis_im"],
                                                                    obs.vis_im[: n * 16])


def test_binms_truncated_file_is_an_error(tmp_path):
    obs = synth.make_observation("c1", seed=3, time_fraction=0.02)
    d = binms.write_binms(obs, str(tmp_path / "t.binMS"))
    with open(os.path.join(d, "visibilities_real.bin"), "r+b") as f:
        f.truncate(100)
    with pytest.raises(ValueError):
        binms.read_binms(d)


def test_paramfile_roundtrip(tmp_path):
    p = binms.write_paramfile(str(tmp_path / "paramfile.txt"), ["/data/a.binMS"], 512, 8, 7,
                              extra={"kernel": "gauss"})
    kv = binms.read_paramfile(p)
    assert kv["grid_size_x"] == "512" and kv["num_w_planes"] == "8" and kv["kernel"] == "gauss"
    assert kv["Datapath1"] == "/data/a.binMS/"


def test_synthetic_config_shapes():
    """Row counts of the imaging workloads: baselines x time steps."""
    cfg = synth.CONFIGS["c1"]
    enu = synth.antenna_enu(cfg, np.random.default_rng(0))
    uvw, nt, nbl = synth.uvw_tracks(cfg, enu)
    assert (nbl, nt, uvw.shape[0]) == (780, 360, 280_800)
    cfg = synth.CONFIGS["c2"]
    uvw, nt, nbl = synth.uvw_tracks(cfg, synth.antenna_enu(cfg, np.random.default_rng(0)))
    assert (nbl, nt) == (1770, 2880)


def test_driver_rejects_missing_paramfile(tmp_path):
    exe = os.path.join(ROOT, "rick_b200", "rick_imager")
    r = subprocess.run([exe, str(tmp_path / "nope.txt")], capture_output=True, text=True)
    assert r.returncode == 2 and "paramfile" in r.stdout


def test_driver_requires_argument():
    exe = os.path.join(ROOT, "rick_b200", "rick_imager")
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 1


def test_noalloc_rejects_sizes_that_would_wrap_its_layout():
    """rick_wstack_noalloc refuses a row count whose record block would not fit
    the static scratch (2^60 rows would wrap a 64-bit byte count) and a
    geometry with 2^32 or more bins, before any device call; the capacity of
    such a geometry is 0 rows."""
    import ctypes as C
    L = R.lib()
    f = L.rick_wstack_noalloc
    f.argtypes = ([C.c_int, C.c_uint64, C.c_uint32, C.c_uint32] + [C.c_void_p] * 6 +
                  [C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p,
                   C.c_void_p])
    f.restype = C.c_int
    buf = np.zeros(16)
    p = buf.ctypes.data            # never dereferenced: the sizes are refused first
    st = f(8, 1 << 60, 8, 2, p, p, p, p, p, p, 1 / 512, 1 / 8, 7, R.KERNELS["kaiser_bessel"],
           512, 512, p, None)
    assert st == R.ERR_INVALID_ARG and "exceed" in R.last_error()
    st = f(1 << 30, 10, 8, 2, p, p, p, p, p, p, 1 / 65536, 1 / (1 << 30), 7,
           R.KERNELS["kaiser_bessel"], 1 << 16, 1 << 16, p, None)
    assert st == R.ERR_INVALID_ARG
    cap = L.rick_wstack_noalloc_capacity
    cap.argtypes = [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_uint64)]
    cap.restype = C.c_int
    rows = C.c_uint64(7)
    assert cap(1 << 30, 1 << 30, 1 << 30, C.byref(rows)) == R.OK and rows.value == 0
