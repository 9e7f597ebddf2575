"""binMS datasets and RICK parameter files.

A binMS directory holds the files scripts/create_binMS.py:210-245 writes:
``ucoord.bin``, ``vcoord.bin``, ``wcoord.bin`` (float64 per row, normalised),
``weights.bin`` (float32 [row][pol]), ``visibilities_real.bin`` and
``visibilities_img.bin`` (float32 [row][chan][pol]) and ``meta.txt`` with the
lines Nmeasures, Nvis, freq_per_chan, polarisations, Ntimes, dt, thours,
baselines, uvmin, uvmax, wmin, wmax (read in that order by init.c:307-318).

The parameter file is the whitespace key/value format of paramfile.txt, parsed
like init.c:129-272 (first token key, second token value, unknown keys ignored).
"""
from __future__ import annotations

import os

import numpy as np

META_KEYS = ["Nmeasures", "Nvis", "freq_per_chan", "polarisations", "Ntimes", "dt", "thours",
             "baselines", "uvmin", "uvmax", "wmin", "wmax"]
META_INT = {"Nmeasures", "Nvis", "freq_per_chan", "polarisations", "Ntimes", "baselines"}

DEFAULT_FILES = dict(ufile="ucoord.bin", vfile="vcoord.bin", wfile="wcoord.bin",
                     weightsfile="weights.bin", visrealfile="visibilities_real.bin",
                     visimgfile="visibilities_img.bin", metafile="meta.txt")


def write_binms(obs, path: str) -> str:
    """Write an Observation (rick_b200.synth) as a binMS directory."""
    os.makedirs(path, exist_ok=True)
    np.asarray(obs.uu, dtype=np.float64).tofile(os.path.join(path, DEFAULT_FILES["ufile"]))
    np.asarray(obs.vv, dtype=np.float64).tofile(os.path.join(path, DEFAULT_FILES["vfile"]))
    np.asarray(obs.ww, dtype=np.float64).tofile(os.path.join(path, DEFAULT_FILES["wfile"]))
    np.asarray(obs.weights, dtype=np.float32).tofile(os.path.join(path, DEFAULT_FILES["weightsfile"]))
    np.asarray(obs.vis_re, dtype=np.float32).tofile(os.path.join(path, DEFAULT_FILES["visrealfile"]))
    np.asarray(obs.vis_im, dtype=np.float32).tofile(os.path.join(path, DEFAULT_FILES["visimgfile"]))
    with open(os.path.join(path, DEFAULT_FILES["metafile"]), "w") as f:
        for k in META_KEYS:
            v = obs.meta[k]
            f.write(f"{int(v)}\n" if k in META_INT else f"{float(v)!r}\n")
        # create_binMS.py:239-244 appends the weight array shape; init.c ignores it
        f.write(f"{obs.meta['Nmeasures']}\n{obs.meta['polarisations']}\n1.0\n")
    return path


def read_meta(path: str) -> dict:
    with open(os.path.join(path, DEFAULT_FILES["metafile"])) as f:
        tok = f.read().split()
    if len(tok) < len(META_KEYS):
        raise ValueError(f"{path}/meta.txt: expected {len(META_KEYS)} values, got {len(tok)}")
    meta = {}
    for k, t in zip(META_KEYS, tok):
        meta[k] = int(float(t)) if k in META_INT else float(t)
    return meta


def read_binms(path: str, drop_last: int = 1000) -> tuple[dict, dict]:
    """Read the rows init.c:413-503 reads: all but the last ``drop_last`` rows
    (init.c:337-339).  Returns (meta, arrays)."""
    meta = read_meta(path)
    n = max(meta["Nmeasures"] - drop_last, 0)
    npol, nchan = meta["polarisations"], meta["freq_per_chan"]

    def rd(name, dt, count):
        fn = os.path.join(path, DEFAULT_FILES[name])
        a = np.fromfile(fn, dtype=dt, count=count)
        if a.size != count:
            raise ValueError(f"{fn}: truncated ({a.size} of {count} values)")
        return a

    arrays = dict(uu=rd("ufile", np.float64, n), vv=rd("vfile", np.float64, n),
                  ww=rd("wfile", np.float64, n), weights=rd("weightsfile", np.float32, n * npol),
                  vis_re=rd("visrealfile", np.float32, n * nchan * npol),
                  vis_im=rd("visimgfile", np.float32, n * nchan * npol))
    return meta, arrays


def write_paramfile(path: str, datapaths: list[str], grid: int, w_planes: int, w_support: int,
                    num_threads: int = 0, extra: dict | None = None) -> str:
    """paramfile.txt layout (keys of init.c:140-272)."""
    lines = [f"ndatasets {len(datapaths)}"]
    for i, d in enumerate(datapaths, 1):
        lines.append(f"Datapath{i} {d.rstrip('/')}/")
    lines += [f"num_threads {num_threads}", f"w_support {w_support}", "reduce_method 0",
              f"grid_size_x {grid}", f"grid_size_y {grid}", f"num_w_planes {w_planes}"]
    lines += [f"{k} {v}" for k, v in DEFAULT_FILES.items()]
    lines += ["outfile grid.txt", "outfile1 coords.txt", "outfile2 grid_real.bin",
              "outfile3 grid_img.bin", "fftfile fft.txt", "fftfile2 fft_real.bin",
              "fftfile3 fft_img.bin", "logfile run.log", "extension .txt",
              "timingfile timings.dat"]
    for k, v in (extra or {}).items():
        lines.append(f"{k} {v}")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
    return path


def read_paramfile(path: str) -> dict:
    """Key/value pairs as init.c:140-272 scans them (pairs of tokens)."""
    with open(path) as f:
        tok = f.read().split()
    return {tok[i]: tok[i + 1] for i in range(0, len(tok) - 1, 2)}
