"""The host driver rick_imager end to end: paramfile + binMS in, the reference's
image files out (fft_real.bin / fft_img.bin, and the FITS images of
fourier_transform.c:227-279 when asked), against the oracle."""
import os
import subprocess

import numpy as np
import pytest

import oracle as O
from rick_b200 import binms, synth
from _util import TOL_FP64, rel_l2

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _read_fits(path):
    raw = open(path, "rb").read()
    cards = {}
    for i in range(0, 2880, 80):
        card = raw[i:i + 80].decode()
        if card.startswith("END"):
            break
        key, _, val = card.partition("=")
        cards[key.strip()] = val.strip()
    assert len(raw) % 2880 == 0
    nx, ny = int(cards["NAXIS1"]), int(cards["NAXIS2"])
    assert cards["SIMPLE"] == "T" and int(cards["BITPIX"]) == -64 and int(cards["NAXIS"]) == 2
    return np.frombuffer(raw[2880:2880 + 8 * nx * ny], dtype=">f8").astype(np.float64), nx, ny


def test_imager_writes_reference_outputs(tmp_path):
    obs = synth.make_observation("c1", seed=23, time_fraction=0.2)
    data = binms.write_binms(obs, str(tmp_path / "c1.binMS"))
    par = binms.write_paramfile(str(tmp_path / "paramfile.txt"), [data], 512, 8, 7,
                                extra={"kernel": "gauss", "fits": 1})
    r = subprocess.run([os.path.join(ROOT, "rick_b200", "rick_imager"), par], cwd=tmp_path,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    re = np.fromfile(tmp_path / "0fft_real.bin", dtype=np.float64)
    im = np.fromfile(tmp_path / "0fft_img.bin", dtype=np.float64)
    ref = O.image(obs, 512, 512, 8, "gauss", 7)
    assert rel_l2(re, ref["image_re"]) < TOL_FP64 and rel_l2(im, ref["image_im"]) < TOL_FP64
    fre, nx, ny = _read_fits(tmp_path / "parallel_real.fits")
    fim, _, _ = _read_fits(tmp_path / "parallel_img.fits")
    assert (nx, ny) == (512, 512)
    assert np.array_equal(fre, re) and np.array_equal(fim, im)
