"""CUDA side of w-plane sharding: the images of a job's plane shards
(rick_plan_desc.w_first / w_count), imaged one after the other on one GPU, add
up to the job's image; rows split exactly between the shards."""
import numpy as np
import pytest

import rick_b200 as R
from rick_b200 import shard
from _util import TOL_FP64, TOL_MIXED, gpu_rows, rel_l2
from test_shard_gloo import GEOM, _partial, _rows

pytestmark = pytest.mark.gpu


def _image(rows_dev, n, nx, ny, nw, precision, planes=None, sel=R.ROWS_ALL):
    import torch
    g = GEOM
    geom = R.Geometry(nx, ny, nw, g["sup"], g["kernel"], precision)
    with R.Plan(geom, n, g["nchan"], g["npol"], device=0, planes=planes) as plan:
        img = torch.empty(2 * nx * ny, dtype=torch.float64, device="cuda")
        plan.image(n, rows_dev, g["res"], g["wmin"], g["wmax"], img[: nx * ny], img[nx * ny:], sel)
        torch.cuda.synchronize()
        return img.cpu().numpy(), plan.stats()


@pytest.mark.parametrize("nx,precision", [(128, "fp64"), (128, "mixed"), (96, "fp64")])
def test_shards_add_up_to_the_image(nx, precision):
    g = GEOM
    rows = _rows()
    n = len(rows[0])
    dev = gpu_rows(*rows)
    whole, st = _image(dev, n, nx, nx, g["nw"], precision)
    counts = np.bincount(shard.plane_of_rows(rows[2], g["nw"]), minlength=g["nw"])
    for ranges in ([shard.plane_range(r, 3, g["nw"]) for r in range(3)],
                   shard.balanced_ranges(counts, 2)):
        total = np.zeros_like(whole)
        gridded = 0
        for first, count in ranges:
            part, sst = _image(dev, n, nx, nx, g["nw"], precision, planes=(first, count))
            total += part
            gridded += sst["rows_gridded"]
            assert sst["rows_gridded"] + sst["rows_other_shard"] + sst["rows_dropped"] == n
        assert gridded == st["rows_gridded"]
        tol = TOL_FP64 if precision == "fp64" else TOL_MIXED
        assert rel_l2(total, whole) < tol
    if nx == 128 and precision == "fp64":
        assert rel_l2(whole, _partial(rows, 0, g["nw"])) < TOL_FP64


def test_shard_outside_the_cube_is_rejected():
    g = GEOM
    geom = R.Geometry(128, 128, g["nw"], g["sup"], g["kernel"], "fp64")
    with pytest.raises(R.RickError) as e:
        R.Plan(geom, 10, 1, 1, device=0, planes=(4, 3))
    assert e.value.status == R.ERR_INVALID_ARG
