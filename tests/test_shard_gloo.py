"""w-plane sharding across ranks, on the CPU: world-size-2 gloo process groups.

Each rank images the rows of its plane range with the oracle (the reference's
own arithmetic restated in C) into a cube whose other planes stay empty, the
ranks all-reduce their images, and the sum equals the unsharded image.  This
covers the partition rules and the exchange step of rick_b200.shard; the CUDA
side of a shard (rick_plan_desc.w_first / w_count) is checked against the same
identity in test_gpu_shard.py.  ``ShardedImager`` itself (its plane choice,
the zero image of a rank without planes, and its all-reduce) runs over gloo
with an oracle-backed stand-in for the CUDA plan."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import oracle as O
from rick_b200 import shard


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rows(seed=11, n=3000, nchan=2, npol=2):
    rng = np.random.default_rng(seed)
    uu = np.clip(0.5 + 0.15 * rng.standard_normal(n), 0, 1)
    vv = np.clip(0.5 + 0.15 * rng.standard_normal(n), 0, 0.999)
    ww = rng.random(n) ** 2 * 0.999          # rows crowd the low planes
    wt = rng.uniform(0.5, 1.5, n * npol).astype(np.float32)
    vr = rng.standard_normal(n * nchan * npol).astype(np.float32)
    vi = rng.standard_normal(n * nchan * npol).astype(np.float32)
    return uu, vv, ww, wt, vr, vi


GEOM = dict(nx=128, ny=128, nw=6, kernel="kaiser_bessel", sup=7, nchan=2, npol=2, res=1 / 300.0,
            wmin=-150.0, wmax=120.0)


def _partial(rows, first, count):
    g = GEOM
    uu, vv, ww, wt, vr, vi = rows
    plane = shard.plane_of_rows(ww, g["nw"])
    keep = np.nonzero((plane >= first) & (plane < first + count))[0]
    nv = g["nchan"] * g["npol"]
    grid, _ = O.wstack(g["kernel"], g["nw"], g["nchan"], g["npol"], uu[keep], vv[keep], ww[keep],
                       vr.reshape(-1, nv)[keep].ravel(), vi.reshape(-1, nv)[keep].ravel(),
                       wt.reshape(-1, g["npol"])[keep].ravel(), 1 / g["nx"], 1 / g["nw"], g["sup"],
                       g["nx"], g["ny"])
    gss = O.fft_planes(grid, g["nw"], g["nx"], g["ny"])
    re, im = O.phase_correction(gss, g["nx"], g["ny"], g["nw"], g["res"], g["wmin"], g["wmax"], True)
    return np.concatenate([re, im])


def _rank_main(rank, world, port, balanced, out_dir):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    rows = _rows()
    if balanced:
        counts = np.bincount(shard.plane_of_rows(rows[2], GEOM["nw"]), minlength=GEOM["nw"])
        first, count = shard.balanced_ranges(counts, world)[rank]
    else:
        first, count = shard.plane_range(rank, world, GEOM["nw"])
    img = torch.from_numpy(_partial(rows, first, count))
    dist.all_reduce(img, op=dist.ReduceOp.SUM)
    np.save(os.path.join(out_dir, f"img{rank}.npy"), img.numpy())
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("balanced", [False, True])
def test_two_rank_plane_shards_sum_to_image(tmp_path, balanced):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), balanced, str(tmp_path)),
                       nprocs=world, start_method="spawn", join=True)
    whole = _partial(_rows(), 0, GEOM["nw"])
    for r in range(world):
        got = np.load(tmp_path / f"img{r}.npy")
        assert O.rel_l2(got, whole) < 1e-12


def test_plane_ranges_partition_the_cube():
    for nw in (1, 5, 8, 32, 64):
        for world in (1, 2, 3, 4, 8):
            ranges = [shard.plane_range(r, world, nw) for r in range(world)]
            assert sum(c for _, c in ranges) == nw
            assert [f for f, _ in ranges] == list(np.cumsum([0] + [c for _, c in ranges])[:-1])
    counts = [500, 300, 100, 50, 30, 10, 5, 5]
    b = shard.balanced_ranges(counts, 3)
    assert sum(c for _, c in b) == len(counts) and all(c >= 1 for _, c in b)
    assert b[0] == (0, 1)                      # the heavy first plane alone
    rows = [sum(counts[f:f + c]) for f, c in b]
    assert max(rows) <= 500


class _OraclePlan:
    """CPU stand-in for rick_b200.Plan with a w-plane shard: the oracle images
    the rows of planes w_first .. w_first+w_count-1 (whole-cube dw, global
    plane index), as rick_plan_image does for a shard plan."""

    def __init__(self, geom, max_rows, nchan, npol, device=0, planes=(0, 0)):
        self.first, self.count = planes

    def image(self, nrows, rows, res, wmin, wmax, img_re, img_im, sel, stream=None):
        import torch
        img = _partial(tuple(np.asarray(r) for r in rows), self.first, self.count)
        n = GEOM["nx"] * GEOM["ny"]
        img_re.copy_(torch.from_numpy(img[:n]))
        img_im.copy_(torch.from_numpy(img[n:]))

    def close(self):
        pass


def _imager_rank(rank, world, port, nw_ranges, out_dir):
    import torch
    import torch.distributed as dist
    import rick_b200 as R
    from rick_b200.shard import ShardedImager
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    g = GEOM
    geom = R.Geometry(g["nx"], g["ny"], g["nw"], g["sup"], g["kernel"], "fp64")
    rows = _rows()
    imager = ShardedImager(geom, len(rows[0]), g["nchan"], g["npol"], ranges=nw_ranges,
                           plan_factory=_OraclePlan)
    img = torch.full((2 * g["nx"] * g["ny"],), float("nan"), dtype=torch.float64)
    imager.image(len(rows[0]), rows, g["res"], g["wmin"], g["wmax"], img)
    np.save(os.path.join(out_dir, f"imager{rank}.npy"), img.numpy())
    np.save(os.path.join(out_dir, f"planes{rank}.npy"), np.array(imager.planes))
    imager.close()
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("ranges", [None, [(0, 6), (6, 0)]])
def test_sharded_imager_reduces_over_gloo(tmp_path, ranges):
    """Two gloo ranks each build a ShardedImager (even split, or every plane on
    rank 0 and none on rank 1) and call its image(): both end with the whole
    image (<= 1e-12 against the unsharded oracle image)."""
    world = 2
    mp.start_processes(_imager_rank, args=(world, _free_port(), ranges, str(tmp_path)),
                       nprocs=world, start_method="spawn", join=True)
    whole = _partial(_rows(), 0, GEOM["nw"])
    want = [shard.plane_range(r, world, GEOM["nw"]) for r in range(world)] if ranges is None \
        else ranges
    for r in range(world):
        assert tuple(np.load(tmp_path / f"planes{r}.npy")) == tuple(want[r])
        got = np.load(tmp_path / f"imager{r}.npy")
        assert O.rel_l2(got, whole) < 1e-12
