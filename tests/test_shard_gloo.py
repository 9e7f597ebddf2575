"""w-plane sharding across ranks, on the CPU: world-size-2 gloo process groups.

Each rank images the rows of its plane range with the oracle (the reference's
own arithmetic restated in C) into a cube whose other planes stay empty, the
ranks all-reduce their images, and the sum equals the unsharded image.  This
covers the partition rules and the exchange step of rick_b200.shard; the CUDA
side of a shard (rick_plan_desc.w_first / w_count) is checked against the same
identity in test_gpu_shard.py."""
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
