"""w-plane sharding of one imaging job over several GPUs (one process per GPU).

The reference splits the grid into v-slabs, one per MPI rank, grids each slab,
and reduces the slabs' cubes before a distributed FFT (gridding.c:139-197,
gridding_nccl.cu:268, cuda_fft.cu).  Here the w-stacked cube is split by
planes instead: every plane's gridding, 2-D FFT and w-correction are
independent, so rank r images the planes of its contiguous range
(rick_plan_desc.w_first / w_count) from all rows -- rows of other planes are
skipped in the binning pass -- and the ranks' partial images add up to the
image.  The only exchange is one sum of the Nx*Ny complex image (FP64): an
all-reduce over NCCL (NVLink/NVSwitch) on GPUs, over gloo in the CPU tests.
"""
from __future__ import annotations

from typing import Optional, Sequence

import numpy as np


def plane_range(rank: int, world: int, nw: int) -> tuple[int, int]:
    """(w_first, w_count) of rank ``rank``: contiguous, the first nw % world
    ranks one plane more.  A rank may get no plane when world > nw."""
    if not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world {world}")
    base, extra = divmod(nw, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def balanced_ranges(rows_per_plane: Sequence[int], world: int) -> list[tuple[int, int]]:
    """Contiguous plane ranges with about equal row counts (rows cluster in a
    few planes when |w| is small): greedy cuts at the running-sum quantiles,
    every rank keeping at least one plane while planes remain."""
    counts = np.asarray(rows_per_plane, dtype=np.float64)
    nw = len(counts)
    if world >= nw:
        return [plane_range(r, world, nw) for r in range(world)]
    cum = np.concatenate([[0.0], np.cumsum(counts)])
    total = cum[-1]
    cuts = [0]
    for r in range(1, world):
        target = total * r / world
        c = int(np.searchsorted(cum, target, side="left"))
        c = max(c, cuts[-1] + 1)                 # at least one plane per rank
        c = min(c, nw - (world - r))             # leave a plane for every later rank
        cuts.append(c)
    cuts.append(nw)
    return [(cuts[r], cuts[r + 1] - cuts[r]) for r in range(world)]


def plane_of_rows(ww, nw: int) -> np.ndarray:
    """w-stacking.cu:145-147: grid_w = (int)(ww / dw), dw = 1 / nw (init.c:12)."""
    dw = 1.0 / nw
    return (np.asarray(ww, dtype=np.float64) / dw).astype(np.int64)


class ShardedImager:
    """One rank's share of a w-plane-sharded imaging job.

    ``image`` runs this rank's planes through a plan (device-resident rows) and
    all-reduces the image over ``group`` (torch.distributed; NCCL for CUDA
    tensors), so every rank ends with the whole image.  ``plan_factory``
    builds the rank's plan (default ``rick_b200.Plan``; called as
    ``plan_factory(geom, max_rows, freq_per_chan, polarizations, device=...,
    planes=(w_first, w_count))``)."""

    def __init__(self, geom, max_rows: int, freq_per_chan: int, polarizations: int,
                 device: int = 0, group=None, ranges: Optional[list] = None,
                 plan_factory=None):
        import torch.distributed as dist
        import rick_b200 as R

        self.group = group
        rank = dist.get_rank(group) if dist.is_initialized() else 0
        world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.planes = ranges[rank] if ranges is not None else plane_range(rank, world,
                                                                          geom.num_w_planes)
        self.world = world
        self.plan = None
        if self.planes[1] > 0:
            factory = plan_factory if plan_factory is not None else R.Plan
            self.plan = factory(geom, max_rows, freq_per_chan, polarizations, device=device,
                                planes=self.planes)
        self.geom = geom

    def image(self, nrows, rows, resolution, wmin, wmax, image, selection=None, stream=None):
        """``image``: one CUDA tensor of 2*Nx*Ny float64 (real plane, then imaginary)."""
        import torch.distributed as dist
        import rick_b200 as R

        n = self.geom.grid_size_x * self.geom.grid_size_y
        sel = R.ROWS_SECTOR0 if selection is None else selection
        if self.plan is not None:
            self.plan.image(nrows, rows, resolution, wmin, wmax, image[:n], image[n:], sel, stream)
        else:
            image.zero_()
        if self.world > 1:
            dist.all_reduce(image, op=dist.ReduceOp.SUM, group=self.group)
        return image

    def stats(self) -> dict:
        return self.plan.stats() if self.plan is not None else {}

    def close(self):
        if self.plan is not None:
            self.plan.close()
            self.plan = None
