"""Benchmark: imaged visibilities/s of the imaging hot path on B200.

Workload (one "step" = one imaging job: binning -> gridding -> per-plane inverse
FFT -> w-correction + plane sum, all rows): the LOFAR-like large single image,
60 stations log-radial to 40 km, 4 h at dec +50, 5 s integrations
(1770 baselines x 2880 steps; 5,096,600 rows after the 1000-row drop), 64
channels x 4 polarisations (1.305e9 visibilities), 200 log-normal point
sources + noise sigma 0.5, grid 4096^2 x 32 w-planes, Kaiser-Bessel support 7.
Synthetic, seeded, generated on the GPU (no dataset ships with the reference).

  value     imaged vis/s with the rows resident in HBM (FP64 plain form, the
            reference's arithmetic), CUDA events on the launching stream,
            max over ranks; inputs (10.6 GB) are larger than L2.
  e2e       the same through rick_plan_image_host (host buffers, pinned;
            H2D of the rows and D2H of the image inside the timed region).
  forms     plain FP64 and mixed (FP32 grid/FFT) side by side, with the mixed
            image's relative L2 error against the FP64 image.
  roofline  the dominant stage: algorithmic bytes / its CUDA-event time over
            the measured HBM copy bandwidth.
  cpu_baseline  the reference's own CPU wstack + phase_correction (compiled from
            its sources, oracle/_ref, OpenMP on all host cores) with scipy's
            FFT (FFTW is absent), on a bounded sample, extrapolated.

--impl reference prints the reference arm (the same CPU path, timed per step).
With N GPUs (torchrun) each rank images its own copy of the job (replicas,
weak scaling; the path needs no collective).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

FP64_NOMINAL_TFLOPS = 37.0   # B200 FP64 (non-tensor) nominal, for the column pass's compute bound
METRIC = "imaged vis/s (1xB200) FP32-mixed vs FP64 plain @<=1e-5 rel err; p50/p99 lat"
WORKLOAD = dict(name="c2", grid=4096, w_planes=32, kernel="kaiser_bessel", w_support=7)
WORKLOAD_TEXT = {
    "c1": "small plain FP64 image: 40-antenna disc, 1 h, 8 chan x 2 pol, 512^2 x 8 w-planes, "
          "Gaussian support 7",
    "c2": "LOFAR-like single image: 5,096,600 rows x 64 chan x 4 pol (1.305e9 vis), 4096^2 x 32 "
          "w-planes, Kaiser-Bessel support 7",
    "c3": "JVLA-like wide field: 27-antenna Y, 6 h, 16 chan x 2 pol, 8192^2 x 64 w-planes, "
          "high-precision Gaussian support 9",
}

# DRAM traffic per launch (dram__bytes_read.sum + dram__bytes_write.sum) that ncu
# measured for each stage's kernel on this workload at full size (FP64 form, one
# metric pass; profiles/traffic_c2.md has the command and the read/write split).
NCU_TRAFFIC = {"bin_count": 126_126_592, "bin_scatter": 10_851_913_216,
               "grid": 459_853_312, "fft": 2_083_898_112, "phase": 2_413_688_064}
# the kernel behind each plan stage on the sparse-aware path (FP64, 4096^2)
STAGE_KERNELS = {"bin_count": "k_bin_count", "bin_scatter": "k_bin_scatter<32,1>",
                 "cube_zero": "k_zero_split_tiles<double>", "grid": "k_grid_tiles<double,8>",
                 "fft": "k_fft_rows<double,12>", "phase": "k_fft_cols_image<double,12,1,1,1>"}


def fp64_gemm_tflops(dev) -> float:
    """FP64 throughput of this GPU as a library GEMM reaches it (cuBLAS through
    torch.matmul, 4096^3, best of 5 after a warm-up): the compute ceiling the
    FP64 column pass is compared with, next to the nominal figure."""
    import torch
    n = 4096
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    torch.matmul(a, b)
    best = float("inf")
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--time-fraction", type=float, default=1.0,
                    help="keep this leading fraction of the time steps (debug only)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--forms", default="fp64,mixed",
                    help="comma list of precision forms to time (fp64 first is the headline)")
    ap.add_argument("--grid", type=int, default=0, help="override the grid size (profiling cases)")
    ap.add_argument("--w-planes", type=int, default=0, help="override the w-planes (profiling)")
    ap.add_argument("--no-batched", action="store_true",
                    help="skip the batched-snapshot leg (256 small jobs, one graph)")
    ap.add_argument("--jobs", type=int, default=256, help="jobs of the batched-snapshot leg")
    ap.add_argument("--workload", default="c2", choices=["c1", "c2", "c3"],
                    help="imaging job of the headline line (c2: the metric's configuration)")
    ap.add_argument("--mode", default="replicas", choices=["replicas", "shard"],
                    help="N>1: independent jobs per GPU (weak scaling) or one job with its "
                         "w-planes split over the GPUs and the image all-reduced (strong)")
    ap.add_argument("--no-served", action="store_true", help="skip the served-stream leg")
    ap.add_argument("--served-requests", type=int, default=300)
    ap.add_argument("--served-rates", type=float, nargs="+", default=[250.0, 500.0, 1000.0, 0.0],
                    help="arrival rates (jobs/s) of the served-stream leg; 0 = all at once")
    ap.add_argument("--only-batched", action="store_true",
                    help="run only the batched-snapshot leg and print its line (profiling)")
    return ap.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 200 ms."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def algorithmic_bytes(n_rows, nvis, npol, records, nx, ny, nw, val_bytes, fft_rows=0):
    """Per-stage algorithmic bytes (the minimum each stage must move).

    With the sparse-aware FFT (fft_rows > 0: the (plane, row) pairs the gridder
    touched) the row pass reads those rows of the cube and writes them to the
    column-blocked buffer, and the column pass reads them back once and writes
    the FP64 image; the cube is not cleared (stage cube_zero only clears the
    row/tile masks and the split tiles)."""
    g = 2 * nw * nx * ny * val_bytes                 # the cube
    rec = 32 * records                                # binned row records
    out = {
        "bin_count": 24 * n_rows,                                   # u,v,w read once
        "bin_scatter": 8 * nvis + n_rows * (24 + 4 * npol) + rec,   # vis+uvw+weights in, records out
        "cube_zero": g,
        "grid": rec + g,                                            # records in, cube out
        "fft": 2 * g,                                               # one read + one write
        "phase": g + 16 * nx * ny,                                  # cube in, FP64 image out
    }
    if fft_rows:
        touched = fft_rows * nx * 2 * val_bytes
        out.update({"cube_zero": 0, "fft": 2 * touched, "phase": touched + 16 * nx * ny})
    return out


def run_ours(args):
    import torch
    import torch.distributed as dist

    import rick_b200 as R
    from rick_b200 import synth

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    cfg = synth.CONFIGS[args.workload]
    t0 = time.time()
    obs = synth.make_observation(cfg, seed=2024, device=str(dev),
                                 time_fraction=args.time_fraction)
    torch.cuda.synchronize()
    gen_s = time.time() - t0
    n = R.rows_read(obs.meta)
    nchan, npol = cfg.nchan, cfg.npol
    nv = nchan * npol
    rows = (obs.uu[:n].contiguous(), obs.vv[:n].contiguous(), obs.ww[:n].contiguous(),
            obs.weights[: n * npol].contiguous(), obs.vis_re[: n * nv].contiguous(),
            obs.vis_im[: n * nv].contiguous())
    nvis = n * nv
    res = R.resolution_of(obs.meta)
    wmin, wmax = obs.meta["wmin"], obs.meta["wmax"]
    nx = ny = args.grid or cfg.grid
    nw = args.w_planes or cfg.w_planes
    stream = torch.cuda.current_stream(dev)

    def barrier():
        if world > 1:
            dist.barrier()

    shard_mode = world > 1 and args.mode == "shard"

    def run_form(precision):
        geom = R.Geometry(nx, ny, nw, cfg.w_support, cfg.kernel, precision)
        img = torch.empty(2 * nx * ny, dtype=torch.float64, device=dev)
        if shard_mode:
            from rick_b200.shard import ShardedImager
            imager = ShardedImager(geom, n, nchan, npol, device=local)
            plan = imager.plan
            step = lambda: imager.image(n, rows, res, wmin, wmax, img, R.ROWS_SECTOR0, stream)
        else:
            plan = R.Plan(geom, n, nchan, npol, device=local)
            step = lambda: plan.image(n, rows, res, wmin, wmax, img[: nx * ny], img[nx * ny:],
                                      R.ROWS_SECTOR0, stream)
        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        launches0 = R.launch_count()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.nvtx.range_push(f"{precision}_timed")
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        launches = R.launch_count() - launches0
        ms = e0.elapsed_time(e1) / args.steps
        barrier()
        # per-stage times (stage events on the same stream), a second pass
        stage, lat = {}, []
        k = max(3, min(args.steps, 10))
        if plan is not None:
            plan.set_timing(True)
        for _ in range(k):
            step()
            s = plan.stage_ms() if plan is not None else {}
            lat.append(sum(s.values()))
            for kk, v in s.items():
                stage[kk] = stage.get(kk, 0.0) + v
        stage = {kk: v / k for kk, v in stage.items()} or {"phase": 0.0}
        stats = plan.stats() if plan is not None else {"records": 0, "rows_gridded": 0,
                                                       "rows_dropped": 0, "work_items": 0}
        if plan is not None:
            plan.set_timing(False)
        image = img.clone()
        closer = imager if shard_mode else plan
        return closer, image, ms, stage, stats, launches, lat

    forms = args.forms.split(",")
    with ClockSampler(local) as clocks:
        plan64, img64, ms64, stage64, stats64, launches, lat64 = run_form("fp64")
    plan64.close()
    if "mixed" in forms:
        planmx, imgmx, msmx, stagemx, statsmx, _, latmx = run_form("mixed")
        err_mixed = float(torch.linalg.vector_norm(imgmx - img64) / torch.linalg.vector_norm(img64))
        err_mixed_maxabs = float((imgmx - img64).abs().max() / img64.abs().max())
        planmx.close()
    else:
        msmx, stagemx, latmx, err_mixed = float("nan"), {}, [float("nan")], None
        err_mixed_maxabs = None

    # max over ranks
    t = torch.tensor([ms64, msmx], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms64, msmx = float(t[0]), float(t[1])
    jobs_done = 1 if shard_mode else world   # one job split over the GPUs, or one per GPU
    value = jobs_done * nvis / (ms64 * 1e-3)

    # ---- e2e through the host C-ABI entry point (pinned host buffers)
    e2e = None
    e2e_bytes = sum(int(r.numel() * r.element_size()) for r in rows) + 16 * nx * ny
    run_e2e = not args.no_e2e and not shard_mode  # shard mode: device-resident rows only
    if run_e2e and world > 1:
        # every rank pins its own copy of the inputs: all ranks skip the leg
        # unless the node's free host memory holds them with room to spare
        import psutil
        fits = world * e2e_bytes <= 0.6 * psutil.virtual_memory().available
        flag = torch.tensor([1 if fits else 0], dtype=torch.int32, device=dev)
        dist.all_reduce(flag, op=dist.ReduceOp.MIN)
        run_e2e = bool(flag.item())
        if not run_e2e:
            e2e = {"value": None, "unit": "vis/s",
                   "skipped": f"{world} ranks x {e2e_bytes / 1e9:.1f} GB of pinned host buffers "
                              "exceed 60 % of the free host memory"}
    if run_e2e:
        # rows copied straight into pinned buffers (no pageable staging copy)
        host = []
        for r in rows:
            h = torch.empty(r.shape, dtype=r.dtype, pin_memory=True)
            h.copy_(r)
            host.append(h)
        h_img = torch.empty(2 * nx * ny, dtype=torch.float64).pin_memory()
        geom = R.Geometry(nx, ny, nw, cfg.w_support, cfg.kernel, "fp64")
        with R.Plan(geom, n, nchan, npol, device=local) as plan:
            # streaming ingest: the samples' host-to-device copies overlap the binning
            slice_rows = max(1, (256 << 20) // (8 * nv))
            call = lambda: plan.ingest(n, host, res, wmin, wmax, h_img[: nx * ny],
                                       h_img[nx * ny:], R.ROWS_SECTOR0, slice_rows=slice_rows)
            call()
            k_e2e = max(1, min(args.steps, 5))
            barrier()
            t0 = time.perf_counter()
            for _ in range(k_e2e):
                call()
            e2e_s = (time.perf_counter() - t0) / k_e2e
        tt = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_s = float(tt[0])
        bi = sum(int(h.numel() * h.element_size()) for h in host)
        e2e = {"value": world * nvis / e2e_s, "unit": "vis/s", "h2d_bytes_per_step": bi,
               "d2h_bytes_per_step": int(h_img.numel() * 8), "steps": k_e2e,
               "ms_per_step": e2e_s * 1e3}
        del host

    hbm, peak_kind = peaks()
    alg = algorithmic_bytes(n, nvis, npol, stats64["records"], nx, ny, nw, 8,
                            stats64.get("fft_rows", 0))
    dom = max(stage64, key=stage64.get)
    achieved = alg[dom] / (stage64[dom] * 1e-3) / 1e9
    roofline = {"kernel": dom, "kernel_name": STAGE_KERNELS.get(dom, dom),
                "bound": "hbm", "achieved": round(achieved, 1),
                "peak": hbm, "unit": "GB/s", "frac": round(achieved / hbm, 4),
                "traffic": NCU_TRAFFIC.get(dom) if args.workload == "c2" else None,
                "peak_source": peak_kind,
                "algorithmic_bytes": alg[dom],
                "stages_ms": {k: round(v, 4) for k, v in stage64.items()},
                "stages_frac": {k: round(alg[k] / (v * 1e-3) / 1e9 / hbm, 4)
                                for k, v in stage64.items() if v > 0 and alg[k] > 0},
                "fft_rows": stats64.get("fft_rows", 0)}
    if dom == "phase" and stats64.get("fft_rows", 0):
        roofline["note"] = ("column FFT + w-correction + plane sum: bound by FP64 issue and "
                            "latency (one 4096-point column of 16 warps per SM), not by HBM")
        # algorithmic FP64 flops of the column pass: a radix-2-equivalent 5 N log2 N per
        # column FFT of every plane (all planes hold data here), plus the w-correction's
        # ~10 flops per pixel and plane
        cols = nx * nw
        flops = cols * 5.0 * ny * math.log2(ny) + 10.0 * nx * ny * nw
        tf = flops / (stage64[dom] * 1e-3) / 1e12
        peak64 = fp64_gemm_tflops(dev)
        roofline["fp64_compute"] = {"achieved_tflops": round(tf, 2), "flops": flops,
                                    "peak_tflops_nominal": FP64_NOMINAL_TFLOPS,
                                    "frac_of_nominal": round(tf / FP64_NOMINAL_TFLOPS, 3),
                                    "peak_tflops_measured": round(peak64, 2),
                                    "frac_of_measured": round(tf / peak64, 3),
                                    "peak_source": "measured here: cuBLAS FP64 GEMM 4096^3 "
                                                   "(torch.matmul float64), best of 5"}
    g8 = 2 * nw * nx * ny * 8
    in_bytes = sum(int(r.numel() * r.element_size()) for r in rows)
    pipe_bytes = 8 * nvis + n * (24 + 4 * npol) + 4 * g8 + 16 * nx * ny
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(obs, n, nchan, npol, nx, ny, nw, cfg, res, wmin, wmax, steps=1)
    line = {
        "metric": METRIC, "value": value, "unit": "vis/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms64, "higher_is_better": True,
        "scaling": "strong" if shard_mode else "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": WORKLOAD_TEXT[args.workload],
                   "rows": n, "visibilities": nvis, "grid": nx, "w_planes": nw,
                   "kernel": cfg.kernel, "w_support": cfg.w_support,
                   "l2": f"inputs ({in_bytes / 1e9:.2f} GB) larger than L2; no flush"
                         if in_bytes > 126e6 else "inputs smaller than L2",
                   "parallelism": (f"w-plane shards x{world} + NCCL image all-reduce" if shard_mode
                                   else f"replicas x{world}"),
                   "time_fraction": args.time_fraction},
        "e2e": e2e, "gpu_launches": launches,
        "roofline": roofline,
        "pipeline_roofline": {"bytes": pipe_bytes, "achieved_gbs": pipe_bytes / (ms64 * 1e-3) / 1e9,
                              "frac": pipe_bytes / (ms64 * 1e-3) / 1e9 / hbm},
        "forms": {"fp64": {"vis_per_s": jobs_done * nvis / (ms64 * 1e-3), "ms": ms64,
                           "stages_ms": stage64,
                           "p50_ms": float(np.percentile(lat64, 50)),
                           "p99_ms": float(np.percentile(lat64, 99))},
                  "mixed": None if "mixed" not in forms else {
                      "vis_per_s": jobs_done * nvis / (msmx * 1e-3), "ms": msmx,
                      "stages_ms": stagemx,
                      "p50_ms": float(np.percentile(latmx, 50)),
                      "p99_ms": float(np.percentile(latmx, 99)),
                      "rel_l2_vs_fp64": err_mixed,
                      "max_abs_vs_fp64_rel_to_peak": err_mixed_maxabs},
                  "mixed_over_fp64": (ms64 / msmx) if "mixed" in forms else None},
        "job": {"rows_gridded": stats64["rows_gridded"], "rows_dropped": stats64["rows_dropped"],
                "records": stats64["records"], "work_items": stats64["work_items"],
                "generate_s": gen_s},
        "cpu_baseline": cpu,
    }
    if not args.no_batched and world == 1:
        ctx, line["batched"] = run_batched(args, dev, stream)
        if not args.no_served:
            big = {"grid": nx, "w_planes": nw, "w_support": cfg.w_support, "kernel": cfg.kernel,
                   "rows_n": n, "nchan": nchan, "npol": npol, "rows": rows, "res": res,
                   "wmin": wmin, "wmax": wmax, "nvis": nvis, "alone_ms": ms64}
            line["served"] = run_served(args, dev, stream, ctx, big)
    if rank == 0:
        line["clocks"] = clocks.summary()
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_batched(args, dev, stream):
    """Batched snapshot imaging: 256 independent ALMA-like jobs (visibility counts
    log-uniform in 1e4-1e7, grids 256^2-2048^2, 4-16 w-planes, 1-4 channels,
    2 polarisations), the mixed form as one autotuned batch replayed from its CUDA
    graph, against every job imaged alone through a plan in the FP64 plain form."""
    import torch
    import rick_b200 as R
    from rick_b200 import synth

    t0 = time.time()
    specs = synth.snapshot_jobs(args.jobs, device=str(dev))
    torch.cuda.synchronize()
    gen_s = time.time() - t0

    def job_list(precision):
        jobs, imgs = [], []
        for sp in specs:
            o, g = sp.obs, sp.grid
            img = torch.empty(2 * g * g, dtype=torch.float64, device=dev)
            geom = R.Geometry(g, g, sp.w_planes, sp.w_support, sp.kernel, precision)
            rows = (o.uu, o.vv, o.ww, o.weights, o.vis_re, o.vis_im)
            jobs.append(R.Job(geom, o.rows, o.cfg.nchan, o.cfg.npol, rows,
                              R.resolution_of(o.meta), o.meta["wmin"], o.meta["wmax"],
                              img[: g * g], img[g * g:]))
            imgs.append(img)
        return jobs, imgs

    total_vis = sum(sp.nvis for sp in specs)
    jobs, imgs = job_list("mixed")
    t0 = time.time()
    batch = R.Batch(jobs, "mixed", device=dev.index or 0)   # autotunes, captures the graph
    create_s = time.time() - t0
    for _ in range(args.warmup):
        batch.run(stream)
    torch.cuda.synchronize()
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    torch.cuda.nvtx.range_push("batched_timed")
    evs[0].record(stream)
    for k in range(args.steps):
        batch.run(stream)
        evs[k + 1].record(stream)
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    per = [evs[k].elapsed_time(evs[k + 1]) for k in range(args.steps)]
    ms = evs[0].elapsed_time(evs[-1]) / args.steps
    st = batch.stats()
    tune = batch.tuning()
    kernels = batch.kernels_per_run()
    mixed_imgs = [im.clone() for im in imgs]
    batch.close()
    del imgs

    # every job alone, FP64 plain form, one plan per job (created untimed)
    alone_ms, errs, alone_each = 0.0, [], []
    for sp, (job, mimg) in zip(specs, zip(jobs, mixed_imgs)):
        o, g = sp.obs, sp.grid
        geom = R.Geometry(g, g, sp.w_planes, sp.w_support, sp.kernel, "fp64")
        with R.Plan(geom, o.rows, o.cfg.nchan, o.cfg.npol, device=dev.index or 0) as plan:
            img = torch.empty(2 * g * g, dtype=torch.float64, device=dev)
            call = lambda: plan.image(o.rows, job.rows, job.resolution, job.wmin, job.wmax,
                                      img[: g * g], img[g * g:], R.ROWS_ALL, stream)
            call()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            call()
            e1.record(stream)
            torch.cuda.synchronize()
            alone_ms += e0.elapsed_time(e1)
            alone_each.append(e0.elapsed_time(e1))
            den = torch.linalg.vector_norm(img)
            errs.append(float(torch.linalg.vector_norm(mimg - img) / den) if den > 0 else 0.0)
    ctx = {"specs": specs, "jobs": jobs, "alone_ms": alone_each}
    return ctx, {"workload": f"{len(specs)} ALMA-like snapshot jobs, {total_vis:.3e} vis, grids "
                        f"256^2-2048^2, 4-16 w-planes, Kaiser-Bessel support 7",
            "visibilities": total_vis, "jobs": len(specs),
            "grids": {str(g): sum(1 for sp in specs if sp.grid == g) for g in (256, 512, 1024, 2048)},
            "mixed_batched": {"vis_per_s": total_vis / (ms * 1e-3), "ms_per_batch": ms,
                              "p50_ms": float(np.percentile(per, 50)),
                              "p99_ms": float(np.percentile(per, 99)),
                              "gpu_launches_per_batch": kernels, "graph_launches_per_batch": 1,
                              "tuning": tune,
                              "create_s": create_s, "rows_gridded": st["rows_gridded"],
                              "fft_rows": st["fft_rows"]},
            "fp64_alone": {"vis_per_s": total_vis / (alone_ms * 1e-3), "ms_total": alone_ms},
            "batched_mixed_over_fp64_alone": alone_ms / ms,
            "rel_l2_mixed_vs_fp64": {"max": max(errs), "median": float(np.median(errs))},
            "generate_s": gen_s}


def run_served(args, dev, stream, ctx, big):
    """Served imaging stream: Poisson arrivals at swept rates, jobs drawn from the
    snapshot mix plus 5% LOFAR-sized jobs (the headline job: 4096^2 x 32, 1.3e9
    vis), device-resident rows, admission by HBM footprint under a 150 GB
    budget, continuous batching on 2 streams.  Reports p50/p99 latency and
    sustained vis/s per rate against imaging the same requests one at a time in
    the FP64 plain form."""
    import torch
    import rick_b200 as R

    specs, alone_ms = ctx["specs"], ctx["alone_ms"]
    rng = np.random.default_rng(777)
    budget = 150 * 10**9

    def request(k_big):
        if k_big:
            g = big["grid"]
            img = torch.empty(2 * g * g, dtype=torch.float64, device=dev)
            job = R.Job(R.Geometry(g, g, big["w_planes"], big["w_support"], big["kernel"], "mixed"),
                        big["rows_n"], big["nchan"], big["npol"], big["rows"], big["res"],
                        big["wmin"], big["wmax"], img[: g * g], img[g * g:], R.ROWS_SECTOR0)
            return job, big["nvis"], big["alone_ms"], img
        i = int(rng.integers(len(specs)))
        sp, base = specs[i], ctx["jobs"][i]
        g = sp.grid
        img = torch.empty(2 * g * g, dtype=torch.float64, device=dev)
        job = R.Job(R.Geometry(g, g, sp.w_planes, sp.w_support, sp.kernel, "mixed"), base.nrows,
                    base.freq_per_chan, base.polarizations, base.rows, base.resolution,
                    base.wmin, base.wmax, img[: g * g], img[g * g:])
        return job, sp.nvis, alone_ms[i], img

    out = {"workload": "Poisson arrivals of snapshot jobs plus 5% LOFAR-sized jobs "
                       "(4096^2 x 32, 1.3e9 vis), mixed form, budget 150 GB, 3 streams; rate 0 = all at once",
           "budget_gb": budget / 1e9, "rates": []}
    n_req = args.served_requests
    torch.cuda.empty_cache()  # the pool reserves the whole budget up front
    with R.Server("mixed", device=dev.index or 0, hbm_budget=budget, max_batch_jobs=64,
                  streams=3) as srv:
        warm = [request(False) for _ in range(8)] + [request(True)]
        for t in [srv.submit(j) for j, _, _, _ in warm]:
            srv.wait(t)
        for rate in args.served_rates:
            reqs = [request(rng.random() < 0.05) for _ in range(n_req)]
            # rate 0: every request at once (the server's capacity)
            arrivals = (np.cumsum(rng.exponential(1.0 / rate, n_req)) if rate > 0
                        else np.zeros(n_req))
            torch.cuda.synchronize()
            tickets = []
            t0 = time.perf_counter()
            for (job, _, _, _), at in zip(reqs, arrivals):
                while time.perf_counter() - t0 < at:
                    pass
                tickets.append(srv.submit(job))
            res = [srv.wait(t) for t in tickets]
            span = time.perf_counter() - t0
            st = srv.stats()
            lat = [r["latency_ms"] for r in res]
            is_big = [v == big["nvis"] for _, v, _, _ in reqs]
            lat_small = [x for x, b in zip(lat, is_big) if not b] or [float("nan")]
            lat_big = [x for x, b in zip(lat, is_big) if b] or [float("nan")]
            vis = sum(v for _, v, _, _ in reqs)
            alone = sum(a for _, _, a, _ in reqs)
            out["rates"].append({
                "rate_jobs_per_s": rate, "jobs": n_req, "big_jobs": sum(1 for j in reqs if j[1] == big["nvis"]),
                "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                # the two populations apart: snapshot jobs, and the LOFAR-sized ones
                "snapshot_p50_ms": float(np.percentile(lat_small, 50)),
                "snapshot_p99_ms": float(np.percentile(lat_small, 99)),
                "large_p50_ms": float(np.percentile(lat_big, 50)),
                "large_max_ms": float(np.max(lat_big)),
                "sustained_vis_per_s": vis / span,
                "fp64_alone_vis_per_s": vis / (alone * 1e-3),
                "served_over_fp64_alone_offered": (vis / span) / (vis / (alone * 1e-3)),
                "mean_batch_jobs": float(np.mean([r["batch_jobs"] for r in res])),
                "peak_gb": st["peak_bytes"] / 1e9})
            del reqs
    # capacity: the highest rate's sustained throughput is bounded by the offered load
    return out


def _threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def cpu_baseline(obs, n, nchan, npol, nx, ny, nw, cfg, res, wmin, wmax, steps=1,
                 target_s=6.0):
    """The reference's CPU path on a bounded sample, extrapolated to the job.

    wstack: the reference's own compiled CPU wstack (oracle/_ref, OpenMP, all host
    threads) on the first S packed rows, scaled by rows/S; FFT: scipy.fft.ifft2 FP64
    (workers = all threads; FFTW is absent) on P planes, scaled by Nw/P;
    phase_correction: the reference's own on P planes, scaled by Nw/P.
    Falls back to the oracle restatement ("port") where oracle/_ref is absent."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    import torch

    threads = _threads()
    kind = "reference" if O.ref_available(cfg.kernel) else "port"
    nv = nchan * npol

    def host(x, count):
        return np.ascontiguousarray(x[:count].cpu().numpy() if hasattr(x, "cpu") else x[:count])

    # a first small sample sizes the real one to about target_s of wstack
    def time_wstack(S):
        uu, vv, ww = host(obs.uu, S), host(obs.vv, S), host(obs.ww, S)
        wt, vr, vi = host(obs.weights, S * npol), host(obs.vis_re, S * nv), host(obs.vis_im, S * nv)
        keep = (ww * nw).astype(np.int64) < nw
        uu, vv, ww = uu[keep], vv[keep], ww[keep]
        wt = wt.reshape(-1, npol)[keep].ravel(); vr = vr.reshape(-1, nv)[keep].ravel()
        vi = vi.reshape(-1, nv)[keep].ravel()
        plane_grid = np.zeros(2 * nw * nx * ny)
        t0 = time.perf_counter()
        if kind == "reference":
            O.ref_lib(cfg.kernel).wstack(nw, len(uu), nchan, npol, uu, vv, ww, vr, vi, wt, 1 / nx,
                                        1 / nw, cfg.w_support, nx, ny, plane_grid, threads, 0)
        else:
            O.wstack(cfg.kernel, nw, nchan, npol, uu, vv, ww, vr, vi, wt, 1 / nx, 1 / nw,
                     cfg.w_support, nx, ny, plane_grid, threads)
        return time.perf_counter() - t0, plane_grid

    S0 = min(n, 20000)
    t_small, _ = time_wstack(S0)
    S = int(min(n, max(S0, S0 * target_s / max(t_small, 1e-3))))
    results = []
    for _ in range(steps):
        t_w, grid = time_wstack(S)
        P = 2
        sub = np.ascontiguousarray(grid[: 2 * P * nx * ny])
        t0 = time.perf_counter()
        gss = O.fft_planes(sub, P, nx, ny, workers=threads)
        t_f = time.perf_counter() - t0
        img_re, img_im = np.zeros(nx * ny), np.zeros(nx * ny)
        t0 = time.perf_counter()
        if kind == "reference":
            O.ref_lib(cfg.kernel).phase_correction(gss, img_re, img_im, nx, ny, P, nx, ny, res,
                                                  wmin, wmax, threads, 0)
        else:
            O.phase_correction(gss, nx, ny, P, res, wmin, wmax, True, threads, img_re, img_im)
        t_p = time.perf_counter() - t0
        est = t_w * (n / S) + (t_f + t_p) * (nw / P)
        results.append(dict(est=est, t_w=t_w, t_f=t_f, t_p=t_p))
    est = float(np.median([r["est"] for r in results]))
    r0 = results[0]
    del torch
    return {"value": n * nv / est, "unit": "vis/s", "cores": threads, "kind": kind,
            "sample": f"wstack on {S} of {n} rows (x{n / S:.1f}), FFT (scipy.fft, FFTW absent) "
                      f"and phase_correction on 2 of {nw} planes (x{nw / 2:.0f}); "
                      f"sample times wstack {r0['t_w']:.2f}s fft {r0['t_f']:.2f}s "
                      f"phase {r0['t_p']:.2f}s",
            "est_job_s": est}


def run_reference(args):
    """Reference arm: the reference's own CPU path, rank 0 only."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import rick_b200  # noqa: F401  (synthetic generator only)
    from rick_b200 import synth
    import torch

    cfg = synth.CONFIGS[args.workload]
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    obs = synth.make_observation(cfg, seed=2024, device=dev, time_fraction=args.time_fraction)
    import rick_b200 as R
    n = R.rows_read(obs.meta)
    nv = cfg.nchan * cfg.npol
    res = R.resolution_of(obs.meta)
    for _ in range(args.warmup):
        pass  # the sample sizing inside cpu_baseline warms the caches
    cpu = cpu_baseline(obs, n, cfg.nchan, cfg.npol, cfg.grid, cfg.grid, cfg.w_planes, cfg, res,
                       obs.meta["wmin"], obs.meta["wmax"], steps=max(1, min(args.steps, 3)))
    line = {"metric": METRIC, "value": cpu["value"], "unit": "vis/s", "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": cpu["est_job_s"] * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD_TEXT[args.workload],
                       "rows": n, "visibilities": n * nv},
            "cpu_baseline": cpu,
            "e2e": {"value": cpu["value"], "unit": "vis/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.only_batched:
        import torch
        dev = torch.device("cuda", 0)
        torch.cuda.set_device(dev)
        print(json.dumps(run_batched(args, dev, torch.cuda.current_stream(dev))[1]), flush=True)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
