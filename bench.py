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

# DRAM traffic per launch (dram__bytes_read.sum + dram__bytes_write.sum) from ncu
# captures of a kernel on a workload at full size, keyed by (workload, kernel);
# each entry names the capture.  A kernel without a capture reports null.
NCU_TRAFFIC = {
    ("c2", "k_fft_cols_pair<double,12>"): (2_312_723_797, "profiles/traffic_c2.md (mean of 3 "
                                           "launches, one-pass dram__bytes_read/write capture)"),
    ("c2", "k_fft_cols_tm<double,12>"): (2_383_968_341, "profiles/traffic_c2.md (mean of 3 "
                                         "launches, one-pass dram__bytes_read/write capture)"),
    ("c2", "k_bin_scatter<32,1>"): (10_851_913_216, "profiles/traffic_c2.md"),
    ("c2", "k_grid_tiles<double,8>"): (459_853_312, "profiles/traffic_c2.md"),
    ("c2", "k_fft_rows<double,12>"): (2_083_898_112, "profiles/traffic_c2.md"),
}


def plan_kernel_name(stage, nx, ny):
    """The kernel behind a plan stage on the sparse-aware path (FP64)."""
    ly = max(int(ny).bit_length() - 1, 0)
    lx = max(int(nx).bit_length() - 1, 0)
    return {"bin_count": "k_bin_count", "bin_scatter": "k_bin_scatter<32,1>",
            "cube_zero": "k_zero_split_tiles<double>", "grid": "k_grid_tiles<double,8>",
            "fft": f"k_fft_rows<double,{lx}>",
            "phase": (f"k_fft_cols_pair<double,{ly}>" if 10 <= ly <= 12
                      else f"k_fft_cols_tm<double,{ly}>")}.get(stage, stage)


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
    ap.add_argument("--no-dropin", action="store_true",
                    help="skip the drop-in leg (wstack + rick_fft_planes + phase_correction on "
                         "host buffers)")
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
        msmx, stagemx, latmx, err_mixed, imgmx = float("nan"), {}, [float("nan")], None, None
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
    host = None
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

    hbm, peak_kind = peaks()
    alg = algorithmic_bytes(n, nvis, npol, stats64["records"], nx, ny, nw, 8,
                            stats64.get("fft_rows", 0))
    dom = max(stage64, key=stage64.get)
    achieved = alg[dom] / (stage64[dom] * 1e-3) / 1e9
    kname = plan_kernel_name(dom, nx, ny)
    traffic = NCU_TRAFFIC.get((args.workload, kname)) if not args.time_fraction < 1 else None
    roofline = {"kernel": dom, "kernel_name": kname,
                "bound": "hbm", "achieved": round(achieved, 1),
                "peak": hbm, "unit": "GB/s", "frac": round(achieved / hbm, 4),
                "traffic": traffic[0] if traffic else None,
                "traffic_source": traffic[1] if traffic else
                ("no ncu capture of this kernel on this workload"),
                "peak_source": peak_kind,
                "algorithmic_bytes": alg[dom],
                "stages_ms": {k: round(v, 4) for k, v in stage64.items()},
                "stages_frac": {k: round(alg[k] / (v * 1e-3) / 1e9 / hbm, 4)
                                for k, v in stage64.items() if v > 0 and alg[k] > 0},
                "fft_rows": stats64.get("fft_rows", 0)}
    if dom == "phase" and stats64.get("fft_rows", 0):
        roofline["note"] = ("column FFT + w-correction + plane sum (per-pixel state in tensor "
                            "memory): bound by FP64 issue, shared-memory traffic and load "
                            "latency, not by HBM (fp64_compute gives the compute roofline)")
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
    dense_bytes = 8 * nvis + n * (24 + 4 * npol) + 4 * g8 + 16 * nx * ny
    sparse_bytes = sum(alg[k] for k in stage64 if k in alg)
    cpu, oracle_err, dropin, ref_img = None, None, None, None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        hrows = _host_rows(host if host is not None else rows)
        cpu, ref_img = cpu_baseline(hrows, nchan, npol, nx, ny, nw, cfg, res, wmin, wmax)
        del hrows
        ref_t = torch.from_numpy(ref_img).to(dev)
        oracle_err = {"oracle": f"the image of the cpu_baseline run ({cpu['kind']} CPU path, "
                                "FP64, in w-plane chunks)"}
        for nm, im in (("fp64", img64), ("mixed", imgmx)):
            if im is None:
                continue
            oracle_err[nm] = {
                "rel_l2": float(torch.linalg.vector_norm(im - ref_t) / torch.linalg.vector_norm(ref_t)),
                "max_abs_rel_to_peak": float((im - ref_t).abs().max() / ref_t.abs().max())}
        del ref_t
    if rank == 0 and world == 1 and not args.no_dropin and args.workload == "c2":
        hrows = _host_rows(host if host is not None else rows)
        dropin = run_dropin(hrows, nchan, npol, nx, ny, nw, cfg, res, wmin, wmax, ref_img)
        del hrows
    del host
    line = {
        "metric": METRIC, "value": value, "unit": "vis/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms64, "higher_is_better": True,
        "scaling": "strong" if shard_mode else "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": config_of(args, cfg, n, nvis, nx, nw, in_bytes, world, shard_mode),
        "e2e": e2e, "gpu_launches": launches,
        "roofline": roofline,
        "pipeline_roofline": {
            "dense_bytes": dense_bytes,
            "dense_frac": dense_bytes / (ms64 * 1e-3) / 1e9 / hbm,
            "dense_note": "the dense algorithm's bytes (a full cube written, FFT-read and "
                          "-written, read by the w-correction): the bar the path is held to",
            "moved_bytes": sparse_bytes,
            "moved_frac": sparse_bytes / (ms64 * 1e-3) / 1e9 / hbm,
            "moved_note": "the bytes the sparse-aware path itself must move (touched rows only)"},
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
                  "mixed_over_fp64": (ms64 / msmx) if "mixed" in forms else None,
                  "vs_oracle": oracle_err},
        "job": {"rows_gridded": stats64["rows_gridded"], "rows_dropped": stats64["rows_dropped"],
                "records": stats64["records"], "work_items": stats64["work_items"],
                "generate_s": gen_s},
        "cpu_baseline": cpu,
        "dropin": dropin,
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
        # warm-up: every grid size of the mix at least once (each size's kernels
        # are loaded on first use), then a few random jobs and a large one
        sizes = sorted({sp.grid for sp in specs})
        warm = []
        for g in sizes:
            i = next(k for k, sp in enumerate(specs) if sp.grid == g)
            sp, base = specs[i], ctx["jobs"][i]
            img = torch.empty(2 * g * g, dtype=torch.float64, device=dev)
            warm.append((R.Job(R.Geometry(g, g, sp.w_planes, sp.w_support, sp.kernel, "mixed"),
                               base.nrows, base.freq_per_chan, base.polarizations, base.rows,
                               base.resolution, base.wmin, base.wmax, img[: g * g], img[g * g:]),
                         0, 0, img))
        warm += [request(False) for _ in range(8)] + [request(True)]
        for t in [srv.submit(j) for j, _, _, _ in warm]:
            srv.wait(t)
        del warm
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


def run_dropin(hrows, nchan, npol, nx, ny, nw, cfg, res, wmin, wmax, ref_img, steps=2):
    """The drop-in entry points in the reference's own call sequence, on
    pageable host buffers as the reference's main allocates them: wstack of
    every row into a zeroed host cube (gridding_cpu.c:187-204), rick_fft_planes
    (fftw_data's arithmetic, fourier_transform.c:13-93), phase_correction into
    zeroed host images (fourier_transform.c:209-216).  One untimed round, then
    `steps` timed rounds (wall clock: each call synchronises); the counters
    show whether the timed rounds created a plan or allocated row buffers."""
    import rick_b200 as R
    R.set_kernel(cfg.kernel)
    R.set_phase_on(True)
    uu, vv, ww, wt, vr, vi = (np.array(a, copy=True) for a in hrows)   # pageable copies
    n = len(uu)
    grid = np.empty(2 * nw * nx * ny)
    gridss = np.empty_like(grid)
    re, im = np.empty(nx * ny), np.empty(nx * ny)

    def one_round(times):
        t0 = time.perf_counter()
        grid.fill(0.0)
        re.fill(0.0)
        im.fill(0.0)
        t1 = time.perf_counter()
        R.wstack(nw, n, nchan, npol, uu, vv, ww, vr, vi, wt, 1.0 / nx, 1.0 / nw, cfg.w_support,
                 nx, ny, grid)
        t2 = time.perf_counter()
        R.fft_planes(grid, nw, nx, ny, out=gridss)
        t3 = time.perf_counter()
        R.phase_correction(gridss, re, im, nx, ny, nw, nx, ny, res, wmin, wmax)
        t4 = time.perf_counter()
        times.append((t1 - t0, t2 - t1, t3 - t2, t4 - t3))

    warm = []
    one_round(warm)
    c0 = R.dropin_counters()
    times = []
    for _ in range(steps):
        one_round(times)
    c1 = R.dropin_counters()
    R.dropin_release()   # its plan and buffers (~28 GB at this size) leave the device
    tt = np.array(times)
    job_s = float(tt[:, 1:].sum(axis=1).mean())
    out = {"workload": "the headline job's rows (all gridded, as wstack grids every row "
                       "given), 4 host buffers pageable", "steps": steps,
           "vis_per_s": n * nchan * npol / job_s, "ms_per_job": job_s * 1e3,
           "ms_wstack": float(tt[:, 1].mean() * 1e3), "ms_fft": float(tt[:, 2].mean() * 1e3),
           "ms_phase": float(tt[:, 3].mean() * 1e3),
           "host_bytes_moved_per_job": int(sum(a.nbytes for a in (uu, vv, ww, wt, vr, vi))
                                           + 5 * grid.nbytes + 4 * re.nbytes),
           "plans_created_in_timed_rounds": c1["plans_created"] - c0["plans_created"],
           "row_allocations_in_timed_rounds": c1["row_allocations"] - c0["row_allocations"]}
    if ref_img is not None:
        img = np.concatenate([re, im])
        out["rel_l2_vs_oracle"] = float(np.linalg.norm(img - ref_img) / np.linalg.norm(ref_img))
    return out


class CpuJob:
    """The reference's CPU path for one imaging job, timed in w-plane chunks.

    A chunk is `chunk_planes` consecutive w-planes of the job.  Its step runs,
    on every host thread: the cube's zeroing, the reference's own compiled CPU
    ``wstack`` (oracle/_ref, OpenMP) once per plane on that plane's packed rows
    with Nw' = 1 and w' = 0 (w enters wstack only through grid_w,
    w-stacking.cu:466-469, so the plane's cells receive exactly the additions
    of the whole-cube call), the per-plane inverse FFT (scipy.fft, FP64,
    workers = all threads; FFTW is absent) and the reference's own
    ``phase_correction`` over the chunk's planes (wmin/wmax shifted to the
    chunk, the chunk image rescaled by planes/Nw after the step; its 32-bit
    cube index stays below 2^32 for chunks of <= 8 planes of 8192^2).  Row
    selection (one rank's sector 0 after the 1000-row drop) and the packing
    of each plane's rows are set-up outside the timed steps, as the
    reference's own kernel timer leaves out its sector packing
    (gridding_cpu.c:88-138).  Steps cycle through the chunks; the job is every
    chunk once.  Falls back to the oracle's restatement ("port") where
    oracle/_ref was not built."""

    def __init__(self, host, nchan, npol, nx, ny, nw, cfg, res, wmin, wmax, threads,
                 chunk_planes=8):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        self.O = O
        self.kind = "reference" if O.ref_available(cfg.kernel) else "port"
        self.threads = threads
        self.nchan, self.npol, self.nx, self.ny, self.nw = nchan, npol, nx, ny, nw
        self.cfg, self.res, self.wmin, self.wmax = cfg, res, wmin, wmax
        self.c = max(1, min(chunk_planes, nw))
        nv = nchan * npol
        uu, vv, ww, wt, vr, vi = host
        rows = O.sector0_rows(vv, len(uu) + 1000, nx, ny, cfg.w_support).astype(np.int64)
        gw = O.plane_of(ww[rows], nw)
        order = rows[np.argsort(gw, kind="stable")]
        gws = np.sort(gw, kind="stable")
        bounds = np.searchsorted(gws, np.arange(nw + 1))
        self.planes = []
        for iw in range(nw):
            r = order[bounds[iw]:bounds[iw + 1]]
            self.planes.append((np.ascontiguousarray(uu[r]), np.ascontiguousarray(vv[r]),
                                np.zeros(len(r)),
                                np.ascontiguousarray(wt.reshape(-1, npol)[r].ravel()),
                                np.ascontiguousarray(vr.reshape(-1, nv)[r].ravel()),
                                np.ascontiguousarray(vi.reshape(-1, nv)[r].ravel())))
        self.nchunks = (nw + self.c - 1) // self.c
        self.cube = np.zeros(2 * self.c * nx * ny)
        self.image_re, self.image_im = np.zeros(nx * ny), np.zeros(nx * ny)
        self.done = [False] * self.nchunks

    def chunk_vis(self, k):
        a = k * self.c
        return sum(len(p[0]) for p in self.planes[a:a + self.c]) * self.nchan * self.npol

    def job_vis(self):
        return sum(self.chunk_vis(k) for k in range(self.nchunks))

    def step(self, k):
        """Chunk k end to end; returns its wall-clock seconds."""
        O, nx, ny, nw = self.O, self.nx, self.ny, self.nw
        a = k * self.c
        c = min(self.c, nw - a)
        cube = self.cube[: 2 * c * nx * ny]
        dx, dw = 1.0 / nx, 1.0 / nw
        sup, kern = self.cfg.w_support, self.cfg.kernel
        dw_ph = (self.wmax - self.wmin) / nw
        wmin_c = self.wmin + a * dw_ph
        img_re, img_im = np.zeros(nx * ny), np.zeros(nx * ny)
        t0 = time.perf_counter()
        cube.fill(0.0)
        for p in range(c):
            uu, vv, ww, wt, vr, vi = self.planes[a + p]
            plane = cube[2 * p * nx * ny: 2 * (p + 1) * nx * ny]
            if self.kind == "reference":
                O.ref_lib(kern).wstack(1, len(uu), self.nchan, self.npol, uu, vv, ww, vr, vi, wt,
                                       dx, dw, sup, nx, ny, plane, self.threads, 0)
            else:
                O.wstack(kern, 1, self.nchan, self.npol, uu, vv, ww, vr, vi, wt, dx, dw, sup, nx,
                         ny, grid=plane, threads=self.threads)
        gss = O.fft_planes(cube, c, nx, ny, workers=self.threads)
        if self.kind == "reference":
            O.ref_lib(kern).phase_correction(gss, img_re, img_im, nx, ny, c, nx, ny, self.res,
                                             wmin_c, wmin_c + c * dw_ph, self.threads, 0)
        else:
            O.phase_correction(gss, nx, ny, c, self.res, wmin_c, wmin_c + c * dw_ph, True,
                               self.threads, img_re, img_im)
        t = time.perf_counter() - t0
        if not self.done[k]:   # the job's image: each chunk once, at the whole cube's dwnorm
            self.image_re += img_re * (c / nw)
            self.image_im += img_im * (c / nw)
            self.done[k] = True
        return t

    def describe(self):
        return (f"the whole job in {self.nchunks} w-plane chunk(s) of {self.c} plane(s) "
                f"({self.job_vis()} visibilities): the reference's own CPU wstack per plane, "
                f"scipy.fft FP64 (FFTW absent), the reference's own phase_correction per chunk; "
                f"{self.threads} OpenMP threads; row selection and packing untimed")


def _host_rows(rows):
    """numpy views (or copies) of the six row arrays on the host."""
    out = []
    for r in rows:
        if hasattr(r, "is_pinned") and r.device.type == "cpu":
            out.append(r.numpy())
        elif hasattr(r, "cpu"):
            out.append(r.cpu().numpy())
        else:
            out.append(np.asarray(r))
    return out


def cpu_baseline(host, nchan, npol, nx, ny, nw, cfg, res, wmin, wmax):
    """The whole job once through CpuJob (every chunk), timed: about 10-30 s of
    CPU work at the LOFAR-like size.  Returns the cpu_baseline object and the
    job's image (the reference's own CPU result for the error figures)."""
    threads = _threads()
    job = CpuJob(host, nchan, npol, nx, ny, nw, cfg, res, wmin, wmax, threads)
    t = sum(job.step(k) for k in range(job.nchunks))
    vis = job.job_vis()
    return ({"value": vis / t, "unit": "vis/s", "cores": threads, "kind": job.kind,
             "sample": job.describe(), "job_s": t},
            np.concatenate([job.image_re, job.image_im]))


def config_of(args, cfg, n, nvis, nx, nw, in_bytes, world, shard_mode=False):
    """The workload description both arms print (the same dict)."""
    return {"workload": WORKLOAD_TEXT[args.workload], "rows": n, "visibilities": nvis,
            "grid": nx, "w_planes": nw, "kernel": cfg.kernel, "w_support": cfg.w_support,
            "l2": (f"inputs ({in_bytes / 1e9:.2f} GB) larger than L2; no flush"
                   if in_bytes > 126e6 else "inputs smaller than L2"),
            "parallelism": (f"w-plane shards x{world} + NCCL image all-reduce" if shard_mode
                            else f"replicas x{world}"),
            "time_fraction": args.time_fraction}


def run_reference(args):
    """Reference arm: the reference's own CPU path (CpuJob), rank 0 only.  Each
    step is one w-plane chunk of the job (steps cycle through the chunks, so K
    steps cover K/chunks whole jobs); W warm-up steps run the same way,
    untimed; value = visibilities of the timed steps / their summed time."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import torch
    import rick_b200 as R
    from rick_b200 import synth

    cfg = synth.CONFIGS[args.workload]
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    obs = synth.make_observation(cfg, seed=2024, device=dev, time_fraction=args.time_fraction)
    n = R.rows_read(obs.meta)
    nv = cfg.nchan * cfg.npol
    host = _host_rows((obs.uu[:n], obs.vv[:n], obs.ww[:n], obs.weights[: n * cfg.npol],
                       obs.vis_re[: n * nv], obs.vis_im[: n * nv]))
    meta = obs.meta
    del obs
    nx = args.grid or cfg.grid
    nw = args.w_planes or cfg.w_planes
    threads = _threads()
    job = CpuJob(host, cfg.nchan, cfg.npol, nx, nx, nw, cfg, R.resolution_of(meta),
                 meta["wmin"], meta["wmax"], threads)
    in_bytes = sum(int(h.nbytes) for h in host)
    del host
    k = 0
    for _ in range(args.warmup):
        job.step(k % job.nchunks)
        k += 1
    t, vis = 0.0, 0
    for _ in range(args.steps):
        t += job.step(k % job.nchunks)
        vis += job.chunk_vis(k % job.nchunks)
        k += 1
    value = vis / t
    line = {"metric": METRIC, "value": value, "unit": "vis/s", "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_of(args, cfg, n, n * nv, nx, nw, in_bytes, world),
            "cpu_baseline": {"value": value, "unit": "vis/s", "cores": threads, "kind": job.kind,
                             "sample": f"{args.steps} steps of one w-plane chunk each "
                                       f"({vis / (job.job_vis() or 1):.2f} jobs); "
                                       + job.describe()},
            "e2e": {"value": value, "unit": "vis/s", "h2d_bytes_per_step": 0,
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
