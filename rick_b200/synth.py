"""Seeded synthetic interferometric observations in RICK's binMS layout.

The reference has no dataset (its paramfile names a LOFAR measurement set that is
not shipped), so observations are synthesised here with the shapes, sizes and
value distributions of the imaging workloads this library is measured on:

* antenna layouts (uniform disc, log-radial, VLA-like Y, compact disc);
* Earth-rotation uvw tracks over an hour-angle range at a declination, one row
  per (time, baseline) pair, time-major like a measurement set;
* point-source skies (log-normal or power-law fluxes) plus complex Gaussian
  noise, all polarisations carrying Stokes I for XX/YY and zero for XY/YX;
* unit weights.

Coordinates are normalised exactly as scripts/create_binMS.py:155-198 does:
``u' = (u + maxg) / (2 maxg)``, ``v' = (v + maxg) / (2 maxg)``,
``w' = (w - minw) / (maxw - minw)`` with ``maxg = max(max|u|, max|v|)``,
``ming = min(min u, min v)`` (offset 0), and the meta lines of
scripts/create_binMS.py:226-245 carry ``uvmin = ming``, ``uvmax = maxg``,
``wmin``, ``wmax`` in wavelengths at the band centre.  As in the reference
(w-stacking.cu:186-200) every channel of a row is gridded at that row's uv; the
visibilities themselves are computed at each channel's own frequency.

Small random draws (antennas, sources) use ``numpy.random.default_rng(seed)``, so
they are identical on every device; visibility sums run in torch on the chosen
device, and the noise comes from a torch generator on that device.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Optional

import numpy as np

C_LIGHT = 299_792_458.0


@dataclasses.dataclass(frozen=True)
class ObsConfig:
    name: str
    layout: str              # "disc", "lograd", "yarms", "compact"
    n_ant: int
    extent_m: float          # disc diameter / max radius / arm length
    latitude_deg: float
    dec_deg: float
    hours: float
    dt_s: float
    nchan: int
    f_lo_hz: float
    f_hi_hz: float
    npol: int
    n_src: int
    flux: str                # "lognormal" or "powerlaw"
    field_deg: float         # diameter of the source field
    noise: float
    grid: int
    w_planes: int
    kernel: str              # "gauss", "gauss_hi", "kaiser_bessel"
    w_support: int


# The imaging workloads.  Array latitudes are not given by the workload
# descriptions; the values below are those of typical sites for each array.
CONFIGS = {
    # Plain FP64 imaging, small: runs on the reference CPU path.
    "c1": ObsConfig("c1", "disc", 40, 3000.0, 45.0, 45.0, 1.0, 10.0, 8, 120e6, 128e6, 2,
                    20, "lognormal", 2.0, 0.1, 512, 8, "gauss", 7),
    # LOFAR-like large single image.
    "c2": ObsConfig("c2", "lograd", 60, 40000.0, 52.9, 50.0, 4.0, 5.0, 64, 130e6, 142e6, 4,
                    200, "lognormal", 5.0, 0.5, 4096, 32, "kaiser_bessel", 7),
    # JVLA-like wide field with a large w range.
    "c3": ObsConfig("c3", "yarms", 27, 21000.0, 34.1, 10.0, 6.0, 2.0, 16, 1.0e9, 1.5e9, 2,
                    500, "powerlaw", 4.0, 0.0, 8192, 64, "gauss_hi", 9),
}


def channel_freqs(cfg: ObsConfig) -> np.ndarray:
    width = (cfg.f_hi_hz - cfg.f_lo_hz) / cfg.nchan
    return cfg.f_lo_hz + width * (np.arange(cfg.nchan) + 0.5)


def antenna_enu(cfg: ObsConfig, rng: np.random.Generator) -> np.ndarray:
    """East/north/up positions in metres, shape (n_ant, 3)."""
    n = cfg.n_ant
    if cfg.layout in ("disc", "compact"):
        r = 0.5 * cfg.extent_m * np.sqrt(rng.random(n))
        th = 2 * np.pi * rng.random(n)
    elif cfg.layout == "lograd":
        r = np.exp(rng.uniform(np.log(30.0), np.log(cfg.extent_m), n))
        th = 2 * np.pi * rng.random(n)
    elif cfg.layout == "yarms":
        per_arm = n // 3
        k = np.arange(1, per_arm + 1)
        radii = cfg.extent_m * (k / per_arm) ** 1.716
        r = np.concatenate([radii] * 3)[:n]
        arms = np.deg2rad(np.array([355.0, 115.0, 236.0]))
        th = np.repeat(arms, per_arm)[:n] + rng.normal(0, 0.002, n)
    else:
        raise ValueError(cfg.layout)
    e, nn = r * np.sin(th), r * np.cos(th)
    return np.stack([e, nn, np.zeros(n)], axis=1)


def uvw_tracks(cfg: ObsConfig, enu: np.ndarray) -> tuple[np.ndarray, int, int]:
    """Earth-rotation uvw (metres) of every (time, baseline) row, time-major."""
    lat, dec = np.deg2rad(cfg.latitude_deg), np.deg2rad(cfg.dec_deg)
    x = -np.sin(lat) * enu[:, 1] + np.cos(lat) * enu[:, 2]
    y = enu[:, 0]
    z = np.cos(lat) * enu[:, 1] + np.sin(lat) * enu[:, 2]
    a1, a2 = np.triu_indices(cfg.n_ant, k=1)
    bx, by, bz = x[a2] - x[a1], y[a2] - y[a1], z[a2] - z[a1]
    ntimes = int(round(cfg.hours * 3600.0 / cfg.dt_s))
    h = (np.arange(ntimes) + 0.5) * cfg.dt_s - 0.5 * cfg.hours * 3600.0
    h = h * (2 * np.pi / 86164.0905)
    sh, ch = np.sin(h)[:, None], np.cos(h)[:, None]
    u = sh * bx + ch * by
    v = -np.sin(dec) * ch * bx + np.sin(dec) * sh * by + np.cos(dec) * bz
    w = np.cos(dec) * ch * bx - np.cos(dec) * sh * by + np.sin(dec) * bz
    uvw = np.stack([u.ravel(), v.ravel(), w.ravel()], axis=1)
    return uvw, ntimes, len(a1)


def sky(cfg: ObsConfig, rng: np.random.Generator) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    rad = np.deg2rad(0.5 * cfg.field_deg)
    r = rad * np.sqrt(rng.random(cfg.n_src))
    th = 2 * np.pi * rng.random(cfg.n_src)
    l, m = r * np.cos(th), r * np.sin(th)
    if cfg.flux == "lognormal":
        s = rng.lognormal(0.0, 1.0, cfg.n_src)
    else:  # power law N(>S) ~ S^-1.6 between 1 mJy and 1 Jy (inverse-CDF draw)
        a, lo, hi = -1.6, 1e-3, 1.0
        q = rng.random(cfg.n_src)
        s = (lo ** a + q * (hi ** a - lo ** a)) ** (1.0 / a)
    return l, m, s


@dataclasses.dataclass
class Observation:
    """One binMS dataset held in memory (arrays are numpy or torch tensors)."""
    cfg: ObsConfig
    uu: object               # float64 [rows] normalised
    vv: object
    ww: object
    weights: object          # float32 [rows * npol]
    vis_re: object           # float32 [rows * nchan * npol]
    vis_im: object
    meta: dict

    @property
    def rows(self) -> int:
        return int(self.meta["Nmeasures"])


def make_observation(cfg: ObsConfig | str, seed: int = 1234, device: str = "cpu",
                     time_fraction: float = 1.0, chunk_rows: int = 65536,
                     nan_fraction: float = 0.0, as_numpy: Optional[bool] = None) -> Observation:
    """Synthesise one observation.

    ``time_fraction`` < 1 keeps only that leading fraction of the time steps (the
    parity tests use this to shrink a workload while keeping its geometry).
    ``nan_fraction`` > 0 sets that fraction of real parts to NaN (the reference
    skips those samples, w-stacking.cu:191-192).  Returns numpy arrays when the
    device is the CPU (or ``as_numpy``), torch tensors on the device otherwise.
    """
    import torch

    if isinstance(cfg, str):
        cfg = CONFIGS[cfg]
    rng = np.random.default_rng(seed)
    enu = antenna_enu(cfg, rng)
    uvw_m, ntimes, nbl = uvw_tracks(cfg, enu)
    if time_fraction < 1.0:
        keep_t = max(1, int(round(ntimes * time_fraction)))
        uvw_m = uvw_m[: keep_t * nbl]
        ntimes = keep_t
    l, m, s = sky(cfg, rng)
    freqs = channel_freqs(cfg)
    f0 = 0.5 * (cfg.f_lo_hz + cfg.f_hi_hz)
    lam0 = C_LIGHT / f0
    uvw = uvw_m / lam0                          # wavelengths at band centre
    rows = uvw.shape[0]

    dev = torch.device(device)
    n_minus_1 = np.sqrt(1.0 - l * l - m * m) - 1.0
    src = torch.tensor(np.stack([l, m, n_minus_1], 0), dtype=torch.float64, device=dev)  # [3,S]
    flux = torch.tensor(s, dtype=torch.complex64, device=dev)
    fscale = torch.tensor(freqs / f0, dtype=torch.float64, device=dev)
    pol_is_i = torch.tensor([1.0, 0.0, 0.0, 1.0] if cfg.npol == 4 else [1.0] * cfg.npol,
                            dtype=torch.float32, device=dev)
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed + 7919)

    uvw_t = torch.tensor(uvw, dtype=torch.float64, device=dev)
    vis_re = torch.empty((rows, cfg.nchan, cfg.npol), dtype=torch.float32, device=dev)
    vis_im = torch.empty_like(vis_re)
    for r0 in range(0, rows, chunk_rows):
        r1 = min(rows, r0 + chunk_rows)
        ph = uvw_t[r0:r1] @ src                  # cycles at f0, [R,S]
        for c in range(cfg.nchan):
            x = ph * fscale[c]
            x = x - torch.floor(x)              # reduce to one turn in FP64
            e = torch.polar(torch.ones_like(x, dtype=torch.float32), (-2 * math.pi * x).float())
            stokes_i = e @ flux                  # [R]
            vis_re[r0:r1, c, :] = stokes_i.real[:, None] * pol_is_i
            vis_im[r0:r1, c, :] = stokes_i.imag[:, None] * pol_is_i
    if cfg.noise > 0:
        vis_re += cfg.noise * torch.randn(vis_re.shape, generator=gen, device=dev)
        vis_im += cfg.noise * torch.randn(vis_im.shape, generator=gen, device=dev)
    if nan_fraction > 0:
        mask = torch.rand(vis_re.shape, generator=gen, device=dev) < nan_fraction
        vis_re[mask] = float("nan")

    # scripts/create_binMS.py:155-198 (offset 0)
    u, v, w = uvw_t[:, 0], uvw_t[:, 1], uvw_t[:, 2]
    minu, maxu = float(u.min()), float(u.abs().max())
    minv, maxv = float(v.min()), float(v.abs().max())
    minw, maxw = float(w.min()), float(w.max())
    ming, maxg = min(minu, minv), max(maxu, maxv)
    uu = (u + maxg) / (2 * maxg)
    vv = (v + maxg) / (2 * maxg)
    ww = (w - minw) / (maxw - minw)
    weights = torch.ones(rows * cfg.npol, dtype=torch.float32, device=dev)
    meta = dict(Nmeasures=rows, Nvis=rows * cfg.nchan * cfg.npol, freq_per_chan=cfg.nchan,
                polarisations=cfg.npol, Ntimes=ntimes, dt=cfg.dt_s,
                thours=cfg.dt_s * ntimes / 3600.0, baselines=nbl, uvmin=ming, uvmax=maxg,
                wmin=minw, wmax=maxw)
    obs = Observation(cfg, uu, vv, ww, weights, vis_re.reshape(-1), vis_im.reshape(-1), meta)
    if as_numpy or (as_numpy is None and dev.type == "cpu"):
        obs = to_numpy(obs)
    return obs


def to_numpy(obs: Observation) -> Observation:
    def cv(x):
        return x.detach().cpu().numpy() if hasattr(x, "detach") else np.asarray(x)
    return dataclasses.replace(obs, uu=cv(obs.uu), vv=cv(obs.vv), ww=cv(obs.ww),
                               weights=cv(obs.weights), vis_re=cv(obs.vis_re),
                               vis_im=cv(obs.vis_im))


# ---- batched snapshot imaging: many small independent jobs ------------------

@dataclasses.dataclass
class BatchJobSpec:
    """One job of the batched-snapshot workload: its observation and image shape."""
    obs: Observation
    grid: int
    w_planes: int
    kernel: str
    w_support: int

    @property
    def nvis(self) -> int:
        return int(self.obs.meta["Nvis"])


def snapshot_jobs(n_jobs: int = 256, seed: int = 4242, device: str = "cpu",
                  vis_range=(1e4, 1e7), grids=(256, 512, 1024, 2048), planes=(4, 16),
                  chans=(1, 4), kernel: str = "kaiser_bessel", w_support: int = 7,
                  scale: float = 1.0) -> list[BatchJobSpec]:
    """ALMA-like compact-array snapshots: 43 antennas within 500 m at latitude
    -23 deg, declination uniform in [-60, +20] deg, 2 s integrations, 1-4
    channels across 99.5-100.5 GHz, 2 polarisations, 5-50 log-normal point
    sources in a 0.01 deg field plus noise 0.1.  Visibility counts log-uniform
    in ``vis_range`` (times ``scale``), grids drawn from ``grids``, w-planes
    uniform in ``planes``.  Seeded per job."""
    rng = np.random.default_rng(seed)
    specs = []
    nbl = 43 * 42 // 2
    for j in range(n_jobs):
        nvis = float(np.exp(rng.uniform(np.log(vis_range[0]), np.log(vis_range[1])))) * scale
        nchan = int(rng.integers(chans[0], chans[1] + 1))
        npol = 2
        rows = max(nbl, int(nvis / (nchan * npol)))
        ntimes = max(1, int(round(rows / nbl)))
        dt = 2.0
        cfg = ObsConfig(f"snap{j}", "compact", 43, 500.0, -23.0,
                        float(rng.uniform(-60.0, 20.0)), ntimes * dt / 3600.0, dt, nchan,
                        99.5e9, 100.5e9, npol, int(rng.integers(5, 51)), "lognormal", 0.01, 0.1,
                        int(rng.choice(grids)), int(rng.integers(planes[0], planes[1] + 1)),
                        kernel, w_support)
        obs = make_observation(cfg, seed=seed * 1000 + j, device=device)
        specs.append(BatchJobSpec(obs, cfg.grid, cfg.w_planes, kernel, w_support))
    return specs
