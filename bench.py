"""Benchmark: DFT sky-model subtraction, component-visibility evals/s.

One step = one pass of the DFT subtract over one chunk of the config-2 dataset
(64 antennas / 2016 baselines, 4 IFs x 256 channels, 4 polarizations, 20000
point components with spectral index), `--rows` records per chunk (default
100800 = 50 integrations; the full 4.032e6-row dataset, ~198 GB, is 40 such
chunks and does not fit in HBM).  Evals = components x rows x channels x IFs.

  value   device-resident: records already in HBM, one kernel launch per step,
          CUDA events on the launch stream.
  e2e     the reference-facing C ABI call ObitCUDASkyModelDFTCalc-equivalent
          (obit_dft_calc) on a pinned HOST buffer: H2D, kernels and D2H per step.

Multi-GPU (torchrun): every rank subtracts the same model from its own chunk
(weak scaling, no data-path collective); the component table is broadcast once.
`--impl reference` times the reference CPU DFT restatement (oracle/_ref) on the
host cores instead.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

FLOPS_PER_EVAL = 10.0  # complex rotate (6) + accumulate (4), algorithmic
# one metric string for every arm and workload, so that lines can be compared
METRIC = "component-visibility evals/s (DFT subtract)"
# parity bound of every GPU line, checked against the FP64 oracle by the -m gpu tests
ACCURACY = {"max_rel_err_bound": 1e-5, "metric": "|V - V_fp64| / sum_c |A_c| per visibility",
            "checked_by": "tests/test_configs_gpu.py, tests/test_dft_gpu.py (-m gpu)"}
# DRAM bytes (read + write) per record of a workload's records, each from one ncu
# capture of the recurrence kernel on a smaller case of the same layout; traffic
# grows in proportion to records, so a launch's traffic is the figure times its
# records.
#   config1: dft_recur_kernel<32, 0> at 42,120 records (65.61 MB read + 13.73 MB written)
#   config2: dft_recur_kernel<32, 1, ..., spectral-factored> at 10,080 records, 160-component tiles
#            (500.25 MB read + 443.94 MB written)
#   config3: dft_recur_kernel<32, 4, ..., mixed> at 4,032 records (202.13 MB read + 150.94 MB written)
#   config4: dft_recur_kernel<32, 0> at 23,808 records (296.35 MB read + 240.85 MB written)
#   config5: dft_recur_batch_kernel<32, 0> over the 96-facet draw at 189,029 records
#            (rows x 0.001; 3,668.0 MB read + 3,567.0 MB written)
#   beam:    dft_beam_mma_kernel<PointSpec> at 4,032 records (232.3 MB read + 147.8 MB written)
#   grid:    grid_apply_kernel at 4,032 records (215.87 MB read + 144.40 MB written)
NCU_DRAM_BYTES_PER_RECORD = {
    "config1": ((65.61e6 + 13.73e6) / 42120, "42,120-record capture (the whole configuration)"),
    "config2": ((500.25e6 + 443.94e6) / 10080, "10,080-record capture (160-component tiles)"),
    "config3": ((202.13e6 + 150.94e6) / 4032, "4,032-record capture"),
    "config4": ((296.35e6 + 240.85e6) / 23808, "23,808-record capture"),
    "config5": ((3668.0e6 + 3567.0e6) / 189029, "189,029-record capture of the same facet draw"),
    "beam": ((232.3e6 + 147.8e6) / 4032, "4,032-record capture of the tensor-core form"),
    "grid": ((215.87e6 + 144.40e6) / 4032, "4,032-record capture"),
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--rows", type=int, default=None,
                    help="records per step (default: 100800 for config2/3, the whole track else)")
    ap.add_argument("--ncomp", type=int, default=None, help="components (default: the config's)")
    ap.add_argument("--flavor", default="recur", choices=["recur", "plain"])
    ap.add_argument("--K", type=int, default=0)
    ap.add_argument("--ct", type=int, default=0)
    ap.add_argument("--Bt", type=int, default=0, help="channel blocks per CTA tile (0: planner)")
    ap.add_argument("--threads", type=int, default=0, help="threads per CTA (128 or 256)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-peak", action="store_true", help="skip the SGEMM FP32 peak measurement")
    ap.add_argument("--cpu-seconds", type=float, default=12.0,
                    help="CPU work of the cpu_baseline leg's sample")
    ap.add_argument("--cpu-step-seconds", type=float, default=2.0,
                    help="reference arm: CPU work per step (the row sample is sized to it)")
    ap.add_argument("--workload", default="config2",
                    choices=["config1", "config2", "config3", "config4", "config5", "beam", "grid"],
                    help="config2: one chunk of the 64-antenna dataset (default); config5: the "
                         "96-facet uneven batch; beam: the beam-corrected DFT on the config-2 "
                         "layout; grid: the gridded model FT on the config-2 layout")
    ap.add_argument("--beam-model", default="pointspec", choices=["pointspec", "gaussspec"],
                    help="beam workload: points with a spectral index (default) or Gaussians (1-60 arcsec) "
                         "with one")
    ap.add_argument("--grid-kernel", default="reference", choices=["reference", "exact"],
                    help="grid: interpolation weights (the reference's table or exact Lagrange)")
    ap.add_argument("--e2e-row-scale", type=float, default=0.002,
                    help="config5: row scale of the host-memory (streamed) end-to-end pass")
    ap.add_argument("--staging-gb", type=float, default=1.0,
                    help="config5: device staging area of the streamed end-to-end pass (GiB)")
    ap.add_argument("--row-scale", type=float, default=0.01,
                    help="config5: fraction of each facet's drawn rows held in HBM")
    ap.add_argument("--no-autotune", action="store_true", help="config5: keep the planner's tile")
    ap.add_argument("--no-compare", action="store_true",
                    help="skip the comparators (config2-4: the FP64-phase plain kernel on the same "
                         "records and a short config-5 batch pass; config5: the per-facet launches)")
    ap.add_argument("--compare-row-scale", type=float, default=0.01,
                    help="row scale of the config-5 batch pass among the comparators")
    return ap.parse_args()


# ---- workload ------------------------------------------------------------------


class Geometry:
    """One bench workload: this rank's rows (u, v, w), the channel frequencies,
    the component table and the record shape."""

    def __init__(self, name, uvw, fa, freq, sky, nstok, nchan, nif, desc):
        self.name, self.uvw, self.fa, self.freq, self.sky = name, uvw, fa, freq, sky
        self.nstok, self.nchan, self.nif, self.desc = nstok, nchan, nif, desc

    @property
    def rows(self):
        return self.uvw.shape[0]

    @property
    def channels(self):
        return self.nchan * self.nif


DEFAULT_ROWS = {"config1": 42120, "config2": 100800, "config3": 100800, "config4": 119040}


def _track(nant, max_bl, nint, freq, seed, rows, rank):
    """rows of a time-major track of nint integrations, this rank's contiguous slice."""
    from obit_b200 import uvdata as U

    pos = U.array_layout(nant, max_bl, np.random.default_rng(seed))
    nbl = nant * (nant - 1) // 2
    per = max(1, (rows + nbl - 1) // nbl)
    i0 = (rank * per) % max(1, nint - per + 1)
    uvw = U.make_uvw(pos, nint, 45.0, 4.0, 34.0, freq).reshape(nint, nbl, 3)
    return uvw[i0:i0 + per].reshape(-1, 3)[:rows]


def workload_geometry(name: str, rank: int, rows: int | None, ncomp: int | None) -> Geometry:
    """The named configuration (seeded as obit_b200.uvdata.config1..4); config2
    and config3 hold one chunk of `rows` records of the 4.032e6-record track."""
    from obit_b200 import uvdata as U

    rows = rows or DEFAULT_ROWS[name]
    if name == "config1":
        freq = 1.4e9
        fa = U.freq_axis(64, 1, freq - 32e6, 1e6)
        uvw = _track(27, 36e3, 120, freq, 1, rows, rank)
        sky = U.make_comps(U.MOD_POINT, ncomp or 1000, np.random.default_rng(3), radius_deg=0.5)
        return Geometry(name, uvw, fa, freq, sky, 2, 64, 1,
                        f"config1: {len(uvw)} records (27 antennas, 351 baselines x 120 "
                        f"integrations) x 1 IF x 64 ch x 2 pol, {sky.ncomp} point components")
    if name in ("config2", "config3"):
        freq = 1.4e9
        fa = U.freq_axis(256, 4, freq - 512e6, 1e6)
        if name == "config2":
            uvw = _track(64, 36e3, 2000, freq, 2, rows, rank)
            sky = U.make_comps(U.MOD_POINT_SPEC, ncomp or 20000, np.random.default_rng(4),
                               radius_deg=1.0, nterm=1, ref_freq=freq)
            what = f"{sky.ncomp} point components with spectral index"
        else:
            uvw = _track(64, 36e3, 2000, freq, 3, rows, rank)
            sky = U.make_comps(U.MOD_GAUSS_SPEC, ncomp or 50000, np.random.default_rng(5),
                               radius_deg=1.0, nterm=1, gauss_frac=0.3, ref_freq=freq)
            what = (f"{sky.ncomp} components (70 % point, 30 % elliptical Gaussian) with "
                    "spectral index")
        return Geometry(name, uvw, fa, freq, sky, 4, 256, 4,
                        f"{name} chunk: {len(uvw)} records (64 antennas, 2016 baselines) x 4 IF x "
                        f"256 ch x 4 pol, {what}; the 4.032e6-record dataset is streamed in such chunks")
    if name == "config4":
        freq = 22e9
        fa = U.freq_axis(64, 8, freq - 512e6, 2e6)
        uvw = _track(32, 8.0e6, 240, freq, 4, rows, rank)
        c = 0.3 * U.DG2RAD / math.sqrt(2.0)
        sky = U.make_comps(U.MOD_POINT, ncomp or 10000, np.random.default_rng(6),
                           radius_deg=2.0 / 60.0, center=(c, c))
        return Geometry(name, uvw, fa, freq, sky, 2, 64, 8,
                        f"config4: {len(uvw)} records (32 antennas to 8000 km, 496 baselines x 240 "
                        f"integrations) at 22 GHz x 8 IF x 64 ch x 2 pol, {sky.ncomp} point "
                        "components within 2 arcmin of a position 0.3 deg from the phase centre")
    raise ValueError(name)


def build_vis(torch, uvw, nstok, nchan, nif, device, seed):
    rows = uvw.shape[0]
    nrparm = 5
    ncorr = nstok * nchan * nif
    lrec = nrparm + 3 * ncorr
    g = torch.Generator(device=device).manual_seed(seed)
    vis = torch.empty((rows, lrec), dtype=torch.float32, device=device)
    c = vis[:, nrparm:].view(rows, ncorr, 3)
    c[:, :, :2] = 0.01 * torch.randn((rows, ncorr, 2), generator=g, device=device)
    c[:, :, 2] = 1.0
    vis[:, 0:3] = torch.from_numpy(uvw.astype(np.float32)).to(device)
    vis[:, 3] = 256.0
    vis[:, 4] = 0.0
    return vis


# ---- clocks ----------------------------------------------------------------------


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.samples.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for n, v in zip(names, s[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(n)
        pw = [float(s[3]) for s in self.samples if s[3].replace(".", "").isdigit()]
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "power_w_max": max(pw) if pw else None,
                "samples": len(self.samples), "reasons": sorted(reasons)}


# ---- peaks -------------------------------------------------------------------------


def fp32_peak_tflops(torch, device) -> float:
    """Measured FP32 peak: cuBLAS SGEMM 8192^3 with TF32 disabled (best of 5)."""
    torch.backends.cuda.matmul.allow_tf32 = False
    n = 8192
    a = torch.randn((n, n), device=device)
    b = torch.randn((n, n), device=device)
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = max(best, 2.0 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    del a, b
    return best


# ---- CPU baseline ------------------------------------------------------------------


def host_info() -> dict:
    """Host cores usable by this process and the CPU model."""
    model = "unknown"
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"nproc": len(os.sched_getaffinity(0)), "cpu_model": model}


class CpuDFT:
    """Reference CPU DFT restatement (oracle/_ref: the reference's ObitSinCosVec /
    ObitExpVec, FP32 phase, rows split over pthreads as ObitSkyModelFTDFT) on a
    row sample of the workload, on every host core.  Used by the cpu_baseline leg
    and by the reference arm, with the same sizing rule: the sample is grown from
    one row per core until one pass takes about `seconds`."""

    def __init__(self, g: Geometry, seconds: float):
        sys.path.insert(0, str(ROOT / "oracle"))
        import oracle
        from obit_b200 import uvdata as U
        from obit_b200.skymodel import SkyModelParams

        self.g = g
        self.cores = oracle.nthreads_default()
        self.have_ref = oracle.have_refcpu()
        self._fn = oracle.apply_refcpu if self.have_ref else oracle.apply_fp64
        self._params = SkyModelParams()
        self._U = U
        nrow = self.cores
        self._set_rows(nrow)
        dt = self.run()
        if dt < seconds / 2:
            nrow = max(self.cores, int(nrow * seconds / max(dt, 1e-3)))
            nrow = min(self.cores * ((nrow + self.cores - 1) // self.cores), g.rows)
            self._set_rows(nrow)

    def _set_rows(self, nrow: int):
        g = self.g
        self.nrow = nrow
        self.uv = self._U.make_uvdata(g.uvw[:nrow], g.nstok, g.nchan, g.nif, g.freq, g.fa,
                                      np.random.default_rng(9))
        self.evals = nrow * g.channels * g.sky.ncomp

    def run(self) -> float:
        """One pass over the sample; wall seconds."""
        t0 = time.perf_counter()
        self._fn(self.uv, self.g.sky, self._params, nthreads=self.cores)
        return time.perf_counter() - t0

    def sample(self) -> str:
        g = self.g
        what = ("restatement of the reference CPU DFT loop (FP32 phase) linked with the reference's own "
                "ObitSinCosVec/ObitExpVec compiled from its sources") if self.have_ref \
            else "FP64 oracle (reference vector math not built)"
        return (f"{self.nrow} rows x {g.channels} channels x {g.sky.ncomp} components per pass ({what}), "
                f"{self.cores} threads")


def cpu_baseline(g: Geometry, seconds: float):
    """The cpu_baseline leg: one sized pass of CpuDFT; returns (evals/s, cores,
    sample text, kind)."""
    c = CpuDFT(g, seconds)
    dt = c.run()
    return c.evals / dt, c.cores, f"{c.sample()}, {dt:.1f} s", "port"


# ---- arms ------------------------------------------------------------------------


def run_reference(args):
    """Reference arm: the reference CPU DFT restatement on every host core, each
    step one pass over a row sample of the same workload (about
    --cpu-step-seconds of CPU work)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    g = workload_geometry(args.workload, 0, args.rows, args.ncomp)
    c = CpuDFT(g, args.cpu_step_seconds)
    for _ in range(args.warmup):
        c.run()
    ts = [c.run() for _ in range(args.steps)]
    v = c.evals * len(ts) / sum(ts) / 1e9
    line = {
        "impl": "reference", "metric": METRIC,
        "value": v, "unit": "Gevals/s", "n_gpus": 0, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * sum(ts) / len(ts), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 (FP32 phase, FP64 component sum)", "data": "synthetic",
        "config": {**config_block(g, nrow_override=c.nrow), "l2": "not applicable (host cores)"},
        "host": host_info(),
        "cpu_baseline": {"value": v, "unit": "Gevals/s", "cores": c.cores, "kind": "port",
                         "sample": c.sample()},
        "e2e": {"value": v, "unit": "Gevals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def config_block(g: Geometry, nrow_override=None, kernel=None):
    rows = nrow_override or g.rows
    return {"workload": g.desc if nrow_override is None else g.desc.replace(f"{g.rows} records", f"{rows} records"),
            "rows_per_step": rows, "components": int(g.sky.ncomp), "channels": g.channels,
            "polarizations": g.nstok, "model": {0: "Point", 10: "PointSpec nterm=1",
                                                11: "GaussSpec nterm=1"}.get(g.sky.modType, str(g.sky.modType)),
            "w_term": True, "l2": "inputs larger than L2" if rows * (5 + 3 * g.nstok * g.channels) * 4 > 126e6
            else "inputs smaller than L2: L2 flushed between steps",
            "kernel": kernel}


def config5_work(row_scale: float, seed: int = 5) -> list[float]:
    """Component-visibility evaluations of each facet of the draw at row_scale
    (the facet sharding's cost)."""
    from obit_b200 import uvdata as U

    return [float(max(1, int(round(nr * row_scale))) * nc * nif * nch)
            for nr, nc, nif, nch in U.config5_facets(seed=seed)]


def config5_data(torch, device, row_scale: float, seed: int = 5, subset=None):
    """The 96-facet uneven workload (seeded draw: components log-uniform in
    [500, 60000], rows log-uniform in [1e5, 1e7] scaled by row_scale, 1-8 IFs x
    32-512 channels, 2 polarizations), point components within 0.5 deg of each
    facet centre; records built on the device.  subset: the facet indices to
    build (a rank's share; every facet is drawn the same either way).  Returns
    (facets, tensors, full-draw evals)."""
    from obit_b200 import uvdata as U
    from obit_b200.batch import Facet
    from obit_b200.skymodel import SkyModelParams

    draw = U.config5_facets(seed=seed)
    full_evals = sum(r * c * i * ch for r, c, i, ch in draw)
    rng = np.random.default_rng(seed)
    pos = U.array_layout(64, 36e3, rng)
    nbl = 2016
    freq = 1.4e9
    track = U.make_uvw(pos, 2000, 45.0, 4.0, 34.0, freq).astype(np.float32)  # (2000 * 2016, 3)
    facets, keep = [], []
    want = set(range(len(draw))) if subset is None else set(subset)
    for k, (nr, nc, nif, nch) in enumerate(draw):
        rows = max(1, int(round(nr * row_scale)))
        r0 = int(rng.integers(0, len(track) - rows + 1)) if rows < len(track) else 0
        if k not in want:
            rng.uniform(-1.0, 1.0, 2)  # the facet centre's draw, as when it is built
            continue
        uvw = track[r0:r0 + rows]
        if len(uvw) < rows:
            uvw = np.resize(track, (rows, 3))
        bw = 128e6  # per IF, channels of bw / nch, IFs contiguous from 1.0 GHz
        fa = U.freq_axis(nch, nif, 1.0e9, bw / nch)
        lrec = 5 + 3 * 2 * nch * nif
        d_vis = torch.empty((rows, lrec), dtype=torch.float32, device=device)
        d_vis[:, 5:].view(rows, -1, 3)[:, :, :2].normal_(0.0, 0.01)
        d_vis[:, 5:].view(rows, -1, 3)[:, :, 2] = 1.0
        d_vis[:, 0:3] = torch.from_numpy(uvw).to(device)
        d_vis[:, 3:5] = 0.0
        c = (float(rng.uniform(-1.0, 1.0)) * U.DG2RAD, float(rng.uniform(-1.0, 1.0)) * U.DG2RAD)
        sky = U.make_comps(U.MOD_POINT, nc, np.random.default_rng(seed * 1000 + k), radius_deg=0.5,
                           center=c)
        d_comps = torch.from_numpy(sky.comps).to(device)
        uv = U.UVData(np.zeros((1, lrec), np.float32), 2, nch, nif, fa[0], fa)
        keep += [d_vis, d_comps]
        facets.append(Facet(uv, sky, SkyModelParams(), d_vis.data_ptr(), rows, d_comps.data_ptr()))
    return facets, keep, full_evals


def _timed_on(torch, stream, fn, steps, warmup, after=None):
    """Total and per-step CUDA-event milliseconds of `steps` calls of fn on stream."""
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    per = []
    e0.record(stream)
    for _ in range(steps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        per.append((a, b))
    e1.record(stream)
    torch.cuda.synchronize()
    if after:
        after()
    return e0.elapsed_time(e1), [a.elapsed_time(b) for a, b in per]


def config5_measure(torch, device, row_scale, steps, warmup, autotune=True, tile=None,
                    compare=True, sampler=None, subset=None):
    """The 96-facet batch (or a rank's `subset` of it): one graph launch of the
    persistent batched kernel per step (autotuned tile unless `tile` fixes it),
    and, with `compare`, one launch per facet of the recurrence and of the
    FP64-phase plain kernel.  Returns a dict of the measurements."""
    from obit_b200 import _lib
    from obit_b200.batch import DFTBatch

    facets, keep, full_evals = config5_data(torch, device, row_scale, subset=subset)
    batch = DFTBatch(facets)
    try:
        info0 = batch.info()
        stream = torch.cuda.Stream(device=device)
        sp = stream.cuda_stream
        t0 = time.perf_counter()
        if tile:
            batch.set_tile(*tile)
        tuned = batch.autotune(sp) if (autotune and not tile) else None
        torch.cuda.synchronize()
        tune_s = time.perf_counter() - t0
        info = batch.info()
        evals = info["evals"]
        if sampler is not None:
            with sampler:
                t_ms, per = _timed_on(torch, stream, lambda: batch.run(sp), steps, warmup, batch.check)
        else:
            t_ms, per = _timed_on(torch, stream, lambda: batch.run(sp), steps, warmup, batch.check)
        out = {"evals": evals, "full_evals": full_evals, "t_ms": t_ms, "per_ms": per,
               "rows": sum(f.nvis for f in facets), "info": info, "info0": info0, "tuned": tuned,
               "tune_s": tune_s, "batch_gevals_s": evals * steps / (t_ms * 1e-3) / 1e9}
        if compare:
            r_ms, _ = _timed_on(torch, stream, lambda: batch.run_per_facet(_lib.OBIT_DFT_RECUR, sp), 1, 1,
                                batch.check)
            p_ms, _ = _timed_on(torch, stream, lambda: batch.run_per_facet(_lib.OBIT_DFT_PLAIN, sp), 1, 0,
                                batch.check)
            out["per_facet_recur_gevals_s"] = evals / (r_ms * 1e-3) / 1e9
            out["per_facet_plain_gevals_s"] = evals / (p_ms * 1e-3) / 1e9
            out["batch_vs_per_facet_plain"] = out["batch_gevals_s"] / out["per_facet_plain_gevals_s"]
            out["batch_vs_per_facet_recur"] = out["batch_gevals_s"] / out["per_facet_recur_gevals_s"]
        return out
    finally:
        batch.close()
        del keep
        torch.cuda.empty_cache()


def config5_e2e(torch, device, row_scale, steps, warmup, staging_bytes, tile=None, subset=None):
    """The batch over HOST records through obit_dft_batch_run_host: every
    facet's records copied once into pinned host memory, then per step one
    graph launch that streams them through a device staging area (H2D, batch
    kernels, D2H) and a synchronize; wall clock per step."""
    from obit_b200.batch import DFTBatch

    facets, keep, _ = config5_data(torch, device, row_scale, subset=subset)
    hosts = [keep[2 * i].cpu().pin_memory() for i in range(len(facets))]
    batch = DFTBatch(facets)
    try:
        if tile:
            batch.set_tile(*tile)
        stream = torch.cuda.Stream(device=device)
        ptrs = [h.data_ptr() for h in hosts]
        for _ in range(warmup):
            info = batch.run_host(ptrs, staging_bytes, stream.cuda_stream)
        torch.cuda.synchronize()
        batch.check()
        t0 = time.perf_counter()
        for _ in range(steps):
            info = batch.run_host(ptrs, staging_bytes, stream.cuda_stream)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        batch.check()
        return {"evals": batch.info()["evals"], "seconds": dt, "waves": info["waves"],
                "h2d_bytes": info["h2d_bytes"], "rows": sum(f.nvis for f in facets)}
    finally:
        batch.close()
        del keep, hosts
        torch.cuda.empty_cache()


def run_config5(args):
    """One step = one pass of the DFT subtract over all 96 facets: one graph
    launch of the persistent batched kernel (autotuned tile), against one
    launch per facet of the recurrence and of the FP64-phase plain kernel.
    Under torchrun every rank takes whole facets (largest first onto the least
    loaded rank, no data-path collective); the time is the max over ranks."""
    import torch
    import torch.distributed as dist

    from obit_b200 import shard

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    subset = shard.facet_assignment(config5_work(args.row_scale), world)[rank] if world > 1 else None
    fixed = any((args.K, args.ct, args.Bt, args.threads))
    tile = (args.K, args.ct, args.Bt, args.threads) if fixed else None
    sampler = ClockSampler(local)
    m = config5_measure(torch, device, args.row_scale, args.steps, args.warmup,
                        autotune=not args.no_autotune, tile=tile,
                        compare=not args.no_compare and world == 1, sampler=sampler, subset=subset)
    info, evals = m["info"], m["evals"]
    t_ms, per = m["t_ms"], m["per_ms"]
    if world > 1:
        t_ms = shard.max_over_ranks(t_ms, device)
        evals = int(sum(config5_work(args.row_scale)))  # every rank's facets
    value = evals * args.steps / (t_ms * 1e-3)
    e2e = None
    if not args.no_e2e:
        # the tuned tile of this rank's batch, on a smaller row sample held in host memory
        t = tile or ((m["tuned"]["K"], m["tuned"]["ct"], m["tuned"]["Bt"], m["tuned"]["threads"])
                     if m["tuned"] else None)
        ee = config5_e2e(torch, device, args.e2e_row_scale, args.steps, 1, args.staging_gb * (1 << 30),
                         tile=t, subset=subset)
        sec = shard.max_over_ranks(ee["seconds"], device) if world > 1 else ee["seconds"]
        tot = int(sum(config5_work(args.e2e_row_scale))) if world > 1 else ee["evals"]
        e2e = {"value": tot * args.steps / sec / 1e9, "unit": "Gevals/s",
               "h2d_bytes_per_step": ee["h2d_bytes"], "d2h_bytes_per_step": ee["h2d_bytes"],
               "timing": "wall clock around obit_dft_batch_run_host + synchronize (graph: waves of "
                         "H2D -> persistent batch kernels -> D2H), max over ranks",
               "workload": f"rows x {args.e2e_row_scale} of the draw in pinned host memory, "
                           f"{ee['waves']} waves through {args.staging_gb} GiB of device staging",
               "evals_per_step": tot}
    comp = {k: m[k] for k in ("per_facet_recur_gevals_s", "per_facet_plain_gevals_s",
                              "batch_vs_per_facet_plain", "batch_vs_per_facet_recur") if k in m}
    peak = float("nan") if args.no_peak else fp32_peak_tflops(torch, device)
    achieved = evals * FLOPS_PER_EVAL / (statistics.mean(per) * 1e-3) / 1e12
    line = {
        "metric": METRIC,
        "value": value / 1e9, "unit": "Gevals/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (split-FP32 phase)",
        "data": "synthetic (seeded facet draw, noise visibilities, random point components)",
        "accuracy": ACCURACY,
        "config": {"workload": f"config5: 96 facets, rows x {args.row_scale} of the drawn 1e5-1e7 "
                               "per facet held in HBM, 1-8 IF x 32-512 ch, 2 pol, 500-60000 point "
                               "components per facet",
                   "evals_per_step": evals, "full_draw_evals": m["full_evals"],
                   "rows": m["rows"], "facets": info["facets"],
                   "l2": "inputs larger than L2",
                   "tile_planner": {k: m["info0"][k] for k in ("K", "ct", "Bt", "R", "threads")},
                   "tile_autotuned": m["tuned"], "autotune_s": m["tune_s"],
                   "launch": f"1 CUDA graph launch per step ({info['launches']} persistent kernel(s), "
                             f"grid {info['grid']})"},
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak,
                     "traffic": NCU_DRAM_BYTES_PER_RECORD["config5"][0] * m["rows"],
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per record ("
                                       + NCU_DRAM_BYTES_PER_RECORD["config5"][1] + ") x records per launch",
                     "peak_source": "measured here: cuBLAS SGEMM 8192^3, TF32 off (best of 5)"},
        "comparators": comp,
        "host": host_info(),
        "cpu_baseline": None, "e2e": e2e,
        "gpu_launches": info["launches"] * args.steps,
        "clocks": sampler.summary(),
    }
    if world > 1:
        line["n_gpus"] = world
        line["config"]["sharding"] = "whole facets per rank (largest first onto the least loaded rank)"
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def run_beam(args):
    """The beam-corrected DFT (obit_dft_set_beam) on the config-2 layout: a chunk
    of `--rows` records (default 20,160 = 10 integrations of 2016 baselines) x 4
    IF x 256 channels x 4 correlations (XX, YY, XY, YX all modelled), 4,000
    point components with spectral index, 2 antenna types, 3 Jones planes, a
    Stokes I sky; seeded Jones matrices near identity.  Device-resident records,
    CUDA events; the per-channel form (FP64 phase, one sin/cos per evaluation)
    on the same records as the comparator.  Algorithmic work per evaluation:
    the phasor (complex rotate, 6 flops) and one complex multiply-accumulate
    per modelled correlation (8 flops each)."""
    import torch

    from obit_b200 import _lib
    from obit_b200 import uvdata as U
    from obit_b200.beam import Beam, baseline_codes
    from obit_b200.skymodel import GPUSkyModel, SkyModelParams

    device = torch.device("cuda", 0)
    torch.cuda.set_device(0)
    rows = args.rows or 20160
    freq = 1.4e9
    fa = U.freq_axis(256, 4, freq - 512e6, 1e6)
    uvw = _track(64, 36e3, 2000, freq, 2, rows, 0)
    mtype = U.MOD_GAUSS_SPEC if args.beam_model == "gaussspec" else U.MOD_POINT_SPEC
    sky = U.make_comps(mtype, args.ncomp or 4000, np.random.default_rng(4), radius_deg=1.0,
                       nterm=1, ref_freq=freq)
    d_vis = build_vis(torch, uvw, 4, 256, 4, device, seed=100)
    d_vis[:, 3] = torch.from_numpy(baseline_codes(64, rows)).to(device)
    lrec = d_vis.shape[1]
    r = np.random.default_rng(7)
    ntype, njc = 2, 3
    jones = np.zeros((ntype, sky.ncomp, njc, 8), np.float32)
    jones[..., 0] = 1.0
    jones[..., 6] = 1.0
    jones += (0.1 * r.standard_normal(jones.shape)).astype(np.float32)
    beam = Beam(np.arange(64) % ntype, (np.arange(1024) * njc // 1024).astype(np.int32), jones)
    d_jones = torch.from_numpy(jones).to(device)
    uvh = U.UVData(np.zeros((1, lrec), np.float32), 4, 256, 4, freq, fa)
    gm = GPUSkyModel("beam-bench")
    gm.DFTInit(sky, uvh, SkyModelParams(nVisPIO=1, numberPoln=2))
    gm.set_beam(beam, d_jones.data_ptr())
    gm.DFTSetMod(sky)
    stream = torch.cuda.Stream(device=device)
    sp = stream.cuda_stream
    evals = rows * 1024 * sky.ncomp
    ncorr = 4
    flops = 6.0 + 8.0 * ncorr
    run = lambda: gm.calc_device(d_vis.data_ptr(), rows, sp)  # noqa: E731
    form = gm.beam_info()
    with torch.cuda.stream(stream):
        sampler = ClockSampler(0)
        for _ in range(args.warmup):
            run()
        torch.cuda.synchronize()
        gm.check()
        with sampler:
            t_ms, launch_ms = _timed_on(torch, stream, run, args.steps, 0, gm.check)
        comp = None
        if not args.no_compare:
            rate = evals * args.steps / (t_ms * 1e-3) / 1e9
            comp = {}
            for name, flavor, what in (
                    ("block_form", _lib.OBIT_DFT_RECUR_CHAIN,
                     "8-channel blocks on the FP32 pipe (packed complex multiply-accumulate per correlation)"),
                    ("per_channel_form", _lib.OBIT_DFT_PLAIN,
                     "one thread per record and channel, FP64 phase, one sin/cos per component-visibility")):
                gm.set_kernel(flavor)
                gm.set_beam(beam, d_jones.data_ptr())
                c_ms, _ = _timed_on(torch, stream, run, 1, 1, gm.check)
                cr = evals / (c_ms * 1e-3) / 1e9
                comp[name] = {"gevals_s": cr, "speedup": rate / cr, "what": what + "; same records, 1 launch"}
    value = evals * args.steps / (t_ms * 1e-3)
    # e2e: the same records from a pinned host buffer through obit_dft_calc
    # (H2D, the beam kernels and D2H inside each synchronous call)
    e2e = None
    if not args.no_e2e:
        host = d_vis.cpu()
        # the descriptor holds all the records, so the wrapper's pinned buffer
        # (nVisPIO records, capped at the descriptor's count) takes the chunk
        uve = U.UVData(host.numpy(), 4, 256, 4, freq, fa)
        ge = GPUSkyModel("beam-e2e")
        ge.DFTInit(sky, uve, SkyModelParams(nVisPIO=rows, numberPoln=2))
        ge.set_beam(beam, d_jones.data_ptr())
        ge.DFTSetMod(sky)
        gi = ge.gpuinfo
        if gi.contents.bufferSize < rows * lrec:
            raise RuntimeError("the pinned record buffer is smaller than the chunk")
        C.memmove(gi.contents.h_data, host.data_ptr(), rows * lrec * 4)
        gi.contents.nvis = rows
        gi.contents.h_visInfo.contents.nvis = rows
        _lib.check(ge._lib.obit_dft_calc(gi))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            _lib.check(ge._lib.obit_dft_calc(gi))
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        e2e = {"value": evals * args.steps / dt / 1e9, "unit": "Gevals/s",
               "h2d_bytes_per_step": rows * lrec * 4, "d2h_bytes_per_step": rows * lrec * 4,
               "timing": "wall clock around the synchronous C-ABI call"}
        ge.DFTShutdown()
        ge.close()
    peak = float("nan") if args.no_peak else fp32_peak_tflops(torch, device)
    achieved = evals * flops / (statistics.mean(launch_ms) * 1e-3) / 1e12
    line = {
        "metric": METRIC, "value": value / 1e9, "unit": "Gevals/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (split-FP32 phase)",
        "data": "synthetic (seeded uvw, noise visibilities, random components and Jones matrices)",
        "accuracy": {**ACCURACY, "checked_by": "tests/test_beam_gpu.py (-m gpu)"},
        "config": {"workload": f"beam: {rows} records (64 antennas, 2016 baselines) x 4 IF x 256 ch x 4 "
                               f"correlations, {sky.ncomp} "
                               f"{'Gaussian' if mtype == U.MOD_GAUSS_SPEC else 'point'} components with "
                               f"spectral index, "
                               f"{ntype} antenna types, {njc} Jones planes, Stokes I sky",
                   "rows_per_step": rows, "components": int(sky.ncomp), "channels": 1024,
                   "correlations": ncorr, "l2": "inputs larger than L2", "timing": "CUDA events around all steps",
                   "beam_form": {0: "blocks, FP32 pipe", 1: "tensor-core (mma.sync TF32, 3-product split)",
                                 2: "per channel"}[form["form"]], "components_per_tile": form["ct"]},
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak, "traffic": NCU_DRAM_BYTES_PER_RECORD["beam"][0] * rows,
                     "traffic_source": "ncu dram__bytes_read + dram__bytes_write of a " +
                                       NCU_DRAM_BYTES_PER_RECORD["beam"][1] + ", scaled by records",
                     "peak_source": "measured here: cuBLAS SGEMM 8192^3, TF32 off (best of 5)",
                     "flops_per_eval": flops,
                     "note": "algorithmic FP32 work of the model (complex rotate + one complex multiply-"
                             "accumulate per correlation); the tensor-core form executes the multiply-"
                             "accumulates as TF32 products (tensor_executed)"},
        "tensor_executed": ({"tf32_tflops": evals * 96.0 / (statistics.mean(launch_ms) * 1e-3) / 1e12,
                             "flops_per_eval": 96.0, "what": "3 mma.sync m16n8k8 TF32 products per 64 evaluations "
                             "(3-product split); ncu puts the pipe at 41 % of its peak on the 4,032-record case"}
                            if form["form"] == 1 else None),
        "comparators": comp, "host": host_info(), "cpu_baseline": None, "e2e": e2e,
        # the tensor-core form runs its coefficient and amplitude prologues before the kernel
        "gpu_launches": args.steps * (3 if form["form"] == 1 else 1), "clocks": sampler.summary(),
    }
    print(json.dumps(line), flush=True)
    gm.DFTShutdown()
    gm.close()


def grid_field(N: int, ncomp: int, cell_asec: float, seed: int = 8):
    """A CLEAN model of `ncomp` components on the cells of the central half of
    an N x N image of cell_asec pixels (2-D field at the phase centre), fluxes
    log-uniform over [1 mJy, 1 Jy]."""
    from obit_b200.comps import CCField, CCModel
    from obit_b200.grid import GridImage

    r = np.random.default_rng(seed)
    cell = cell_asec / 3600.0
    ix = r.integers(-N // 4, N // 4, ncomp)
    iy = r.integers(-N // 4, N // 4, ncomp)
    flux = np.exp(r.uniform(math.log(1e-3), 0.0, ncomp)).astype(np.float32)
    f = CCField(flux=flux, deltaX=(ix * -cell).astype(np.float32), deltaY=(iy * cell).astype(np.float32),
                crvalRA=0.0, crvalDec=34.0, do3D=False, cdeltX=-cell, cdeltY=cell)
    return f, GridImage(N, N, N / 2 + 1, N / 2 + 1), CCModel(uvRA=0.0, uvDec=34.0)


def run_grid(args):
    """The gridded model FT (obit_dft_grid_*) on the config-2 layout: a chunk of
    `--rows` records (default 20,160 = 10 integrations of 2016 baselines) x 4 IF
    x 256 channels x 4 polarizations (the first two subtracted), against a
    CLEAN model of `--ncomp` components (default 20,000) on the cells of a
    4096 x 4096 image of 0.25 arcsec pixels (an 8192 x 8192 grid: the plane
    reaches 1.8 x the longest baseline).  value: model visibilities (record x
    channel x IF) per second of the apply kernel on device-resident records,
    CUDA events; setup: the field's gridding, FFT and plane (wall clock of the
    blocking create call); e2e: the host-records call (H2D, kernel, D2H per
    step).  dft_equivalent: components x model visibilities per second, the
    DFT's metric for the same model and records."""
    import torch

    from obit_b200 import grid as GR
    from obit_b200.skymodel import OP_SUB, SkyModelParams

    device = torch.device("cuda", 0)
    torch.cuda.set_device(0)
    rows = args.rows or 20160
    ncomp = args.ncomp or 20000
    N = 4096
    freq = 1.4e9
    from obit_b200 import uvdata as U
    fa = U.freq_axis(256, 4, freq - 512e6, 1e6)
    uvw = _track(64, 36e3, 2000, freq, 2, rows, 0)
    f, img, m = grid_field(N, ncomp, 0.25)
    kernel = GR.KERNEL_EXACT if args.grid_kernel == "exact" else GR.KERNEL_REFERENCE
    d_vis = build_vis(torch, uvw, 4, 256, 4, device, seed=100)
    lrec = d_vis.shape[1]
    uvh = U.UVData(np.zeros((1, lrec), np.float32), 4, 256, 4, freq, fa)
    p = SkyModelParams(op=OP_SUB)
    d_fs = torch.from_numpy(np.ascontiguousarray(uvh.fscale)).to(device)
    stream = torch.cuda.Stream(device=device)
    sp = stream.cuda_stream
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    gf = GR.GridField(f, img, m, kernel=kernel, stream=sp)
    setup_ms = (time.perf_counter() - t0) * 1e3
    setups = []
    for _ in range(3):  # repeat the set-up (plans and allocations included)
        t0 = time.perf_counter()
        GR.GridField(f, img, m, kernel=kernel, stream=sp).close()
        setups.append((time.perf_counter() - t0) * 1e3)
    info = gf.info()
    nvisch = rows * 1024
    run = lambda: gf.FTGrid_device(uvh, d_vis.data_ptr(), rows, p, d_fscale=d_fs.data_ptr(), stream=sp)  # noqa: E731
    with torch.cuda.stream(stream):
        sampler = ClockSampler(0)
        for _ in range(args.warmup):
            run()
        torch.cuda.synchronize()
        with sampler:
            t_ms, launch_ms = _timed_on(torch, stream, run, args.steps, 0)
    value = nvisch * args.steps / (t_ms * 1e-3)
    e2e = None
    if not args.no_e2e:
        h = torch.empty((rows, lrec), dtype=torch.float32, pin_memory=True)
        h.copy_(d_vis.cpu())
        uvp = U.UVData(h.numpy(), 4, 256, 4, freq, fa)
        vi, _fs = GR.vis_info(uvp, p)
        lib = gf._lib
        call = lambda: lib.obit_dft_grid_apply_host(gf._h, C.byref(vi), p.op, 1.0, 0,  # noqa: E731
                                                    C.c_void_p(h.data_ptr()), rows, C.c_void_p(sp))
        call()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            assert call() == 0
        te = (time.perf_counter() - t0) / args.steps
        e2e = {"value": nvisch / te / 1e9, "unit": "G model visibilities/s",
               "h2d_bytes_per_step": rows * lrec * 4, "d2h_bytes_per_step": rows * lrec * 4,
               "what": "obit_dft_grid_apply_host on pinned host records: H2D, kernel, D2H, synchronized"}
    # algorithmic DRAM bytes of a launch: the selected correlations of every record
    # read and written (2 polarizations x 1024 channels x 12 bytes, twice) and u, v, w
    algo = rows * (3 * 4 + 2 * 2 * 1024 * 12)
    mean_launch = statistics.mean(launch_ms)
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    achieved = algo / (mean_launch * 1e-3) / 1e9
    gather = nvisch * 25 * 13 * 16 / (mean_launch * 1e-3) / 1e12
    cpu = None
    if not args.no_cpu:
        cpu = grid_cpu_baseline(f, img, m, uvw, fa, freq, args.cpu_seconds)
    line = {
        "metric": "model visibilities/s (gridded model FT subtract)", "value": value / 1e9,
        "unit": "G model visibilities/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded uvw, noise visibilities, components on random cells)",
        "accuracy": {"bound": "|V - V_oracle| / sum|flux| < 1e-5 (reference kernel, against the oracle's "
                              "restatement); exact kernel against the DFT oracle < 1e-5",
                     "checked_by": "tests/test_grid_gpu.py (-m gpu)"},
        "config": {"workload": f"grid: {rows} records (64 antennas, 2016 baselines) x 4 IF x 256 ch x 4 pol "
                               f"(2 subtracted), {info['ncomp']} components on the cells of a {N} x {N} "
                               f"image (0.25 arcsec), {info['nx']} x {info['ny']} grid",
                   "rows_per_step": rows, "components": info["ncomp"], "kernel": args.grid_kernel,
                   "l2": "inputs larger than L2 (records); the plane (%.0f MB) is read through L2" %
                         (info["ny"] * (info["nxp"] + 1) * 8 / 1e6),
                   "timing": "CUDA events around all steps"},
        "setup_ms": {"first": setup_ms, "repeat_median": statistics.median(setups),
                     "what": "obit_dft_grid_create (host gridding, cuFFT plan and R2C, taper and conjugate "
                             "columns), wall clock, blocking"},
        "dft_equivalent": {"gevals_s": ncomp * value / 1e9,
                           "gevals_s_with_setup": ncomp * nvisch * args.steps /
                           ((t_ms + statistics.median(setups)) * 1e-3) / 1e9,
                           "what": "components x model visibilities per second: the DFT metric for the same "
                                   "model and records (one set-up per step counted in the second figure)"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "traffic": NCU_DRAM_BYTES_PER_RECORD["grid"][0] * rows,
                     "traffic_source": "ncu dram__bytes_read + dram__bytes_write of a " +
                                       NCU_DRAM_BYTES_PER_RECORD["grid"][1] + ", scaled by records",
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs",
                     "note": "algorithmic bytes are the records' selected correlations read and written; the "
                             "kernel's limit is its window gathers through L1/L2 (25 rows x 13 16-byte pairs "
                             "per model visibility)",
                     "gather_tb_s": gather},
        "host": host_info(), "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": args.steps,
        "clocks": sampler.summary(),
    }
    print(json.dumps(line), flush=True)
    gf.close()


def grid_cpu_baseline(f, img, m, uvw, fa, freq, seconds):
    """The reference's gridded-model loop restated in C (oracle/refcpu_grid.c,
    single precision, records split over pthreads as ObitSkyModelFTGrid) on a
    record sample, every host core; the plane from the oracle's FFT (not timed)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle
    import oracle_grid as OG
    from obit_b200 import uvdata as U
    from obit_b200.skymodel import OP_SUB, SkyModelParams

    gm = OG.build(f, OG.GridImage(img.nx, img.ny, img.crpixX, img.crpixY), m)
    cores = oracle.nthreads_default()
    p = SkyModelParams(op=OP_SUB)
    nrow = cores
    while True:
        uv = U.make_uvdata(uvw[:nrow], 4, 256, 4, freq, fa, np.random.default_rng(9))
        t0 = time.perf_counter()
        OG.apply_c(gm, uv, p, nthreads=cores)
        dt = time.perf_counter() - t0
        if dt >= seconds / 2 or nrow >= len(uvw):
            break
        nrow = min(len(uvw), max(nrow * 2, int(nrow * seconds / max(dt, 1e-3))))
    return {"value": nrow * 1024 / dt / 1e9, "unit": "G model visibilities/s", "cores": cores, "kind": "port",
            "sample": f"{nrow} records x 1024 channels (2 polarizations subtracted), {dt:.1f} s: "
                      "oracle/refcpu_grid.c, the reference's ThreadSkyModelFTGrid loop in single precision"}


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.workload == "config5":
        run_config5(args)
        return
    if args.workload == "beam":
        run_beam(args)
        return
    if args.workload == "grid":
        run_grid(args)
        return

    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    from obit_b200 import _lib, shard
    from obit_b200 import uvdata as U
    from obit_b200.skymodel import GPUSkyModel, SkyModelParams

    g = workload_geometry(args.workload, rank, args.rows, args.ncomp)
    uvw, fa, freq, sky = g.uvw, g.fa, g.freq, g.sky
    if world > 1:  # replicate the component table from rank 0 (one broadcast, outside timing)
        sky.comps = shard.broadcast_model(torch.from_numpy(sky.comps).to(device)).cpu().numpy()
    rows = uvw.shape[0]
    nstok, nchan, nif = g.nstok, g.nchan, g.nif
    d_vis = build_vis(torch, uvw, nstok, nchan, nif, device, seed=100 + rank)
    lrec = d_vis.shape[1]

    # host-side descriptor and the GPU sky model (C host mirror -> C ABI)
    want_e2e = not args.no_e2e
    host = torch.empty((rows, lrec), dtype=torch.float32, pin_memory=True) if want_e2e else None
    if want_e2e:
        host.copy_(d_vis.cpu())
        uvh = U.UVData(host.numpy(), nstok, nchan, nif, freq, fa)
    else:
        uvh = U.UVData(np.zeros((rows, lrec), np.float32)[:1], nstok, nchan, nif, freq, fa)
        uvh.vis = np.zeros((1, lrec), np.float32)
    params = SkyModelParams(nVisPIO=rows if want_e2e else 1, GPU_no=local, numberPoln=2)
    gm = GPUSkyModel(f"bench{rank}")
    gm.DFTInit(sky, uvh, params)
    flavor = _lib.OBIT_DFT_PLAIN if args.flavor == "plain" else _lib.OBIT_DFT_RECUR
    gm.set_kernel(flavor, args.K, args.ct, args.Bt, args.threads)
    gm.DFTSetMod(sky)
    lib = _lib.load()

    stream = torch.cuda.Stream(device=device)
    sp = stream.cuda_stream
    evals = rows * nchan * nif * sky.ncomp

    def barrier():
        if world > 1:
            dist.barrier()

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            gm.calc_device(d_vis.data_ptr(), rows, sp)
    torch.cuda.synchronize()
    gm.check()
    barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    per_launch = []
    # records smaller than L2 (126 MB, x2 margin) would stay cached between
    # steps: overwrite a 512 MB buffer before each step and time the launches
    flush = torch.empty(128 << 20, dtype=torch.float32, device=device) if rows * lrec * 4 < 252e6 else None
    with sampler:
        ev0.record(stream)
        for _ in range(args.steps):
            if flush is not None:
                with torch.cuda.stream(stream):
                    flush.fill_(1.0)
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            gm.calc_device(d_vis.data_ptr(), rows, sp)
            b.record(stream)
            per_launch.append((a, b))
        ev1.record(stream)
        torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    gm.check()
    launch_ms = [a.elapsed_time(b) for a, b in per_launch]
    t_ms = ev0.elapsed_time(ev1) if flush is None else sum(launch_ms)
    if world > 1:
        t_ms = shard.max_over_ranks(t_ms, device)
    value = world * evals * args.steps / (t_ms * 1e-3)

    # e2e: host buffer through obit_dft_calc (H2D + kernels + D2H inside)
    e2e = None
    if want_e2e:
        gi = gm.gpuinfo
        C.memmove(gi.contents.h_data, host.data_ptr(), rows * lrec * 4)
        gi.contents.nvis = rows
        gi.contents.h_visInfo.contents.nvis = rows
        for _ in range(1):
            _lib.check(lib.obit_dft_calc(gi))
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            _lib.check(lib.obit_dft_calc(gi))
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        if world > 1:
            dt = shard.max_over_ranks(dt, device)
        e2e = {"value": world * evals * args.steps / dt / 1e9, "unit": "Gevals/s",
               "h2d_bytes_per_step": rows * lrec * 4, "d2h_bytes_per_step": rows * lrec * 4,
               "timing": "wall clock around the synchronous C-ABI call, max over ranks"}

    # comparators on one GPU, measured in the same run: the FP64-phase plain
    # kernel on the same device-resident records, and a short pass of the
    # multi-facet batch against one plain launch per facet
    comp = None
    if world == 1 and not args.no_compare:
        comp = {}
        if args.flavor == "recur":
            gm.set_kernel(_lib.OBIT_DFT_PLAIN, 0, 0, 0, 0)
            pt_ms, _ = _timed_on(torch, stream, lambda: gm.calc_device(d_vis.data_ptr(), rows, sp), 2, 1,
                                 gm.check)
            pl = evals * 2 / (pt_ms * 1e-3) / 1e9
            gm.set_kernel(flavor, args.K, args.ct, args.Bt, args.threads)
            comp["same_records"] = {
                "plain_fp64_phase_gevals_s": pl, "recur_vs_plain": (value / 1e9) / pl,
                "what": "FP64-phase plain kernel (one sin/cos per component-visibility) on the same "
                        "records and model, 2 launches"}
            if gm.plan_info()["specFactored"]:
                # the chain form of the same recurrence (no spectral factoring)
                gm.set_kernel(_lib.OBIT_DFT_RECUR_CHAIN, args.K, args.ct, args.Bt, args.threads)
                ch_ms, _ = _timed_on(torch, stream, lambda: gm.calc_device(d_vis.data_ptr(), rows, sp),
                                     2, 1, gm.check)
                ch = evals * 2 / (ch_ms * 1e-3) / 1e9
                gm.set_kernel(flavor, args.K, args.ct, args.Bt, args.threads)
                comp["same_records"].update({
                    "recur_chain_form_gevals_s": ch, "factored_vs_chain": (value / 1e9) / ch,
                    "chain_what": "the recurrence with the chain form for spectral point models "
                                  "(OBIT_DFT_RECUR_CHAIN), same records, 2 launches"})
    if world == 1 and not args.no_compare and args.workload == "config2":
        m = config5_measure(torch, device, args.compare_row_scale, 2, 1, autotune=True, compare=True)
        comp["config5_batch"] = {
            "what": f"config 5: 96 uneven facets, rows x {args.compare_row_scale} of the draw resident; "
                    "one CUDA-graph launch of the persistent batch (autotuned tile) vs one launch "
                    "per facet",
            "evals_per_pass": m["evals"], "batch_gevals_s": m["batch_gevals_s"],
            "per_facet_recur_gevals_s": m["per_facet_recur_gevals_s"],
            "per_facet_plain_gevals_s": m["per_facet_plain_gevals_s"],
            "batch_vs_per_facet_plain": m["batch_vs_per_facet_plain"],
            "batch_vs_per_facet_recur": m["batch_vs_per_facet_recur"],
            "tile_autotuned": m["tuned"]}

    line = None
    if rank == 0:
        peak = float("nan") if args.no_peak else fp32_peak_tflops(torch, device)
        avg_launch_s = statistics.mean(launch_ms) * 1e-3
        achieved = evals * FLOPS_PER_EVAL / avg_launch_s / 1e12
        cpu = None
        if not args.no_cpu:
            v, cores, sample, kind = cpu_baseline(g, args.cpu_seconds)
            cpu = {"value": v / 1e9, "unit": "Gevals/s", "cores": cores, "kind": kind, "sample": sample}
        pi = gm.plan_info()
        kern = (f"{args.flavor} K={pi['K']} ct={pi['ct']} Bt={pi['Bt']} R={pi['R']} "
                f"threads={pi['threads']}" + (" spectral-factored" if pi["specFactored"] else ""))
        line = {
            "metric": METRIC,
            "value": value / 1e9, "unit": "Gevals/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 (split-FP32 phase)" if args.flavor == "recur" else "f32 (FP64 phase)",
            "data": "synthetic (seeded uvw, noise visibilities, random components)",
            "accuracy": ACCURACY,
            "config": {**config_block(g, kernel=kern),
                       "timing": "sum of per-launch CUDA-event times, L2 flushed before each"
                       if flush is not None else "CUDA events around all steps"},
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak,
                         "traffic": NCU_DRAM_BYTES_PER_RECORD[g.name][0] * rows
                         if (args.flavor == "recur" and g.name in NCU_DRAM_BYTES_PER_RECORD) else None,
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per record ("
                                           + NCU_DRAM_BYTES_PER_RECORD.get(g.name, (0, "no capture"))[1]
                                           + ") x records per launch",
                         "peak_source": "measured here: cuBLAS SGEMM 8192^3, TF32 off (best of 5)",
                         "flops_per_eval": FLOPS_PER_EVAL},
            "comparators": comp,
            "host": host_info(),
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": args.steps,
            "clocks": sampler.summary(),
        }
        print(json.dumps(line), flush=True)
    gm.DFTShutdown()
    gm.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
