#!/usr/bin/env python
"""Benchmark: welch on 64 channels x 2^20 float32 samples (nperseg=1024, noverlap=512, hann,
density, fs=48 kHz) on B200 -- the headline workload of mlx-signal's spectral path.

Usage:
    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
For N > 1 launch under torchrun (one rank per GPU); every rank processes its own 64-channel
batch (channels are independent: replicas, no data-path collective) and the timing is the max
over ranks.

Printed (rank 0, one JSON line):
  value        whole-job algorithmic throughput in GB/s (input read once + PSD written once)
               with the input resident in HBM, timed with CUDA events over exactly K steps
  e2e          the same metric through the public API (mlx_signal_b200.welch) from pinned host
               memory: host->device copy, kernels and the device->host read of the PSD per step
  roofline     the fused welch step (k_welch_half + its reduction) against the measured HBM
               copy bandwidth of MEASURED_PEAKS.json
  cpu_baseline the reference's CPU route (scipy.signal.welch on float32) over a process pool on
               the box's host cores (rank 0, N=1 only)
  clocks       NVML-sampled SM clock and throttle reasons during the timed regions
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

C, NSAMP, NPERSEG, NOVERLAP, FS = 64, 1 << 20, 1024, 512, 48000.0
HOP = NPERSEG - NOVERLAP
NBINS = NPERSEG // 2 + 1
ALG_BYTES = C * NSAMP * 4 + C * NBINS * 4  # input read once + PSD written once
#: published device time of the reference on this workload (Apple M4 Max, MLX backend)
PUBLISHED_DEVICE_MS = 3.63
WORKLOAD = "welch 64ch x 2^20 f32, nperseg=1024, noverlap=512, hann, density, fs=48000"
METRIC = "welch 64ch x 2^20 HBM GB/s (algorithmic bytes / device time)"
#: accuracy bar of the headline PSD: max relative error on bins above 1e-6 of the row peak
ACCURACY_BAR = 1e-5


def rel_err_bins(got, ref, floor: float = 1e-6) -> float:
    """Max relative error of `got` against the float64 reference over the bins whose magnitude
    exceeds `floor` x the peak of their row. A shape mismatch or a non-finite value raises
    RuntimeError, so a broken result is never reported beside a measurement."""
    got, ref = np.asarray(got), np.asarray(ref)
    if got.shape != ref.shape:
        raise RuntimeError(f"accuracy check: result shape {got.shape} != reference {ref.shape}")
    if not (np.isfinite(got).all() and np.isfinite(ref).all()):
        raise RuntimeError("accuracy check: non-finite values in the result or the reference")
    mag = np.abs(ref)
    if mag.size == 0:
        return 0.0
    keep = mag > floor * mag.max(axis=-1, keepdims=True)
    if not keep.any():
        return 0.0
    return float(np.max(np.abs(got - ref)[keep] / mag[keep]))


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-secondary", action="store_true")
    ap.add_argument("--seed", type=int, default=2)
    ap.add_argument("--serving-seconds", type=float, default=10.0,
                    help="arrival window per rate of the serving sweep (the config's 10 s)")
    ap.add_argument("--serving-per-request-seconds", type=float, default=2.0,
                    help="above 5 k req/s offered, the plain per-request path (capacity ~7 k "
                         "req/s) is driven with this many seconds of the same schedule")
    ap.add_argument("--serving-extra-rates", action="store_true",
                    help="also run 100 k and 200 k req/s (beyond the config's 1 k-50 k)")
    return ap.parse_args()


def config_dict(world: int) -> dict:
    """The workload description, identical in both arms."""
    return {
        "workload": WORKLOAD,
        "channels": C,
        "samples": NSAMP,
        "nperseg": NPERSEG,
        "noverlap": NOVERLAP,
        "per_gpu_batch": f"{C} channels",
        "parallelism": f"replicas x{world} (independent channels, no collective)",
        "l2": "input 268 MB > 126 MB L2 each step (no flush needed)",
    }


# ---------------------------------------------------------------------------------------------
# clocks (NVML sampling thread)
# ---------------------------------------------------------------------------------------------

_REASONS = {
    0x1: "gpu_idle",
    0x2: "applications_clocks_setting",
    0x4: "sw_power_cap",
    0x8: "hw_slowdown",
    0x10: "sync_boost",
    0x20: "sw_thermal_slowdown",
    0x40: "hw_thermal_slowdown",
    0x80: "hw_power_brake_slowdown",
    0x100: "display_clock_setting",
}


class ClockSampler:
    """Samples SM clock and clock-event reasons every ~2 ms while `active` is set."""

    def __init__(self, torch_dev: int):
        self.samples: list[tuple[int, int]] = []
        self.max_mhz = None
        self.ok = False
        self.active = threading.Event()
        self._stop = threading.Event()
        try:
            import pynvml

            pynvml.nvmlInit()
            self.nv = pynvml
            handle = None
            try:
                import torch

                props = torch.cuda.get_device_properties(torch_dev)
                bus = f"{props.pci_domain_id:08x}:{props.pci_bus_id:02x}:{props.pci_device_id:02x}.0"
                handle = pynvml.nvmlDeviceGetHandleByPciBusId(bus.encode())
            except Exception:
                handle = pynvml.nvmlDeviceGetHandleByIndex(torch_dev)
            self.h = handle
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(handle, pynvml.NVML_CLOCK_SM)
            self.ok = True
        except Exception:
            self.ok = False
        self.thread = threading.Thread(target=self._run, daemon=True)
        if self.ok:
            self.thread.start()

    def _run(self):
        nv = self.nv
        while not self._stop.is_set():
            if self.active.is_set():
                try:
                    mhz = nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)
                    try:
                        rs = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                    except Exception:
                        rs = nv.nvmlDeviceGetCurrentClocksThrottleReasons(self.h)
                    self.samples.append((int(mhz), int(rs)))
                except Exception:
                    pass
                time.sleep(0.002)
            else:
                time.sleep(0.001)

    def summary(self):
        if not self.ok:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvml unavailable"]}
        self._stop.set()
        self.thread.join(timeout=1)
        reasons = set()
        for _, rs in self.samples:
            for bit, name in _REASONS.items():
                if rs & bit:
                    reasons.add(name)
        mhz = [m for m, _ in self.samples]
        return {
            "sm_mhz": statistics.median(mhz) if mhz else None,
            "sm_max_mhz": self.max_mhz,
            "reasons": sorted(reasons),
            "samples": len(mhz),
        }


# ---------------------------------------------------------------------------------------------
# workload
# ---------------------------------------------------------------------------------------------


def make_input(seed: int, device):
    """Seeded synthetic config-2 input on the device: N(0,1) + 1..4 sinusoids per channel with
    frequencies in (0, fs/2) and amplitudes in [0.1, 2] (phase computed in float64)."""
    import torch

    g = torch.Generator(device=device)
    g.manual_seed(seed)
    x = torch.randn((C, NSAMP), generator=g, device=device, dtype=torch.float32)
    rs = np.random.default_rng(seed)
    t = torch.arange(NSAMP, device=device, dtype=torch.float64) / FS
    for c in range(C):
        for _ in range(int(rs.integers(1, 5))):
            f = float(rs.uniform(0.0, FS / 2))
            a = float(rs.uniform(0.1, 2.0))
            ph = torch.remainder(2.0 * math.pi * f * t, 2.0 * math.pi)
            x[c] += (a * torch.sin(ph)).to(torch.float32)
    return x


def make_pair(seed: int, device):
    """Seeded cross-spectral pair: x ~ N(0,1) (C x 2^20 float32); y = 0.7 x delayed by a seeded
    circular shift s_c in [0, 64] per channel + 0.3 N(0,1)."""
    import torch

    g = torch.Generator(device=device)
    g.manual_seed(seed)
    x = torch.randn((C, NSAMP), generator=g, device=device, dtype=torch.float32)
    shifts = np.random.default_rng(seed).integers(0, 65, size=C)
    y = 0.3 * torch.randn((C, NSAMP), generator=g, device=device, dtype=torch.float32)
    for c in range(C):
        y[c] += 0.7 * torch.roll(x[c], int(shifts[c]))
    return x, y, shifts


def traffic_from_profiles():
    """DRAM bytes per launch of the welch kernel from the committed ncu summary, if present."""
    p = ROOT / "profiles" / "welch_64x2p20_n1024_ncu.md"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.strip().startswith("dram_bytes_per_launch:"):
            try:
                return int(line.split(":", 1)[1].strip().replace(",", ""))
            except ValueError:
                return None
    return None


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


# ---------------------------------------------------------------------------------------------
# CPU legs (oracle / reference CPU route)
# ---------------------------------------------------------------------------------------------


def cpu_welch_rate(x_np: np.ndarray, channels: int, repeats: int):
    """scipy.signal.welch (float32 input) over a spawn process pool using every host core;
    returns (GB/s of algorithmic bytes, cores, seconds per repeat)."""
    from oracle import cpu_reference

    cores = os.cpu_count() or 1
    sample = np.ascontiguousarray(x_np[:channels])
    kw = dict(fs=FS, nperseg=NPERSEG, noverlap=NOVERLAP)
    cpu_reference.pool_map_rows("welch", (sample[:cores],), cores, **kw)  # warm the workers
    times = []
    for _ in range(repeats):
        t0 = time.perf_counter()
        cpu_reference.pool_map_rows("welch", (sample,), cores, **kw)
        times.append(time.perf_counter() - t0)
    sec = statistics.median(times)
    bytes_sample = channels * NSAMP * 4 + channels * NBINS * 4
    return bytes_sample / sec / 1e9, cores, sec


def run_reference(args, rank, world):
    """`--impl reference`: the reference's CPU route timed on the host (rank 0 only)."""
    if rank != 0:
        return
    rs = np.random.default_rng(args.seed)
    x_np = rs.standard_normal((C, NSAMP)).astype(np.float32)
    t = np.arange(NSAMP) / FS
    for c in range(C):
        for _ in range(int(rs.integers(1, 5))):
            x_np[c] += (rs.uniform(0.1, 2.0) * np.sin(2 * np.pi * rs.uniform(0, FS / 2) * t)).astype(
                np.float32
            )
    from oracle import cpu_reference

    cores = os.cpu_count() or 1
    kw = dict(fs=FS, nperseg=NPERSEG, noverlap=NOVERLAP)
    # size each step so the whole K+W run stays within ~2 minutes
    t0 = time.perf_counter()
    cpu_reference.pool_map_rows("welch", (x_np[: min(C, cores)],), cores, **kw)
    per_ch = (time.perf_counter() - t0) / max(1, min(C, cores)) * min(C, cores) / max(1, min(cores, C))
    budget = 120.0 / max(1, args.steps + args.warmup)
    channels = int(max(1, min(C, budget / max(per_ch, 1e-3) * min(cores, C))))
    sample = np.ascontiguousarray(x_np[:channels])
    for _ in range(args.warmup):
        cpu_reference.pool_map_rows("welch", (sample,), cores, **kw)
    times = []
    for _ in range(args.steps):
        t1 = time.perf_counter()
        cpu_reference.pool_map_rows("welch", (sample,), cores, **kw)
        times.append(time.perf_counter() - t1)
    cpu_reference.close_pool()
    total = sum(times)
    bytes_step = channels * NSAMP * 4 + channels * NBINS * 4
    value = bytes_step * len(times) / total / 1e9
    line = {
        "metric": METRIC,
        "value": value,
        "unit": "GB/s",
        "impl": "reference",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": total / len(times) * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded N(0,1) + 1-4 sinusoids per channel)",
        "config": config_dict(world),
        "cpu_baseline": {
            "value": value,
            "unit": "GB/s",
            "cores": cores,
            "kind": "port",
            "sample": f"{channels} of {C} channels per step; scipy.signal.welch on float32 "
                      f"(the reference's CPU route, spectral.py:433-450) over a {cores}-process "
                      "pool split by channel",
        },
        "e2e": {"value": value, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------------------------


def timed(fn, steps, warmup, dist=None, clocks=None):
    """Run fn warmup times, then exactly `steps` times between CUDA events (barrier + sync on
    both sides); returns max-over-ranks milliseconds per step."""
    import torch

    for _ in range(warmup):
        fn()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    s = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if clocks is not None:
        clocks.active.set()
    e0.record(s)
    for _ in range(steps):
        fn()
    e1.record(s)
    torch.cuda.synchronize()
    if clocks is not None:
        clocks.active.clear()
    if dist is not None:
        dist.barrier()
    ms = e0.elapsed_time(e1) / steps
    if dist is not None:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    return ms


def serving_accuracy(pool, seed):
    """Served results against the float64 oracle on a seeded sample of both request kinds: a
    Poisson burst (20 k req/s for 30 ms: ~180 welch requests, ~420 stream chunks over 8 of the
    streams, so every sampled stream gets tens of chunks) run through the server in the mix.
    welch: scipy.signal.welch on the request upcast to float64; stream chunks: the frames of
    every chunk of a stream, in order, against scipy.signal.stft(concat(stream chunks),
    boundary=None, padded=False) in float64."""
    import scipy.signal as sps
    import torch

    from mlx_signal_b200 import serving as sv

    srv = sv.SpectralServer(hbm_budget=4 << 30, max_batch=1024, slots=3, keep_results=True)
    sched = sv.poisson_schedule(20000.0, 0.03, pool, seed=seed, n_streams=8)
    rids = [srv.submit_welch(x, nperseg=p["nperseg"]) if k == sv.KIND_WELCH
            else srv.submit_chunk(p["stream"], x) for _, k, x, p in sched]
    srv.drain()
    torch.cuda.synchronize()
    welch_rel = welch_norm = 0.0
    nwelch = 0
    chunks: dict[int, list] = {}
    for rid, (_, k, x, p) in zip(rids, sched):
        if k == sv.KIND_WELCH:
            if nwelch >= 40:
                continue
            nwelch += 1
            got = srv.result(rid).double().cpu().numpy()
            _, ref = sps.welch(x.double().cpu().numpy(), nperseg=p["nperseg"])
            nseg = (x.shape[-1] - p["nperseg"]) // (p["nperseg"] // 2) + 1
            welch_norm = max(welch_norm, float(np.max(np.abs(got - ref)) / np.max(np.abs(ref))))
            if nseg >= 8:  # single low-power bins of fewer segments carry FFT rounding
                welch_rel = max(welch_rel, rel_err_bins(got, ref))
        else:
            chunks.setdefault(p["stream"], []).append((rid, x))
    frame_norm = frame_rel = 0.0
    nframes = 0
    for st, items in chunks.items():
        u = torch.cat([x for _, x in items]).double().cpu().numpy()
        _, _, zref = sps.stft(u, window="hann", nperseg=srv.sN, noverlap=srv.sN - srv.shop,
                              boundary=None, padded=False)
        for rid, _ in items:
            f0, z = srv.result(rid)
            z = z.cpu().numpy().astype(np.complex128)
            if z.shape[1] == 0:
                continue
            ref = zref[:, f0 : f0 + z.shape[1]]
            nframes += z.shape[1]
            frame_norm = max(frame_norm, float(np.max(np.abs(z - ref)) / np.max(np.abs(ref))))
            frame_rel = max(frame_rel, rel_err_bins(z.T, ref.T))
    del srv
    return {
        "welch_requests_checked": nwelch,
        "welch_max_rel_err_bins_nseg_ge_8": welch_rel,
        "welch_max_abs_err_rel_peak": welch_norm,
        "stream_frames_checked": nframes,
        "streams_checked": len(chunks),
        "stream_frames_max_abs_err_rel_peak": frame_norm,
        "stream_frames_max_rel_err_bins": frame_rel,
        "bars": "welch <= 1e-5 relative on bins above 1e-6 of the peak; single stft frames "
                "<= 2e-6 of the frame peak (norm-wise)",
        "pass": bool(welch_rel <= 1e-5 and frame_norm <= 2e-6),
    }


def serving_sweep(seconds, per_request_seconds=2.0, extra_rates=False, seed=21):
    """Config 5: open-loop Poisson arrivals at 1 k - 50 k req/s for `seconds` each (70%
    streaming-STFT chunks of 4096-65536 samples over 256 streams, nperseg 1024 / hop 256; 30%
    welch requests of 1-16 channels x 2^14-2^20 samples, nperseg 256 or 1024) through the
    continuous-batching server and, on the same schedule, through the plain per-request path.
    Inputs are resident device views of a 1 GiB pool. The plain path saturates near 7 k req/s,
    so above 5 k offered it is driven with the first `per_request_seconds` of the schedule (its
    throughput is capacity-bound either way)."""
    import torch

    from mlx_signal_b200 import serving as sv

    rates = [1000, 5000, 10000, 20000, 50000] + ([100000, 200000] if extra_rates else [])
    dev = torch.device("cuda", torch.cuda.current_device())
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    pool = torch.randn(1 << 28, generator=g, device=dev)
    out = {"arrival_seconds_per_rate": seconds, "hbm_budget_bytes": 4 << 30,
           "oracle_accuracy": serving_accuracy(pool, seed + 1)}
    for rate in rates:
        srv = sv.SpectralServer(hbm_budget=4 << 30, max_batch=1024, slots=3)
        sv.run_schedule(srv, sv.poisson_schedule(rate, 0.05, pool, seed=seed + 2))  # warm-up
        srv.stats = sv.ServerStats()
        sched = sv.poisson_schedule(float(rate), seconds, pool, seed=seed + rate)
        b = sv.run_schedule(srv, sched).summary()
        torch.cuda.synchronize()
        psched = sched if rate <= 5000 else sched[: int(rate * min(seconds, per_request_seconds))]
        p = sv.run_per_request(psched).summary()
        torch.cuda.synchronize()
        out[f"rate_{rate}"] = {
            "offered": len(sched),
            "per_request_driven_with": len(psched),
            "batched": {k: b[k] for k in ("req_per_s", "p50_ms", "p99_ms", "mean_batch",
                                          "batches", "peak_inflight_bytes")},
            "per_request": {k: p[k] for k in ("req_per_s", "p50_ms", "p99_ms")},
            "throughput_ratio": b["req_per_s"] / p["req_per_s"] if p["req_per_s"] else None,
        }
        del srv, sched, psched
    del pool
    torch.cuda.empty_cache()
    return out


def cpu_row_rate(fn_name, arrays, bytes_per_row, repeats=2, **kw):
    """The reference's CPU route (scipy.signal through oracle.cpu_reference) on a row sample over
    a spawn process pool of every host core: (GB/s of algorithmic bytes, cores, rows)."""
    from oracle import cpu_reference

    cores = os.cpu_count() or 1
    rows = arrays[0].shape[0]
    cpu_reference.pool_map_rows(fn_name, tuple(a[: min(rows, cores)] for a in arrays), cores, **kw)
    times = []
    for _ in range(repeats):
        t0 = time.perf_counter()
        cpu_reference.pool_map_rows(fn_name, arrays, cores, **kw)
        times.append(time.perf_counter() - t0)
    return bytes_per_row * rows / statistics.median(times) / 1e9, cores, rows


def with_cpu(entry, rate):
    gbs, cores, rows = rate
    entry["cpu_baseline"] = {"GB/s": gbs, "cores": cores, "kind": "port",
                             "sample": f"{rows} of {C} channels, scipy.signal on float32 "
                                       f"over a {cores}-process pool"}
    entry["speedup_vs_cpu"] = entry["GB/s"] / gbs
    return entry


def secondary(x, steps, warmup, dist, clocks):
    """Cheaper side measurements of the other configs (device-resident inputs)."""
    import torch

    import mlx_signal_b200 as msig
    from mlx_signal_b200 import _kernels

    out = {}
    peak, _ = measured_peak()
    win = torch.from_numpy(
        __import__("scipy.signal", fromlist=["get_window"]).get_window("hann", NPERSEG).astype(
            np.float32)).cuda()
    scale = 1.0 / (FS * float((win.double() ** 2).sum()))
    win_s = (win.double() * math.sqrt(scale)).float()
    x3, y, shifts = make_pair(7, x.device)
    k = max(3, min(steps, 20))
    # hann + constant detrend: the public csd / coherence apply the detrend as a spectral
    # correction (the window's low-bin DFT), as the calls below do
    lo_s = _kernels.window_low_spectrum(win_s.cpu().numpy(), NPERSEG)
    wd_s = torch.from_numpy(lo_s[0]).to(x.device) if lo_s is not None else None
    lo_r = _kernels.window_low_spectrum(win.cpu().numpy(), NPERSEG)
    wd_r = torch.from_numpy(lo_r[0]).to(x.device) if lo_r is not None else None
    ms = timed(lambda: _kernels.cross_mean("csd", x3, y, win_s, NPERSEG, NPERSEG, HOP, 1, True,
                                           wdft=wd_s),
               k, warmup, dist, clocks)
    b = 2 * C * NSAMP * 4 + C * NBINS * 8
    out["csd_64x2p20"] = {"ms": ms, "GB/s": b / ms / 1e6, "frac_hbm": b / ms / 1e6 / peak}
    ms = timed(lambda: _kernels.cross_mean("coherence", x3, y, win, NPERSEG, NPERSEG, HOP, 1,
                                           wdft=wd_r),
               k, warmup, dist, clocks)
    b = 2 * C * NSAMP * 4 + C * NBINS * 4
    out["coherence_64x2p20"] = {"ms": ms, "GB/s": b / ms / 1e6, "frac_hbm": b / ms / 1e6 / peak}
    coh = _kernels.cross_mean("coherence", x3, y, win, NPERSEG, NPERSEG, HOP, 1, wdft=wd_r)
    out["coherence_64x2p20"]["range"] = [float(coh.min()), float(coh.max())]
    out["csd_64x2p20"]["data"] = out["coherence_64x2p20"]["data"] = (
        "x ~ N(0,1); y = 0.7 roll(x, s_c) + 0.3 N(0,1), s_c seeded in [0, 64] per channel")
    del coh
    nseg = (NSAMP - NPERSEG) // HOP + 1
    # hann + constant detrend: the public spectrogram applies the detrend as a spectral correction
    low = _kernels.window_low_spectrum(win_s.cpu().numpy(), NPERSEG)
    wd = torch.from_numpy(low[0]).to(x.device) if low is not None else None
    ms = timed(lambda: _kernels.frames("power", x, win_s, NPERSEG, NPERSEG, HOP, 1, True,
                                       wdft=wd),
               k, warmup, dist, clocks)
    b = C * NSAMP * 4 + C * nseg * NBINS * 4
    out["spectrogram_psd_64x2p20"] = {"ms": ms, "GB/s": b / ms / 1e6,
                                      "frac_hbm": b / ms / 1e6 / peak}
    wsp = (win.double() / float(win.double().sum())).float()
    ms = timed(lambda: _kernels.frames("stft", x, wsp, NPERSEG, NPERSEG, HOP, 0, True,
                                       ext=NPERSEG // 2, ext_mode="zeros",
                                       n_total=NSAMP + NPERSEG),
               k, warmup, dist, clocks)
    nseg_s = (NSAMP + NPERSEG - NPERSEG) // HOP + 1
    b = C * NSAMP * 4 + C * nseg_s * NBINS * 8
    out["stft_64x2p20"] = {"ms": ms, "GB/s": b / ms / 1e6, "frac_hbm": b / ms / 1e6 / peak}
    # istft of that stft (fused inverse FFT + overlap-add + normalisation), round-trip error
    z = _kernels.frames("stft", x, wsp, NPERSEG, NPERSEG, HOP, 0, True, ext=NPERSEG // 2,
                        ext_mode="zeros", n_total=NSAMP + NPERSEG)
    wsum = float(win.double().sum())
    ms = timed(lambda: _kernels.istft_fused(z, win, wsum, NPERSEG, HOP), k, warmup, dist, clocks)
    xr = _kernels.istft_fused(z, win, wsum, NPERSEG, HOP)[:, NPERSEG // 2 : NPERSEG // 2 + NSAMP]
    rt = float((xr - x).abs().max() / x.abs().max())
    b = C * nseg_s * NBINS * 8 + C * NSAMP * 4
    out["istft_64x2p20"] = {"ms": ms, "GB/s": b / ms / 1e6, "frac_hbm": b / ms / 1e6 / peak,
                            "roundtrip_max_err_rel_peak": rt}
    # the reference's CPU route on a channel sample, beside each GPU figure (rank 0, N = 1)
    if dist is None:
        ncpu = min(C, os.cpu_count() or 1)
        xs = x[:ncpu].cpu().numpy()
        x3s = x3[:ncpu].cpu().numpy()
        ys = y[:ncpu].cpu().numpy()
        kw = dict(fs=FS, nperseg=NPERSEG, noverlap=NOVERLAP)
        with_cpu(out["csd_64x2p20"], cpu_row_rate("csd", (x3s, ys), 2 * NSAMP * 4 + NBINS * 8,
                                                  **kw))
        with_cpu(out["coherence_64x2p20"],
                 cpu_row_rate("coherence", (x3s, ys), 2 * NSAMP * 4 + NBINS * 4, **kw))
        with_cpu(out["spectrogram_psd_64x2p20"],
                 cpu_row_rate("spectrogram", (xs,), NSAMP * 4 + nseg * NBINS * 4,
                              window="hann", **kw))
        with_cpu(out["stft_64x2p20"],
                 cpu_row_rate("stft", (xs,), NSAMP * 4 + nseg_s * NBINS * 8, window="hann", **kw))
        zs = z[:ncpu].transpose(1, 2).contiguous().cpu().numpy()  # (rows, nfreq, nseg)
        with_cpu(out["istft_64x2p20"],
                 cpu_row_rate("istft", (zs,), nseg_s * NBINS * 8 + NSAMP * 4, window="hann", **kw))
        from oracle import cpu_reference

        cpu_reference.close_pool()
    del x3, y, z, xr
    out["general_shapes"] = general_shapes(x, dist, clocks, peak)
    out["batched_512_uneven"] = batched_uneven(dist, clocks, peak)
    out["rfft_1x2p23"] = large_rfft(dist, clocks, peak)
    out["rfft_irfft_3x2p22"] = odd_factor_rfft(dist, clocks, peak)
    out["tc_dft32_stage"] = tc_dft32_stage(dist, clocks)
    out["fft_consumers"] = fft_consumers(dist, clocks, peak)
    out["reference_published_rows"] = published_rows(dist, clocks)
    return out


def general_shapes(x, dist, clocks, peak):
    """welch and stft on the 64 x 2^20 input with a non-power-of-two nperseg (1000): fused
    Bluestein kernels; the composed path (strided frames + cuFFT) timed beside them, and the
    accuracy against float64 scipy on two channels."""
    import torch
    import scipy.signal as sps

    import mlx_signal_b200 as msig

    res = {}
    nps = 1000
    b = C * NSAMP * 4 + C * (nps // 2 + 1) * 4
    ms = timed(lambda: msig.welch(x, fs=FS, nperseg=nps), 10, 3, dist, clocks)
    # the same call on the composed path (what non-power-of-two shapes cost without the kernels)
    win = torch.from_numpy(sps.get_window("hann", nps).astype(np.float32)).to(x.device)

    def composed():
        fr = x.unfold(-1, nps, nps // 2)
        fr = (fr - fr.mean(dim=-1, keepdim=True)) * win
        return torch.fft.rfft(fr, dim=-1).abs().square().mean(dim=-2)

    ms_c = timed(composed, 5, 2, dist, clocks)
    res["welch_64x2p20_n1000"] = {"ms": ms, "GB/s": b / ms / 1e6, "frac_hbm": b / ms / 1e6 / peak,
                                  "composed_cufft_ms": ms_c,
                                  "kernel": "k_blue_welch<11> (M = 2048 chirp-z)"}
    x16 = x[:16]
    nf = (NSAMP + nps - nps) // (nps // 2) + 1
    bs = 16 * NSAMP * 4 + 16 * nf * (nps // 2 + 1) * 8
    ms = timed(lambda: msig.stft(x16, fs=FS, nperseg=nps), 10, 3, dist, clocks)
    res["stft_16x2p20_n1000"] = {"ms": ms, "GB/s": bs / ms / 1e6, "frac_hbm": bs / ms / 1e6 / peak}
    if dist is None:
        xs = x[:2].cpu().numpy().astype(np.float64)
        _, p_ref = sps.welch(xs, fs=FS, nperseg=nps)
        _, p = msig.welch(x[:2], fs=FS, nperseg=nps)
        p = p.cpu().numpy()
        m = p_ref > 1e-6 * p_ref.max(axis=-1, keepdims=True)
        res["welch_64x2p20_n1000"]["max_rel_err"] = float(np.max(np.abs(p - p_ref)[m] / p_ref[m]))
    return res


#: the reference's published device times for this path (Apple M4 Max, MLX 0.32.2, float32;
#: median of 9 after 3 warm-ups): (label, ms)
PUBLISHED_ROWS = {
    "welch_1x2p22_n4096": 0.65,
    "welch_256x2p16_n256": 0.98,
    "csd_64x2p20_n1024": 7.68,
    "coherence_64x2p20_n1024": 8.40,
    "spectrogram_16x2p20_n1024": 1.31,
    "stft_16x2p20_n1024": 1.25,
    "istft_16x2p20_n1024": 1.50,
}


def published_rows(dist, clocks, seed=13):
    """Our time on each shape the reference publishes a device time for, through the public API
    with device-resident float32 input (host argument handling included, as in the reference's
    'device' column; 'ms_graph_replay' is the same launch sequence replayed as a CUDA graph, i.e.
    the device time alone), and the small welch (1 x 2^16, nperseg 256): public API, and a
    CUDA-graph replay of the same launch sequence."""
    import torch

    import mlx_signal_b200 as msig
    from mlx_signal_b200 import graphs

    dev = torch.device("cuda", torch.cuda.current_device())
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    big = torch.randn((64, 1 << 20), generator=g, device=dev)
    y = torch.randn((64, 1 << 20), generator=g, device=dev)
    x16 = big[:16]
    w4096 = torch.randn((1, 1 << 22), generator=g, device=dev)
    w256 = torch.randn((256, 1 << 16), generator=g, device=dev)
    _, _, z16 = msig.stft(x16, nperseg=1024)
    calls = {
        "welch_1x2p22_n4096": lambda: msig.welch(w4096, nperseg=4096),
        "welch_256x2p16_n256": lambda: msig.welch(w256, nperseg=256),
        "csd_64x2p20_n1024": lambda: msig.csd(big, y, nperseg=1024),
        "coherence_64x2p20_n1024": lambda: msig.coherence(big, y, nperseg=1024),
        "spectrogram_16x2p20_n1024": lambda: msig.spectrogram(x16, nperseg=1024, noverlap=512,
                                                              window="hann"),
        "stft_16x2p20_n1024": lambda: msig.stft(x16, nperseg=1024),
        "istft_16x2p20_n1024": lambda: msig.istft(z16, nperseg=1024),
    }
    res = {}
    for name, fn in calls.items():
        ms = timed(fn, 20, 3, dist, clocks)
        # the same call's launch sequence captured once and replayed: its device time alone
        try:
            replay = graphs.GraphedCall(fn)
            ms_dev = timed(replay, 20, 3, dist, clocks)
            del replay
        except RuntimeError as e:  # reported, not fatal: the public-API number stands alone
            torch.cuda.synchronize()
            ms_dev = f"capture failed: {str(e).splitlines()[0][:120]}"
        res[name] = {"ms": ms, "ms_graph_replay": ms_dev,
                     "reference_device_ms_m4max": PUBLISHED_ROWS[name],
                     "speedup_vs_reference_published": PUBLISHED_ROWS[name] / ms}
    # small welch (config 1): 1 x 2^16 N(0,1) + a unit sinusoid at 0.1 fs, fs = 1, nperseg 256
    # (launch-bound)
    x1 = torch.randn((1, 1 << 16), generator=g, device=dev)
    x1 += torch.sin(2.0 * math.pi * 0.1 * torch.arange(1 << 16, device=dev,
                                                        dtype=torch.float64)).float()
    ms_api = timed(lambda: msig.welch(x1, fs=1.0, nperseg=256), 50, 5, dist, clocks)
    _, call = graphs.graphed_welch(x1, fs=1.0, nperseg=256)
    ms_graph = timed(lambda: call(x1), 50, 5, dist, clocks)
    res["small_welch_1x2p16_n256"] ={"ms_public_api": ms_api, "ms_cuda_graph_replay": ms_graph,
                                        "alg_bytes": (1 << 16) * 4 + 129 * 4,
                                        "note": "launch-bound: microseconds, not roofline"}
    return res


def fft_consumers(dist, clocks, peak, seed=9):
    """The long-FFT consumers on power-of-two sizes the three-pass kernels take, each against
    scipy (float64 result, one host call) on the same float32 input."""
    import torch
    import scipy.signal as sps

    import mlx_signal_b200 as msig

    dev = torch.device("cuda", torch.cuda.current_device())
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    n = 1 << 22
    x = torch.randn(n, generator=g, device=dev)
    y = torch.randn(n, generator=g, device=dev)
    h = torch.randn(1025, generator=g, device=dev)
    xh, yh, hh = x.cpu().numpy(), y.cpu().numpy(), h.cpu().numpy()
    cases = {
        "hilbert_2p23": (lambda: msig.hilbert(torch.cat([x, y])),
                         lambda: sps.hilbert(np.concatenate([xh, yh])), (1 << 23) * 12),
        "fftconvolve_2p22_x_2p22": (lambda: msig.fftconvolve(x, y),
                                    lambda: sps.fftconvolve(xh, yh), 2 * n * 4 + (2 * n - 1) * 4),
        "oaconvolve_2p22_x_1025": (lambda: msig.oaconvolve(x, h),
                                   lambda: sps.oaconvolve(xh, hh), n * 4 + 1025 * 4 + (n + 1024) * 4),
        "resample_2p22_to_3x2p20": (lambda: msig.resample(x, 3 << 20),
                                    lambda: sps.resample(xh, 3 << 20), n * 4 + (3 << 20) * 4),
    }
    res = {}
    for name, (gpu, cpu, nbytes) in cases.items():
        ms = timed(gpu, 10, 2, dist, clocks)
        res[name] = {"ms": ms, "GB/s": nbytes / ms / 1e6, "frac_hbm": nbytes / ms / 1e6 / peak}
        if dist is not None:  # host-side checks and baselines at N = 1 only
            continue
        got = gpu()
        ref = cpu()
        err = float(np.max(np.abs(got.cpu().numpy() - ref)) / np.max(np.abs(ref)))
        t = []
        for _ in range(2):
            t0 = time.perf_counter()
            cpu()
            t.append(time.perf_counter() - t0)
        cpu_gbs = nbytes / min(t) / 1e9
        res[name].update({"max_abs_err_rel_peak_vs_scipy_f64": err,
                          "cpu_baseline": {"GB/s": cpu_gbs, "cores": 1, "kind": "port",
                                           "sample": "the full transform, one scipy call"},
                          "speedup_vs_cpu": nbytes / ms / 1e6 / cpu_gbs})
    return res


def batched_uneven(dist, clocks, peak, nreq=512, seed=11):
    """512 independent welch requests (channels ~ U{1..64}, length 2^U(12, 22), nperseg uniform
    in {256, 1024, 4096}, noverlap = nperseg/2, N(0,1) float32, generated on the device) in ONE
    persistent launch, against the plain per-request path (one `welch` call each)."""
    import torch
    import scipy.signal as sps

    import mlx_signal_b200 as msig
    from mlx_signal_b200 import _lib, batch as mb

    dev = torch.device("cuda", torch.cuda.current_device())
    rs = np.random.default_rng(seed)
    shapes = []
    for _ in range(nreq):
        ch = int(rs.integers(1, 65))
        N = int(rs.choice([256, 1024, 4096]))
        n = max(int(2 ** rs.uniform(12, 22)), N)
        shapes.append((ch, n, N))
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    xs = [torch.randn((ch, n), generator=g, device=dev) for ch, n, _ in shapes]
    in_bytes = sum(ch * n * 4 for ch, n, _ in shapes)
    out_bytes = sum(ch * (N // 2 + 1) * 4 for ch, _, N in shapes)
    jobs = [mb.prepare_welch(x, nperseg=N) for x, (_, _, N) in zip(xs, shapes)]
    reqs = [j.req for j in jobs]
    lib = _lib.load()
    d, w = mb.plan(reqs)
    addr, count, _owner = mb._as_array(reqs)
    ws = torch.zeros(w, dtype=torch.uint8, device=dev)
    host = torch.empty(d, dtype=torch.uint8, pin_memory=True)
    _lib.check(lib.sp_batch_encode(addr, count, ws.data_ptr(), ws.numel(), host.data_ptr(),
                                   host.numel()), "sp_batch_encode")
    desc = host.to(dev)

    def run_batch():
        _lib.check(lib.sp_batch_run(desc.data_ptr(), ws.data_ptr(), 0,
                                    torch.cuda.current_stream().cuda_stream), "sp_batch_run")

    ms_b = timed(run_batch, 5, 2, dist, clocks)
    plain = {}

    def run_plain():
        for i, (x, (_, _, N)) in enumerate(zip(xs, shapes)):
            plain[i] = msig.welch(x, nperseg=N)[1]

    ms_p = timed(run_plain, 3, 1, dist, clocks)
    # accuracy. Per request: max relative error on bins above 1e-6 of each row's peak (requests
    # averaging >= 8 segments; with fewer, single low-power bins carry float32 FFT rounding
    # beyond 1e-5) and, for every request, max |error| / max |reference|.
    def errs(got, ref, nseg):
        g = got.double()
        r = ref.double()
        keep = r.abs() > 1e-6 * r.abs().amax(dim=-1, keepdim=True)
        rel = float(((g - r).abs()[keep] / r.abs()[keep]).max()) if nseg >= 8 else 0.0
        return rel, float((g - r).abs().max() / r.abs().max())

    nseg_of = [(n - N) // (N // 2) + 1 for _, n, N in shapes]
    rel_single = norm_single = 0.0
    for i, j in enumerate(jobs):
        a, b2 = errs(j.out, plain[i], nseg_of[i])
        rel_single, norm_single = max(rel_single, a), max(norm_single, b2)
    rel_scipy = norm_scipy = 0.0
    idx = sorted(range(nreq), key=lambda k: shapes[k][0] * shapes[k][1])
    pick = idx[:4] + [k for k in idx if nseg_of[k] >= 8][:4]
    for i in (pick if dist is None else []):  # host scipy checks at N = 1 only
        _, pref = sps.welch(xs[i].double().cpu().numpy(), nperseg=shapes[i][2])
        a, b2 = errs(jobs[i].out.cpu(), torch.from_numpy(pref), nseg_of[i])
        rel_scipy, norm_scipy = max(rel_scipy, a), max(norm_scipy, b2)
    gbs = (in_bytes + out_bytes) / ms_b / 1e6
    res = {
        "requests": nreq,
        "input_GB": in_bytes / 1e9,
        "ms_batched": ms_b,
        "GB/s": gbs,
        "frac_hbm": gbs / peak,
        "req_per_s_batched": nreq / ms_b * 1e3,
        "ms_per_request_plain": ms_p,
        "req_per_s_plain": nreq / ms_p * 1e3,
        "speedup_vs_plain": ms_p / ms_b,
        "vs_single_request_path": {"max_rel_err_bins_nseg_ge_8": rel_single,
                                   "max_abs_err_rel_peak_all": norm_single},
        "vs_scipy_f64_8_requests": {"max_rel_err_bins_nseg_ge_8": rel_scipy,
                                    "max_abs_err_rel_peak_all": norm_scipy},
        "segments_per_request": {"min": int(min(nseg_of)), "median": int(np.median(nseg_of)),
                                 "max": int(max(nseg_of))},
        "launches_per_batch": 2,  # the 4096 class, then the other classes as its dependent
        "grid": int(lib.sp_batch_max_grid()),
    }
    del xs, jobs, ws, desc, plain
    torch.cuda.empty_cache()
    return res


def tc_dft32_stage(dist, clocks, seed=17):
    """The radix-32 DFT stage on the tensor cores (sp_dft32_tc_c64: FP16 head/tail splits, three
    products, FP32 accumulation) on the vector count of one radix-32 pass of the 64 x 2^20 welch
    (65,504 pair transforms x 32 columns): its tensor-core rate with the operands staged (the MMA
    chain repeated 16 times) and end to end, its error against float64 numpy, and what one pass
    costs at that rate beside the whole CUDA-core welch."""
    import torch

    from mlx_signal_b200 import _kernels

    dev = torch.device("cuda", torch.cuda.current_device())
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    nvec = 65504 * 32
    z = torch.complex(torch.randn(nvec, 32, generator=g, device=dev),
                      torch.randn(nvec, 32, generator=g, device=dev))
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    res = {"vectors": nvec, "mma": "tcgen05 kind::f16 M128 N64 K192 (3 split products)"}
    for reps in (1, 16):
        ms = timed(lambda: _kernels.dft32_tc(z, reps=reps, err=err), 10, 3, dist, clocks)
        res[f"reps{reps}_ms"] = ms
        res[f"reps{reps}_tc_tflops_issued"] = nvec * 2 * 64 * 192 * reps / ms / 1e9
    res["tc_time_per_pass_ms"] = res["reps16_ms"] / 16
    res["error_word"] = int(err.item())
    if dist is None:
        y = _kernels.dft32_tc(z[:8192])
        ref = np.fft.fft(z[:8192].cpu().numpy().astype(np.complex128), axis=-1)
        e = np.abs(y.cpu().numpy() - ref).max(axis=-1) / np.abs(ref).max(axis=-1)
        res["max_err_rel_peak_vs_numpy_f64"] = float(e.max())
        res["median_err_rel_peak_vs_numpy_f64"] = float(np.median(e))
    del z
    return res


def large_rfft(dist, clocks, peak, log_n=23, seed=5):
    """1 x 2^23 float32 N(0,1) real FFT through the three-pass path, against numpy float64."""
    import torch

    from mlx_signal_b200 import _lib

    n = 1 << log_n
    dev = torch.device("cuda", torch.cuda.current_device())
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    x = torch.randn(n, generator=g, device=dev)
    X = torch.empty(n // 2 + 1, dtype=torch.complex64, device=dev)
    lib = _lib.load()
    ws = torch.empty(int(lib.sp_fft_workspace_size(n // 2, 1)), dtype=torch.uint8, device=dev)

    def step():
        _lib.check(lib.sp_rfft_c64(x.data_ptr(), X.data_ptr(), 1, n, n // 2 + 1, ws.data_ptr(),
                                   ws.numel(), torch.cuda.current_stream().cuda_stream),
                   "sp_rfft_c64")

    ms = timed(step, 20, 3, dist, clocks)
    b = n * 4 + (n // 2 + 1) * 8
    if dist is not None:  # host-side checks and baselines at N = 1 only
        return {"ms": ms, "GB/s": b / ms / 1e6, "frac_hbm": b / ms / 1e6 / peak, "launches": 4}
    ms_cufft = timed(lambda: torch.fft.rfft(x), 20, 3, dist, clocks)
    xh = x.cpu().numpy()
    ref = np.fft.rfft(xh.astype(np.float64))
    err = float(np.max(np.abs(X.cpu().numpy() - ref)) / np.max(np.abs(ref)))
    t_cpu = []
    for _ in range(3):  # numpy.fft.rfft on float32, one transform on one core
        t0 = time.perf_counter()
        np.fft.rfft(xh)
        t_cpu.append(time.perf_counter() - t0)
    cpu = b / statistics.median(t_cpu) / 1e9
    return {"ms": ms, "GB/s": b / ms / 1e6, "frac_hbm": b / ms / 1e6 / peak,
            "max_abs_err_rel_peak_vs_numpy_f64": err, "launches": 4,
            "cufft_ms": ms_cufft, "speedup_vs_cufft": ms_cufft / ms,
            "cpu_baseline": {"GB/s": cpu, "cores": 1, "kind": "port",
                             "sample": "the full 2^23 transform, numpy.fft.rfft"},
            "speedup_vs_cpu": b / ms / 1e6 / cpu}


def odd_factor_rfft(dist, clocks, peak, n=3 << 22, seed=6):
    """Real transforms of an odd-factor length (n = 3 2^22: three decimated branches of packed
    2^21-point transforms around one radix-3 kernel on each side) through the C-ABI, against
    cuFFT (torch.fft) on the same device input and float64 numpy. The public API routes the
    inverse here and the forward to cuFFT (faster at every measured odd-factor size)."""
    import torch

    from mlx_signal_b200 import _lib

    dev = torch.device("cuda", torch.cuda.current_device())
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    x = torch.randn(n, generator=g, device=dev)
    X = torch.empty(n // 2 + 1, dtype=torch.complex64, device=dev)
    y = torch.empty(n, device=dev)
    lib = _lib.load()
    ws = torch.empty(int(lib.sp_fft_workspace_size(n // 2, 1)), dtype=torch.uint8, device=dev)

    def fwd():
        _lib.check(lib.sp_rfft_c64(x.data_ptr(), X.data_ptr(), 1, n, n // 2 + 1, ws.data_ptr(),
                                   ws.numel(), torch.cuda.current_stream().cuda_stream), "rfft")

    def inv():
        _lib.check(lib.sp_irfft_f32(X.data_ptr(), n // 2 + 1, n // 2 + 1, y.data_ptr(), 1, n,
                                    ws.data_ptr(), ws.numel(),
                                    torch.cuda.current_stream().cuda_stream), "irfft")

    fwd()
    Xc = X.clone()
    b = n * 4 + (n // 2 + 1) * 8
    res = {"n": n}
    for name, ours, libf in (("rfft", fwd, lambda: torch.fft.rfft(x)),
                             ("irfft", inv, lambda: torch.fft.irfft(Xc, n=n))):
        ms = timed(ours, 20, 3, dist, clocks)
        ms_lib = timed(libf, 20, 3, dist, clocks)
        res[name] = {"ms": ms, "GB/s": b / ms / 1e6, "frac_hbm": b / ms / 1e6 / peak,
                     "cufft_ms": ms_lib, "speedup_vs_cufft": ms_lib / ms}
    if dist is None:
        fwd()
        inv()
        xh = x.cpu().numpy().astype(np.float64)
        ref = np.fft.rfft(xh)
        res["rfft"]["max_abs_err_rel_peak_vs_numpy_f64"] = float(
            np.max(np.abs(X.cpu().numpy() - ref)) / np.max(np.abs(ref)))
        ref_b = np.fft.irfft(X.cpu().numpy().astype(np.complex128), n=n)
        res["irfft"]["max_abs_err_rel_peak_vs_numpy_f64"] = float(
            np.max(np.abs(y.cpu().numpy() - ref_b)) / np.max(np.abs(ref_b)))
    res["launches_per_call"] = 5
    return res


def summarize(sec: dict) -> dict:
    """A compact digest of the side measurements (rounded), printed as the line's last key."""
    def r(v, d=3):
        return None if v is None else float(f"{v:.{d}g}")

    out = {}
    sp = sec.get("serving_poisson")
    if sp:
        rows = {}
        for k, v in sp.items():
            if k.startswith("rate_"):
                b, p = v["batched"], v["per_request"]
                rows[k[5:]] = [r(b["req_per_s"]), r(b["p50_ms"]), r(b["p99_ms"]),
                               r(p["req_per_s"]), r(p["p99_ms"]), r(v["throughput_ratio"])]
        out["serving"] = {"window_s": sp["arrival_seconds_per_rate"],
                          "cols": "batched req/s, p50 ms, p99 ms | per-request req/s, p99 ms | "
                                  "ratio", "rates": rows}
        acc = sp["oracle_accuracy"]
        out["serving_vs_f64_oracle"] = {
            "welch_rel": r(acc["welch_max_rel_err_bins_nseg_ge_8"]),
            "frames_norm": r(acc["stream_frames_max_abs_err_rel_peak"]),
            "n": [acc["welch_requests_checked"], acc["stream_frames_checked"]],
            "pass": acc["pass"]}
    ms = {}
    for k in ("csd_64x2p20", "coherence_64x2p20", "spectrogram_psd_64x2p20", "stft_64x2p20",
              "istft_64x2p20"):
        if k in sec:
            ms[k.replace("_64x2p20", "")] = [r(sec[k]["ms"] * 1e3), r(sec[k]["frac_hbm"])]
    if "batched_512_uneven" in sec:
        bu = sec["batched_512_uneven"]
        ms["batch512"] = [r(bu["ms_batched"] * 1e3), r(bu["frac_hbm"]), r(bu["speedup_vs_plain"])]
    if "rfft_1x2p23" in sec:
        rf = sec["rfft_1x2p23"]
        ms["rfft_2p23"] = [r(rf["ms"] * 1e3), r(rf["frac_hbm"])]
        if "cufft_ms" in rf:
            ms["rfft_2p23"].append(r(rf["speedup_vs_cufft"]))
    if "rfft_irfft_3x2p22" in sec:
        mx = sec["rfft_irfft_3x2p22"]
        for k in ("rfft", "irfft"):
            ms[k + "_3x2p22"] = [r(mx[k]["ms"] * 1e3), r(mx[k]["frac_hbm"]),
                                 r(mx[k]["speedup_vs_cufft"])]
    out["us_and_frac_hbm"] = ms
    if "tc_dft32_stage" in sec:
        tc = sec["tc_dft32_stage"]
        out["tc_dft32_pass"] = {"us": r(tc["tc_time_per_pass_ms"] * 1e3),
                                "tflops": r(tc["reps16_tc_tflops_issued"]),
                                "err": r(tc.get("max_err_rel_peak_vs_numpy_f64"))}
    return out


def run_ours(args, rank, world, local_rank, dist):
    import torch

    import mlx_signal_b200 as msig
    from mlx_signal_b200 import _kernels

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    clocks = ClockSampler(local_rank)
    x = make_input(args.seed + rank, dev)
    torch.cuda.synchronize()

    # accuracy gate on all 64 channels against the float64 oracle (scipy.signal.welch on the
    # input upcast to float64, fanned out over the host cores): max relative error <= 1e-5 on
    # bins above 1e-6 of each row's peak, for the public call here and for the output of the
    # timed launcher step after the timed region
    from oracle import cpu_reference

    f, p = msig.welch(x, fs=FS, nperseg=NPERSEG, noverlap=NOVERLAP)
    pref = cpu_reference.pool_map_rows("welch_f64", (x.cpu().numpy(),), os.cpu_count() or 1,
                                       fs=FS, nperseg=NPERSEG, noverlap=NOVERLAP)
    max_rel = rel_err_bins(p.double().cpu().numpy(), pref)
    if max_rel > ACCURACY_BAR:  # a fast wrong answer is not a measurement
        raise RuntimeError(f"accuracy gate failed: max relative error {max_rel:.3e} on bins above "
                           f"1e-6 of the peak exceeds {ACCURACY_BAR:g}")

    # device-resident throughput through the C-ABI launcher
    win = msig.spectral.device_vector(
        (msig.windows._window_np("hann", NPERSEG)
         * math.sqrt(1.0 / (FS * float((msig.windows._window_np("hann", NPERSEG) ** 2).sum()))))
        .astype(np.float32))

    low = _kernels.window_low_spectrum(win.cpu().numpy(), NPERSEG)
    wdft = None if low is None else torch.from_numpy(low[0]).to(dev)

    last = {}

    def step():  # the same C-ABI entry mlx_signal_b200.welch uses for this shape
        last["p"] = _kernels.welch_mean(x, win, NPERSEG, NPERSEG, HOP, 1, True, wdft=wdft)

    ms = timed(step, args.steps, args.warmup, dist, clocks)
    step_rel = rel_err_bins(last["p"].double().cpu().numpy(), pref)
    if step_rel > ACCURACY_BAR:
        raise RuntimeError(f"accuracy gate failed on the timed step's output: max relative error "
                           f"{step_rel:.3e} exceeds {ACCURACY_BAR:g}")
    max_rel = max(max_rel, step_rel)
    value = world * ALG_BYTES / (ms * 1e-3) / 1e9
    launches = 2 * args.steps

    # end to end: pinned host input -> public API -> host PSD, every step
    x_host = torch.empty((C, NSAMP), dtype=torch.float32, pin_memory=True)
    x_host.copy_(x.cpu())
    res = {}

    def step_e2e():
        _, pp = msig.welch(x_host, fs=FS, nperseg=NPERSEG, noverlap=NOVERLAP)
        res["p"] = pp.cpu()

    ms_e2e = timed(step_e2e, args.steps, max(3, args.warmup), dist, clocks)
    e2e_value = world * ALG_BYTES / (ms_e2e * 1e-3) / 1e9
    launches += 2 * args.steps

    peak, peak_kind = measured_peak()
    achieved = ALG_BYTES / (ms * 1e-3) / 1e9
    sec = None
    if not args.no_secondary and world == 1:  # side measurements at N = 1 only
        sec = secondary(x, args.steps, 2, dist, clocks)
        if args.serving_seconds > 0:
            sec["serving_poisson"] = serving_sweep(args.serving_seconds,
                                                   args.serving_per_request_seconds,
                                                   args.serving_extra_rates)
    clk = clocks.summary()

    cpu = None
    if rank == 0 and world == 1:
        rate, cores, secs = cpu_welch_rate(x.cpu().numpy(), C, 3)
        from oracle import cpu_reference

        cpu_reference.close_pool()
        cpu = {"value": rate, "unit": "GB/s", "cores": cores, "kind": "port",
               "sample": f"all {C} channels x 2^20, median of 3 ({secs:.2f} s each); "
                         f"scipy.signal.welch on float32 (the reference's CPU route, "
                         f"spectral.py:433-450) over a {cores}-process pool split by channel"}
    if rank == 0:
        line = {
            "metric": METRIC,
            "value": value,
            "unit": "GB/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": value / world / (ALG_BYTES / (PUBLISHED_DEVICE_MS * 1e-3) / 1e9),
            "dtype": "f32",
            "data": "synthetic (seeded N(0,1) + 1-4 sinusoids per channel, generated on device)",
            "config": config_dict(world),
            "max_rel_err": max_rel,
            "roofline": {
                "bound": "hbm",
                "kernel": "k_welch_half<nfft=1024, spectral detrend> + k_reduce_mean, launched as "
                          "programmatic dependents (one sp_welch_f32_ex call)",
                "achieved": achieved,
                "peak": peak,
                "peak_kind": peak_kind,
                "unit": "GB/s",
                "frac": achieved / peak,
                "traffic": traffic_from_profiles(),
                "alg_bytes_per_launch": ALG_BYTES,
            },
            "e2e": {
                "value": e2e_value,
                "unit": "GB/s",
                "ms_per_step": ms_e2e,
                "h2d_bytes_per_step": C * NSAMP * 4,
                "d2h_bytes_per_step": C * NBINS * 4,
                "api": "mlx_signal_b200.welch(pinned host tensor) -> .cpu()",
            },
            "gpu_launches": launches,
            "clocks": clk,
            "baseline_published": {"device_ms": PUBLISHED_DEVICE_MS, "hw": "Apple M4 Max"},
        }
        if cpu is not None:
            line["cpu_baseline"] = cpu
        if sec is not None:
            line["secondary"] = sec
            line["summary"] = summarize(sec)  # last key: stays in a truncated stdout tail
        print(json.dumps(line), flush=True)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as tdist

        torch.cuda.set_device(local_rank)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                 device_id=torch.device("cuda", local_rank))
        dist = tdist
    try:
        run_ours(args, rank, world, local_rank, dist)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
