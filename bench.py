#!/usr/bin/env python
"""Throughput benchmark of the teuk-kokkos RK4 hot path on B200.

Workload (one "step" = one classical RK4 step of every solve in a batch):
plain FP64 linear Kerr ringdown, a = 0.7, M = 1, L = 1, nr = 1025, SBP
D10-5, m = -4..4, ell <= 16 (ntheta = 25), seeded Gaussian pulses in
ell = 2, m = +-2 (centre 8M, width 0.8M, amplitude 1e-3) plus seeded
1e-6 band-projected noise, dt = 0.1 h (inside the measured RK4 stability
limit; the CFL 0.25 bound of the reference driver holds).  Each GPU advances
a batch of
``--batch`` such solves (weak scaling: per-GPU work fixed as N grows, no
collective on the data path).

  python bench.py [--gpus N --steps K --warmup W] [--impl b200|reference]

Prints one JSON line (rank 0).  ``value`` is whole-job grid-point updates/s
(steps * modes * nr * ntheta per solve, the reference's metric) from CUDA
events on the engine's stream, max over ranks; ``e2e`` is the same metric
through the C ABI with host buffers (initial-state upload from pinned host
memory and a per-step device->host read of every solve's endpoint waveform
inside the timed region).  ``--impl reference`` times the reference's own
CPU implementation (teuk-kokkos headers built against the Kokkos-API host
shim, all host threads) on the same workload, one RK4 step of one of its
solves per benchmark step, without mapping the engine library.

Beside the headline the line carries (rank 0, one GPU): ``split_precision``
(the same batch with split-precision transforms), ``uneven_batch`` (256
solves of uneven shape in one set of launches against the same solves one
at a time), ``serving`` (a Poisson stream of the serving mix through the
continuous-batching server, p50 / p99 time-to-waveform), ``second_order``
(the quadratic-source solve, FP64 and split precision) and the reference
build's rate on the host cores (``cpu_baseline``).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO / "teuk-kokkos_b200"))

METRIC = ("grid-point updates/s, p99 latency: batched split-prec vs plain "
          "FP64 @<=1e-9 err")
UNIT = "grid-point updates/s"
FALLBACK_HBM_GBS = 6650.0
PASSES_PER_STEP = 14  # compulsory modal passes of the fused stage schedule
SECOND_ORDER_BYTES_PER_POINT = 17 * 16 * 13  # 3,536 B per nodal point and step
L2_BYTES = 126 * 1024 * 1024


def parse_args():
    p = argparse.ArgumentParser(description=__doc__,
                                formatter_class=argparse.RawDescriptionHelpFormatter)
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=1000)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", choices=["b200", "reference"], default="b200")
    p.add_argument("--batch", type=int, default=64,
                   help="solves per GPU (default 64: 405 MB of state, > L2)")
    p.add_argument("--cpu-seconds", type=float, default=15.0,
                   help="target length of the CPU-baseline sample")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-serving", action="store_true")
    p.add_argument("--no-second-order", action="store_true")
    p.add_argument("--serve-requests", type=int, default=64,
                   help="requests of the continuous-batching measurement")
    p.add_argument("--serve-steps", type=int, default=100,
                   help="RK4 steps per serving request")
    p.add_argument("--no-uneven", action="store_true")
    p.add_argument("--no-split", action="store_true")
    p.add_argument("--so-steps", type=int, default=20,
                   help="timed RK4 steps of the quadratic-source solve")
    p.add_argument("--uneven-steps", type=int, default=20,
                   help="timed RK4 steps of the 256-solve uneven batch")
    return p.parse_args()


def workload_config(batch: int):
    from teuk_b200 import workloads as wl
    config, pulse, dt = wl.kerr_ringdown()
    return {
        "workload": "kerr_ringdown a=0.7 M=1 L=1 nr=1025 d10-5 m=-4..4 "
                    "ell<=16 ntheta=25 dt=0.1h (cfl<=0.25)",
        "solves_per_gpu": batch,
        "dt": dt,
        "dissipation": config.dissipation,
        "grid_points_per_solve": wl.grid_points(config),
        "storage": "band (modal) coefficients, complex128",
        "l2": f"inputs larger than L2: {batch} solves x "
              f"{wl.modal_values(config) * 16 / 1e6:.1f} MB state per buffer",
    }, config, pulse, dt


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """SM clock and clock-event reasons of one GPU during a timed region:
    read-only NVML queries every `period_s` from a thread, plus one sample
    when the sampler starts and one when it stops, so even a region of a
    few tens of milliseconds carries its own record.  Falls back to
    `nvidia-smi -lms 200` when NVML cannot be opened."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"),
               ("hw_power_brake", "nvmlClocksEventReasonHwPowerBrakeSlowdown"))
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,"
              "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_uuid: str | None, period_s: float = 0.01):
        self.samples = []  # (sm_mhz, sm_max_mhz, set of reason names)
        self.period = period_s
        self.proc = None
        self.nvml = None
        self.handle = None
        self._stop = threading.Event()
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nvml = pynvml
            if device_uuid:
                self.handle = pynvml.nvmlDeviceGetHandleByUUID(device_uuid)
            else:
                self.handle = pynvml.nvmlDeviceGetHandleByIndex(0)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(
                self.handle, pynvml.NVML_CLOCK_SM)
        except Exception:
            self.nvml = None
        if self.nvml is not None:
            self._sample()
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
            return
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}",
               "--format=csv,noheader,nounits", "-lms", "200"]
        if device_uuid:
            cmd += ["-i", device_uuid]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read_smi, daemon=True)
        self.thread.start()

    def _sample(self):
        nv = self.nvml
        try:
            sm = nv.nvmlDeviceGetClockInfo(self.handle, nv.NVML_CLOCK_SM)
            bits = nv.nvmlDeviceGetCurrentClocksEventReasons(self.handle)
        except Exception:
            return
        names = {name for name, const in self.REASONS
                 if bits & getattr(nv, const, 0)}
        self.samples.append((float(sm), float(self.max_mhz), names))

    def _poll(self):
        while not self._stop.wait(self.period):
            self._sample()

    def _read_smi(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9 or not parts[1].replace(".", "").isdigit():
                continue
            names = {n for n, flag in zip(("hw_slowdown", "hw_thermal_slowdown",
                                            "sw_thermal_slowdown", "sw_power_cap"),
                                           parts[5:9])
                     if flag.lower() == "active"}
            self.samples.append((float(parts[1]), float(parts[2]), names))

    def stop(self):
        if self.nvml is not None:
            self._stop.set()
            self.thread.join(timeout=2)
            self._sample()
            source = "nvml"
        elif self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.thread.join(timeout=2)
            source = "nvidia-smi"
        else:
            return {"sm_mhz": None, "sm_max_mhz": None,
                    "reasons": ["unsampled"], "samples": 0}
        sm = [x[0] for x in self.samples]
        reasons = set()
        for x in self.samples:
            reasons |= x[2]
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(x[1] for x in self.samples) if sm else None,
                "reasons": sorted(reasons), "samples": len(self.samples),
                "source": source}


def device_uuid(torch, device: int):
    try:
        uuid = str(torch.cuda.get_device_properties(device).uuid)
        return uuid if uuid.startswith("GPU-") else "GPU-" + uuid
    except Exception:
        return None


def measured_hbm_peak():
    path = REPO / "MEASURED_PEAKS.json"
    try:
        data = json.loads(path.read_text())
        return float(data["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def recorded_traffic(kernel: str, algorithmic_bytes_per_launch: float):
    """DRAM bytes per stage launch from the committed ncu summary of
    `kernel` (key=value lines: dram_bytes_per_launch,
    algorithmic_bytes_per_launch of the captured case, the benchmark's own
    64-solve size), scaled to this launch by the units processed."""
    path = REPO / "profiles" / f"{kernel}_kerr_ringdown64_traffic.txt"
    try:
        data = {}
        for line in path.read_text().splitlines():
            if "=" in line and not line.startswith("#"):
                k, v = line.split("=", 1)
                data[k.strip()] = float(v)
        per_unit = data["dram_bytes_per_launch"] / data["algorithmic_bytes_per_launch"]
        return per_unit * algorithmic_bytes_per_launch
    except Exception:
        return None


# ---------------------------------------------------------------- serving
def solve_alone_seconds(tb, config, pulse, dt, steps: int, stream):
    """Device seconds of `steps` RK4 steps of one solve alone (the plain
    FP64 one-solve-at-a-time path), CUDA events on its stream, after two
    untimed steps."""
    import torch

    p = tb.Pipeline(config)
    p.set_stream(stream.cuda_stream)
    p.initialize_gaussian(pulse)
    p.step(0.0, dt, 2)
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(stream)
    p.step(2 * dt, dt, steps)
    b.record(stream)
    b.synchronize()
    p.close()
    return a.elapsed_time(b) / 1e3


def one_at_a_time_rate(tb, wl, kinds, steps: int):
    """Plain FP64 path, one solve at a time: device grid-point updates/s of
    a representative solve of each request kind (CUDA events)."""
    import torch

    stream = torch.cuda.Stream()
    rates = {}
    for kind, (config, pulse, dt) in kinds.items():
        seconds = solve_alone_seconds(tb, config, pulse, dt, steps, stream)
        rates[kind] = steps * wl.grid_points(config) / seconds
    return rates


def serving_run(tb, wl, capacity: float, requests: int, steps: int,
                seed: int = 20260101, precision: int = 0):
    """Poisson stream of the serving mix through the continuous-batching
    server (transforms in `precision`) at ~80 % of its capacity, against the
    plain FP64 path one solve at a time; returns the 'serving' record."""
    import torch

    mix = wl.serving_mix(requests, seed)
    kinds = {}
    for kind, c, pulse, dt in mix:
        kinds.setdefault(kind, (c, pulse, dt))
    alone = one_at_a_time_rate(tb, wl, kinds, min(steps, 20))
    work = [steps * wl.grid_points(c) for _, c, _, _ in mix]
    # offered load: 80 % of the rate at which the batched server would
    # finish the mix, estimated from the batched linear rate and the
    # second-order solves' own rate
    seconds_needed = sum(w / (alone[k] if k == "second_order" else capacity)
                         for w, (k, *_r) in zip(work, mix))
    rate = 0.8 * len(mix) / seconds_needed
    rng = np.random.Generator(np.random.PCG64(seed + 1))
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=requests))
    arrivals -= arrivals[0]
    free, _ = torch.cuda.mem_get_info()
    budget = int(min(150e9, 0.8 * free))
    server = tb.Server(hbm_budget_bytes=budget, precision=precision)
    ids = []
    t0 = time.perf_counter()
    while True:
        now = time.perf_counter() - t0
        while len(ids) < requests and arrivals[len(ids)] <= now:
            _, c, pulse, dt = mix[len(ids)]
            ids.append(server.submit(c, pulse, dt, steps))
        st = server.stats()
        if st.active + st.queued == 0:
            if len(ids) == requests:
                break
            time.sleep(max(0.0, arrivals[len(ids)] - now))
            continue
        server.advance(4)
    makespan = time.perf_counter() - t0
    latencies = np.array([server.result(i)[1] for i in ids])
    by_kind = {}
    for (kind, *_r), lat in zip(mix, latencies):
        by_kind.setdefault(kind, []).append(lat)
    st = server.stats()
    alone_seconds = sum(w / alone[k] for w, (k, *_r) in zip(work, mix))
    server.close()
    device_rate = st.grid_point_updates / st.device_seconds
    counts = {k: len(v) for k, v in by_kind.items()}
    return {
        "precision": "split" if precision == tb.PRECISION_SPLIT else "fp64",
        "requests": requests,
        "mix": "40% schwarzschild a=0 nr=257 d8-4 ell<=8; 30% kerr_ringdown "
               "a=0.7 nr=1025 d10-5 ell<=16; 20% second_order a=0.9 nr=1025 "
               "ntheta=48 ell<=10/20 source on from t=0; 10% extremal a=0.99 "
               "nr=4097 ell<=24 ntheta=37 m=-4..4",
        "drawn": counts,
        "reduced_from": "4096 requests at each configuration's own step "
                        f"count; here {requests} requests x {steps} RK4 steps "
                        "so the run fits the benchmark's time budget",
        "steps_per_request": steps,
        "arrivals": f"Poisson, {rate:.2f}/s (80% of the estimated capacity)",
        "p50_time_to_waveform_s": float(np.percentile(latencies, 50)),
        "p99_time_to_waveform_s": float(np.percentile(latencies, 99)),
        "p50_p99_by_kind_s": {k: [float(np.percentile(v, 50)),
                                  float(np.percentile(v, 99))]
                              for k, v in by_kind.items()},
        "throughput": float(sum(work) / makespan),
        "device_throughput": float(device_rate),
        "one_at_a_time_device_throughput": float(sum(work) / alone_seconds),
        "one_at_a_time_by_kind": alone,
        "batched_vs_one_at_a_time": float(device_rate / (sum(work) / alone_seconds)),
        "unit": UNIT,
        "batched_steps": int(st.steps),
        "makespan_s": makespan,
        "rebuilds": int(st.rebuilds),
        "rebuild_host_s": float(st.rebuild_seconds),
    }


# ---------------------------------------------------------------- uneven batch
def uneven_batch_run(tb, wl, steps: int, options=None, label="fp64"):
    """The batched uneven-instance configuration: 256 first-order solves of
    uneven shape in one set of stage launches per RK4 step (graph replay),
    against the same solves one at a time."""
    import torch

    solves = wl.uneven_batch()
    configs = [c for c, _, _ in solves]
    batch = tb.Batch(configs, options or tb.LaunchOptions(autotune=True))
    stream = torch.cuda.Stream()
    batch.set_stream(stream.cuda_stream)
    for i, (_, pulse, _) in enumerate(solves):
        batch.initialize_gaussian(i, pulse)
    dts = [dt for _, _, dt in solves]
    batch.step(dts, steps=3, graph=True)
    batch.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(stream)
    batch.step(dts, steps=steps, graph=True)
    b.record(stream)
    b.synchronize()
    seconds = a.elapsed_time(b) / 1e3
    gp = sum(wl.grid_points(c) for c in configs)
    kernels = batch.stage_kernels()
    strips = batch.strip_rows()
    batch.close()
    alone = 0.0
    for c, pulse, dt in solves:
        alone += solve_alone_seconds(tb, c, pulse, dt, 3, stream) / 3
    return {
        "workload": "256 first-order solves: a U[0,0.95], nr from "
                    "{257,513,1025,2049}, ell_max U{8..20}, m=-2..2, d10-5, "
                    "Gaussian in ell=2 m=+-2 (centre U[6,14]M, width "
                    "U[0.5,1.5]M), dt=0.1h (cfl<=0.25); one seeded draw",
        "precision": label,
        "steps": steps, "reduced_from": "5000 RK4 steps per solve",
        "value": gp * steps / seconds, "unit": UNIT,
        "ms_per_step": 1e3 * seconds / steps,
        "one_at_a_time": gp / alone,
        "batched_vs_one_at_a_time": (gp * steps / seconds) / (gp / alone),
        "stage_kernel_groups": {"streaming": kernels[0], "tile": kernels[1]},
        "strip_rows": strips,
    }


# ---------------------------------------------------------------- second order
def second_order_rate(tb, wl, config, pulse, dt, steps: int, options=None):
    """Device grid-point updates/s of the quadratic-source solve (CUDA
    events on its stream, after two untimed steps)."""
    import torch

    p = tb.Pipeline(config, options)
    stream = torch.cuda.Stream()
    p.set_stream(stream.cuda_stream)
    p.initialize_gaussian(pulse)
    p.step(0.0, dt, 2)
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(stream)
    p.step(2 * dt, dt, steps)
    b.record(stream)
    b.synchronize()
    state = p.get_state()
    p.close()
    if not np.all(np.isfinite(state)):
        raise RuntimeError("second-order benchmark state is not finite")
    return steps * wl.grid_points(config) / (a.elapsed_time(b) / 1e3), state


def second_order_run(tb, wl, steps: int, cpu_steps: int):
    """The quadratic-source configuration (full 13-field stage graph with
    the source active) on the GPU, FP64 and split-precision transforms,
    beside the reference build on the host cores for a few steps of the
    same solve."""
    config, pulse, dt = wl.second_order_self_coupling()
    gp = wl.grid_points(config)
    gpu_rate, state64 = second_order_rate(tb, wl, config, pulse, dt, steps)
    split_rate, state_split = second_order_rate(
        tb, wl, config, pulse, dt, steps,
        tb.LaunchOptions(precision=tb.PRECISION_SPLIT))
    split_dev = max(
        float(np.max(np.abs(state_split[:, f] - state64[:, f])) /
              max(np.max(np.abs(state64[:, f])), 1e-300))
        for f in range(state64.shape[1]))
    # eight such solves (different seeds) at once through the server: they
    # run as replicas of one nodal pipeline, stepped by the same launches
    import torch
    replicas = 8
    server = tb.Server(hbm_budget_bytes=int(0.5 * torch.cuda.mem_get_info()[0]))
    rng = np.random.Generator(np.random.PCG64(20260202))
    for i in range(replicas):
        modes = [(2, m, 1e-2 * complex(rng.standard_normal(), rng.standard_normal()))
                 for m in (-2, 2)]
        server.submit(config, tb.GaussianPulse(center=pulse.center,
                                               width=pulse.width, modes=modes),
                      dt, steps + 2)
    server.advance(2)  # admission, initial data, graph capture
    st0 = server.stats()
    while server.advance(4) > 0:
        pass
    st = server.stats()
    server.close()
    batched_rate = (st.grid_point_updates - st0.grid_point_updates) / (
        st.device_seconds - st0.device_seconds)
    peak, peak_kind = measured_hbm_peak()
    # state-streaming floor: 17 passes x 16 B x 13 fields per nodal point
    # and RK4 step
    achieved = gpu_rate * SECOND_ORDER_BYTES_PER_POINT / 1e9
    sys.path.insert(0, str(REPO / "tests"))
    import oracle_bindings as ob

    ref_rate, cores = None, os.cpu_count()
    if ob.ref_available(threads=True):
        ref = ob.RefPipeline(config, threads=True)
        ref.initialize_gaussian(pulse)
        t0 = time.perf_counter()
        ref.step(0.0, dt, cpu_steps)
        ref_rate = cpu_steps * gp / (time.perf_counter() - t0)
        ref.close()
    return {
        "workload": "a=0.9 nr=1025 d10-5 parents m=+-2 ell<=10, targets "
                    "m={-4,0,4} ell<=20, ntheta=48, source unrestricted "
                    "(active), Gaussian parents amp 1e-2",
        "value": gpu_rate, "unit": UNIT, "steps": steps,
        "replicated": {"solves": replicas, "value": batched_rate, "unit": UNIT,
                       "vs_one_solve": batched_rate / gpu_rate,
                       "how": "8 requests of this shape submitted together to "
                              "the server: replicas of one nodal pipeline, "
                              "device time of the server steps"},
        "split_precision": {
            "value": split_rate, "unit": UNIT, "vs_fp64": split_rate / gpu_rate,
            "max_field_deviation_vs_fp64": split_dev,
            "method": "angular operators through BF16 digit slices (5 per "
                      "operand), FP32 accumulation, FP64 recombination"},
        "reference_cpu": ref_rate, "reference_cores": cores,
        "reference_steps": cpu_steps,
        "dtype": "f64", "storage": "nodal (m, 13 fields, r, theta)",
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak,
                     "algorithmic_bytes_per_point_step": SECOND_ORDER_BYTES_PER_POINT,
                     "peak_source": f"{peak_kind} hbm_gbs", "scope": "whole step"},
    }


# ---------------------------------------------------------------- CPU side
def mapped_repo_libraries():
    """Shared libraries of this repository mapped into this process."""
    try:
        maps = Path("/proc/self/maps").read_text()
    except OSError:
        return []
    found = set()
    for line in maps.splitlines():
        path = line.split()[-1] if line.split() else ""
        if path.endswith(".so") and path.startswith(str(REPO)):
            found.add(str(Path(path).relative_to(REPO)))
    return sorted(found)


def cpu_reference_samples(config, pulse, dt, warmup: int, samples: int | None,
                          seconds: float = 15.0, warm_seconds: float = 3.0):
    """The reference implementation on the host cores (oracle/_ref, thread
    pool over every core), else the C restatement (port, one core).  One
    sample = one RK4 step of one solve of the workload.  Untimed steps run
    first: at least `warmup`, and for at least `warm_seconds` (the
    reference's first steps of a fresh pipeline run at about half its
    steady rate, measured on the GPU boxes' hosts); then `samples` samples
    (or as many as fit in about `seconds`) are timed one by one.  Returns
    (grid-point updates/s over the timed samples, description)."""
    sys.path.insert(0, str(REPO / "tests"))
    import oracle_bindings as ob
    from teuk_b200 import workloads as wl

    threads = os.cpu_count() or 1
    os.environ.setdefault("TEUK_SHIM_NUM_THREADS", str(threads))
    if ob.ref_available(threads=True):
        pipe = ob.RefPipeline(config, threads=True)
        pipe.initialize_gaussian(pulse)
        kind, cores = "reference", int(os.environ["TEUK_SHIM_NUM_THREADS"])
    else:
        pipe = ob.OraclePipeline(config)
        state = np.zeros(config.shape(), dtype=np.complex128)
        pipe.set_state(state + wl.band_noise(config, 1, 1e-3))
        kind, cores = "port", 1
    t = 0.0
    untimed = 0
    warm_start = time.perf_counter()
    while untimed < max(warmup, 1) or time.perf_counter() - warm_start < warm_seconds:
        t0 = time.perf_counter()
        pipe.step(t, dt, 1)
        last = time.perf_counter() - t0
        t += dt
        untimed += 1
    if samples is None:
        samples = max(3, min(2000, int(seconds / max(last, 1e-6))))
    times = []
    for _ in range(samples):
        t0 = time.perf_counter()
        pipe.step(t, dt, 1)
        times.append(time.perf_counter() - t0)
        t += dt
    pipe.close()
    gp = wl.grid_points(config)
    total = sum(times)
    rates = sorted(gp / x for x in times)
    return gp * samples / total, {
        "kind": kind, "cores": cores,
        "sample": f"{samples} timed RK4 steps (after {untimed} untimed, at least "
                  f"{warm_seconds:g} s) of one solve of the workload ({gp} grid "
                  "points per step)",
        "seconds": total, "steps": samples,
        "per_step_rate": {"min": rates[0], "median": statistics.median(rates),
                          "max": rates[-1]},
    }


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    meta, config, pulse, dt = workload_config(args.batch)
    # Each reference step is a bounded sample of the workload: one RK4 step
    # of one of its solves, on every host core.
    value, info = cpu_reference_samples(config, pulse, dt, args.warmup,
                                        args.steps)
    native = mapped_repo_libraries()
    if any("libteuk_b200" in n for n in native):
        raise RuntimeError("the reference arm mapped the B200 engine library")
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * info["seconds"] / info["steps"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded Gaussian pulses)",
        "config": meta, "impl": "reference",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": info["cores"],
                         "kind": info["kind"], "sample": info["sample"],
                         "per_step_rate": info["per_step_rate"]},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "gpu_launches": 0,
        "native_libraries": native,
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- GPU side
def build_batch(tb, wl, config, pulse, batch_size, seed0, pinned, options=None):
    """A batch of `batch_size` copies of the workload with seeded amplitudes
    and noise.  Initial states are linear combinations of two unit-amplitude
    Gaussian states (the system is linear) plus the seeded noise; they are
    written into the pinned host tensor `pinned` (batch, *shape)."""
    import torch
    probe = tb.Pipeline(config)
    units = []
    for m in (2, -2):
        probe.initialize_gaussian(tb.GaussianPulse(center=pulse.center,
                                                   width=pulse.width,
                                                   modes=[(2, m, 1.0)]))
        units.append(probe.get_state())
    probe.close()
    batch = tb.Batch([config] * batch_size, options)
    rng = np.random.Generator(np.random.PCG64(seed0))
    for i in range(batch_size):
        a = 1e-3 * complex(rng.standard_normal(), rng.standard_normal())
        b = 1e-3 * complex(rng.standard_normal(), rng.standard_normal())
        state = a * units[0] + b * units[1] + wl.band_noise(config, seed0 + i)
        pinned[i].copy_(torch.from_numpy(state))
        batch.set_state(i, pinned[i])
    return batch


def b200_arm(args):
    import torch

    import teuk_b200 as tb
    from teuk_b200 import distributed as td
    from teuk_b200 import workloads as wl

    info = td.rank_info()
    world, rank, local = info.world_size, info.rank, info.local_rank
    torch.cuda.set_device(local)
    tb.set_device(local)  # the engine's own CUDA runtime
    td.init("nccl", device=torch.device("cuda", local))

    meta, config, pulse, dt = workload_config(args.batch)
    shape = config.shape()
    B = args.batch
    pinned = torch.empty((B, *shape), dtype=torch.complex128, pin_memory=True)
    # strip lengths chosen by the engine's autotuner at build (results are
    # bit-identical for any choice)
    tuned = tb.LaunchOptions(autotune=True)
    batch = build_batch(tb, wl, config, pulse, B, 1000 * (rank + 1), pinned, tuned)
    stream = torch.cuda.Stream()
    batch.set_stream(stream.cuda_stream)
    dts = [dt] * B

    barrier = td.barrier

    # warm-up (graph capture happens here)
    batch.step(dts, steps=max(args.warmup, 0), graph=True)
    batch.synchronize()
    torch.cuda.synchronize()

    sampler = ClockSampler(device_uuid(torch, local))
    barrier()
    torch.cuda.synchronize()
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    start.record(stream)
    batch.step(dts, steps=args.steps, graph=True)
    end.record(stream)
    end.synchronize()
    torch.cuda.synchronize()
    barrier()
    clocks = sampler.stop()
    ms = start.elapsed_time(end)
    # the evolved states stay bounded (a blown-up run would time the same)
    endpoint = batch.endpoint_modal()
    if not np.all(np.isfinite(endpoint)) or np.max(np.abs(endpoint)) > 1.0:
        raise RuntimeError("benchmark state is not finite and bounded")
    gp = wl.grid_points(config)
    # every rank advanced its own B solves: whole-job units / slowest rank
    value, slowest = td.whole_job_rate(B * gp * args.steps, ms / 1e3, "cuda")
    ms_max = slowest * 1e3
    launches_per_step = batch.launches_per_step()

    # roofline of the stage kernel (four launches per RK4 step)
    modal = wl.modal_values(config) * B
    bytes_per_step = PASSES_PER_STEP * 16 * modal
    launches = launches_per_step * args.steps
    per_launch_s = (ms / 1e3) / launches
    algorithmic_per_launch = bytes_per_step / launches_per_step
    achieved = algorithmic_per_launch / per_launch_s / 1e9
    peak, peak_kind = measured_hbm_peak()
    streaming, _ = batch.stage_kernels()
    kernel = "stream_stage_kernel" if streaming else "stage_kernel"
    strip_rows = batch.strip_rows()
    traffic = recorded_traffic(kernel, algorithmic_per_launch)

    # the same batch with split-precision transforms (BF16 digit slices,
    # FP32 accumulation, FP64 recombination), same inputs and steps
    split = None
    if not args.no_split:
        sbatch = build_batch(tb, wl, config, pulse, B, 1000 * (rank + 1), pinned,
                             tb.LaunchOptions(precision=tb.PRECISION_SPLIT,
                                              autotune=True))
        sbatch.set_stream(stream.cuda_stream)
        sbatch.step(dts, steps=max(args.warmup, 0), graph=True)
        sbatch.synchronize()
        barrier()
        torch.cuda.synchronize()
        s0 = torch.cuda.Event(enable_timing=True)
        s1 = torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        sbatch.step(dts, steps=args.steps, graph=True)
        s1.record(stream)
        s1.synchronize()
        barrier()
        s_value, s_slowest = td.whole_job_rate(B * gp * args.steps,
                                               s0.elapsed_time(s1) / 1e3, "cuda")
        a_end = batch.endpoint_modal()
        b_end = sbatch.endpoint_modal()
        dev = float(np.max(np.abs(a_end - b_end)) / max(np.max(np.abs(a_end)), 1e-300))
        split = {"value": s_value, "unit": UNIT,
                 "ms_per_step": 1e3 * s_slowest / args.steps,
                 "vs_fp64": s_value / value,
                 "endpoint_deviation_vs_fp64": dev,
                 "method": "streaming-kernel transforms through BF16 digit "
                           "slices (5 per operand, 15 products), FP32 "
                           "accumulation, FP64 recombination; stencils, RK "
                           "and projection FP64"}
        sbatch.close()

    # end-to-end through the C ABI with host buffers
    e2e = None
    if not args.no_e2e:
        n_end = batch.endpoint_modal_count()
        waveform = torch.empty(n_end, dtype=torch.complex128, pin_memory=True)
        barrier()
        torch.cuda.synchronize()
        e_start = torch.cuda.Event(enable_timing=True)
        e_end = torch.cuda.Event(enable_timing=True)
        e_start.record(stream)
        for i in range(B):
            batch.set_state(i, pinned[i])
        for _ in range(args.steps):
            batch.step(dts, steps=1, graph=True)
            batch.endpoint_modal(waveform)
        e_end.record(stream)
        e_end.synchronize()
        barrier()
        e_value, e_slowest = td.whole_job_rate(
            B * gp * args.steps, e_start.elapsed_time(e_end) / 1e3, "cuda")
        e_ms = e_slowest * 1e3
        state_bytes = wl.state_bytes(config) * B
        e2e = {"value": e_value, "unit": UNIT,
               "h2d_bytes_per_step": (state_bytes + 8 * B) / args.steps,
               "d2h_bytes_per_step": 16 * n_end,
               "ms_per_step": e_ms / args.steps}

    second_order = None
    if rank == 0 and world == 1 and not args.no_second_order:
        second_order = second_order_run(tb, wl, args.so_steps, 2)

    uneven = None
    if rank == 0 and world == 1 and not args.no_uneven:
        uneven = uneven_batch_run(tb, wl, args.uneven_steps)

    serving = serving_split = None
    if rank == 0 and world == 1 and not args.no_serving:
        serving = serving_run(tb, wl, value, args.serve_requests,
                              args.serve_steps)
        if not args.no_split:
            serving_split = serving_run(tb, wl, value, args.serve_requests,
                                        args.serve_steps,
                                        precision=tb.PRECISION_SPLIT)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        value_cpu, info = cpu_reference_samples(config, pulse, dt, 3, None,
                                                args.cpu_seconds)
        cpu = {"value": value_cpu, "unit": UNIT, "cores": info["cores"],
               "kind": info["kind"], "sample": info["sample"],
               "per_step_rate": info["per_step_rate"]}

    if rank == 0:
        meta = dict(meta)
        meta["parallelism"] = f"{world} GPU x {B} independent solves (no collective)"
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded Gaussian pulses + band noise)",
            "config": meta,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic,
                         "kernel": f"{kernel}<D10-5, free-damped>",
                         "strip_rows": strip_rows,
                         "strip_rows_source": "autotuner (batch build)",
                         "peak_source": f"{peak_kind} hbm_gbs",
                         "algorithmic_bytes_per_launch": algorithmic_per_launch},
            "cpu_baseline": cpu,
            "split_precision": split,
            "e2e": e2e,
            "serving": serving,
            "serving_split_precision": serving_split,
            "uneven_batch": uneven,
            "second_order": second_order,
            "gpu_launches": launches,
            "clocks": clocks,
            "native_libraries": mapped_repo_libraries(),
            "state_check": "endpoint waveform coefficients finite and below 1 "
                           "after the timed steps",
        }
        print(json.dumps(line), flush=True)
    batch.close()
    td.finalize()


def main():
    args = parse_args()
    if args.impl == "reference":
        reference_arm(args)
    else:
        b200_arm(args)


if __name__ == "__main__":
    main()
