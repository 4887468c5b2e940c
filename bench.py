"""Benchmark of the aligned-spin frequency-domain path on B200.

``python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]``

One step is one pass of the path over the 4096-binary batch (IMRPhenomXAS,
masses uniform 5-100 Msun, aligned spins uniform [-0.99, 0.99], distance
100-5000 Mpc, isotropic inclination, phi_ref uniform, f_ref 20 Hz; seeded
synthetic draws) on ``linspace(20, 1024, 4017)``: the FP64 set-up of the
tables and the FP32 polarizations with double-float phase (complex64 out,
263 MB a step: larger than L2, so no flush is needed). The headline value is
binary x frequency evaluations per second, device-resident; ``e2e`` is the
same through ``waveformx_b200.torch.polarizations_function`` with pinned
host buffers (inputs copied in and the strain copied out every step).

Under torchrun each rank evaluates its own batch (weak scaling; NCCL only
for the barrier and the max of the timings). ``--impl reference`` times the
CPU oracle (the NumPy float64 restatement of the reference's algorithm) on
the host cores on a bounded sample of the same workload.

The ``detail`` block adds the plain FP64 form, IMRPhenomD, the fused
likelihood with its gradient (1024 x 4017 and 65536 x 8192), the unfused
FP64 forward + backward, the ragged batch (16384 binaries on their own
grids), and the accuracy against the oracle on a subset.
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

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

MTSUN_SI = 4.925490947641267e-06
METRIC = "XAS (binary×freq) evals/s fwd & fwd+grad, FP32-comp vs FP64 GPU, mismatch≤1e-6"
N_BATCH, GRID = 4096, (20.0, 1024.0, 4017)
#: Algorithmic work per evaluation of the FP32 forward on a shared grid:
#: 16 bytes written (two complex64), 128 FP32 flops (FMA = 2).
BYTES_PER_EVAL = 16
FLOPS_PER_EVAL = 128


def draw_batch(rng, n):
    """The 4096-binary batch's draws: masses uniform 5-100 sorted m1 >= m2,
    chi uniform [-0.99, 0.99], distance uniform 100-5000 Mpc, cos(iota)
    uniform [-1, 1], phi_ref uniform [0, 2 pi), f_ref = 20 Hz."""
    m = rng.uniform(5.0, 100.0, size=(n, 2))
    chi = rng.uniform(-0.99, 0.99, size=(n, 2))
    return np.stack([m.max(1), m.min(1), chi[:, 0], chi[:, 1], rng.uniform(100.0, 5000.0, n),
                     np.arccos(rng.uniform(-1.0, 1.0, n)), rng.uniform(0.0, 2 * np.pi, n), np.full(n, 20.0)], 1)


def psd(f):
    return (f / 20.0) ** -4 + 2.0 + (f / 200.0) ** 2


# ---------------------------------------------------------------------------
# distributed plumbing


def init_dist():
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    elif torch.cuda.is_available():
        torch.cuda.set_device(local)
    return rank, world, local


def barrier(world):
    import torch

    torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        torch.cuda.synchronize()


def max_over_ranks(value, world):
    if world == 1:
        return value
    import torch
    import torch.distributed as dist

    t = torch.tensor([value], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------
# clocks


def _sample_clocks(index, interval, stop, queue, go):
    """The clock sampler's process: NVML's SM clock and clock-event reasons
    of GPU ``index`` every ``interval`` seconds from ``go`` (the timed work
    queued) until ``stop``, then the rows (``(sm_mhz, reasons mask)``) on
    ``queue``."""
    import pynvml

    pynvml.nvmlInit()
    handle = pynvml.nvmlDeviceGetHandleByIndex(index)
    rows = []
    queue.put("ready")
    go.wait(timeout=60)
    while not stop.is_set():
        rows.append((pynvml.nvmlDeviceGetClockInfo(handle, pynvml.NVML_CLOCK_SM),
                     pynvml.nvmlDeviceGetCurrentClocksEventReasons(handle)))
        time.sleep(interval)
    queue.put(rows)


class Clocks:
    """Samples of the SM clock and the clock-event (throttle) reasons during
    the timed region: NVML read every 2 ms by a separate process (so that
    the sampling takes no time from the process that launches the work;
    nvidia-smi's query line from a thread as the fallback), plus one sample
    on entry and one on exit. The process samples from :meth:`queued` on:
    its NVML queries, taken while the host issued the timed region's
    launches, delayed them (measured: 20 pipelined batches 70-76 us a batch
    without the sampler, 80-85 with it sampling from the start)."""

    NAMES = {"hw_slowdown": "HwSlowdown", "hw_thermal_slowdown": "HwThermalSlowdown",
             "sw_thermal_slowdown": "SwThermalSlowdown", "sw_power_cap": "SwPowerCap",
             "hw_power_brake": "HwPowerBrakeSlowdown"}

    def __init__(self, device):
        self.rows = []
        self.stop = threading.Event()
        self.thread = None
        self.process = None
        self.nvml = None
        try:
            import pynvml
            import torch

            pynvml.nvmlInit()
            self.nvml_index = torch.cuda._get_nvml_device_index(device) \
                if hasattr(torch.cuda, "_get_nvml_device_index") else device.index
            self.handle = pynvml.nvmlDeviceGetHandleByIndex(self.nvml_index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.handle, pynvml.NVML_CLOCK_SM)
            self.bits = {k: getattr(pynvml, "nvmlClocksEventReason" + v) for k, v in self.NAMES.items()}
            self.nvml = pynvml
        except Exception:  # no NVML: sample nvidia-smi
            self.index = device.index

    def _row(self, sm, mask):
        return (sm, self.max_mhz, {k for k, b in self.bits.items() if mask & b})

    def sample(self):
        if self.nvml is not None:
            self.rows.append(self._row(self.nvml.nvmlDeviceGetClockInfo(self.handle, self.nvml.NVML_CLOCK_SM),
                                       self.nvml.nvmlDeviceGetCurrentClocksEventReasons(self.handle)))
            return
        q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                  "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5).stdout
            parts = [p.strip() for p in out.strip().split(",")]
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            self.rows.append((float(parts[0]), float(parts[1]),
                              {n for n, v in zip(names, parts[2:]) if v.lower().startswith("active")}))
        except (OSError, ValueError, IndexError, subprocess.TimeoutExpired):
            pass

    def _run(self):
        while not self.stop.wait(0.2):
            self.sample()

    def __enter__(self):
        self.sample()
        if self.nvml is not None:
            import multiprocessing

            ctx = multiprocessing.get_context("spawn")
            self.mp_stop = ctx.Event()
            self.mp_go = ctx.Event()
            self.queue = ctx.Queue()
            self.process = ctx.Process(target=_sample_clocks,
                                       args=(self.nvml_index, 0.002, self.mp_stop, self.queue, self.mp_go),
                                       daemon=True)
            self.process.start()
            try:
                self.queue.get(timeout=120)
            except Exception:  # the sampler did not start: the entry and exit samples stand
                self.process.terminate()
                self.process = None
        else:
            self.thread = threading.Thread(target=self._run, daemon=True)
            self.thread.start()
        return self

    def queued(self):
        """The timed work is queued: the sampling process starts."""
        if self.process is not None:
            self.mp_go.set()

    def __exit__(self, *exc):
        if self.process is not None:
            self.mp_go.set()
            self.mp_stop.set()
            try:
                self.rows.extend(self._row(sm, mask) for sm, mask in self.queue.get(timeout=60))
            except Exception:
                pass
            self.process.join(timeout=10)
            if self.process.is_alive():
                self.process.terminate()
        self.sample()
        if self.thread is not None:
            self.stop.set()
            self.thread.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        sm = [r[0] for r in self.rows]
        loaded = [s for s in sm if s > 0.5 * max(sm)]
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": max(r[1] for r in self.rows),
                "reasons": sorted(set().union(*(r[2] for r in self.rows))), "samples": len(self.rows),
                "source": "nvml" if self.nvml is not None else "nvidia-smi"}


# ---------------------------------------------------------------------------
# the B200 arm


def timed(fn, steps, warmup, world, events=None):
    """ms per step of ``fn`` (device time, CUDA events, max over ranks)."""
    import torch

    for _ in range(warmup):
        fn()
    barrier(world)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    device_ahead(steps)
    start.record()
    for _ in range(steps):
        fn()
    stop.record()
    barrier(world)
    return max_over_ranks(start.elapsed_time(stop) / steps, world)


def device_ahead(steps):
    """Queue a bounded spin of the device (~0.2 ms a step at 1965 MHz,
    1 s at most) ahead of ``steps`` timed steps: the host enqueues them all
    while it runs, so that events recorded after it bracket device work, not
    the host's launch latency."""
    import torch

    torch.cuda._sleep(min(400_000 * steps, 2_000_000_000))


def timed_stream(model, params, freqs, precision, steps, warmup, world):
    """ms per batch of ``steps`` batches through the batch pipeline
    (``polarizations_stream``; device time, CUDA events, max over ranks)."""
    import torch

    from waveformx_b200.pipeline import polarizations_stream

    def run(k):
        for _ in polarizations_stream(model, [params] * k, freqs, f_min=freqs[:1].double(), precision=precision):
            pass

    run(warmup)
    barrier(world)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    run(steps)
    stop.record()
    barrier(world)
    return max_over_ranks(start.elapsed_time(stop) / steps, world)


def timed_batches(model, params, freqs, precision, steps, warmup, world):
    """ms per batch of ``steps`` batches queued by one library call
    (``polarizations_batches``: the set-ups of a group of batches during the
    previous group's forwards, outputs alternating between two slots;
    device time, CUDA events, max over ranks)."""
    import torch

    from waveformx_b200.pipeline import Pipeline, polarizations_batches

    with Pipeline(params.device) as pipe:
        ring = polarizations_batches(model, params.unsqueeze(0).expand(warmup, -1, -1).contiguous(), freqs,
                                     f_min=freqs[:1].double(), precision=precision, ring=2, pipeline=pipe)[:2]
        batches = params.unsqueeze(0).expand(steps, -1, -1).contiguous()
        barrier(world)
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        polarizations_batches(model, batches, freqs, f_min=freqs[:1].double(), precision=precision, ring=2,
                              out=ring, pipeline=pipe)
        stop.record()
        barrier(world)
    return max_over_ranks(start.elapsed_time(stop) / steps, world)


def graphed(fn):
    """``fn`` captured in a CUDA graph (after two warm-up calls on a side
    stream): the graph's replay."""
    import torch

    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        for _ in range(2):
            fn()
    torch.cuda.current_stream().wait_stream(side)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        fn()
    return graph.replay


def b200_arm(args, rank, world, local):
    import torch

    from waveformx_b200 import _lib, ops
    from waveformx_b200 import torch as wt

    device = torch.device("cuda", local)
    rng = np.random.default_rng(1234 + rank)
    params_np = draw_batch(rng, N_BATCH).astype(np.float32)
    f_np = np.linspace(*GRID).astype(np.float32)
    params = torch.as_tensor(params_np.astype(np.float64), device=device)
    freqs = torch.as_tensor(f_np, device=device)
    f_min = freqs[:1].double()
    launches = {"n": 0}
    kernel_ms = []

    def step_device(record=False):
        tables = ops.setup("IMRPhenomXAS", params, f_min, precision=_lib.FP32)
        if record:
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            hp, hc = ops.polarizations("IMRPhenomXAS", tables.table, freqs)
            b.record()
            kernel_ms.append((a, b))
        else:
            hp, hc = ops.polarizations("IMRPhenomXAS", tables.table, freqs)
        launches["n"] += 2
        return hp, hc

    # device-resident, one batch after the other: the forward kernel's own
    # time (the roofline) and the serial step
    for _ in range(args.warmup):
        step_device()
    barrier(world)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # (the events bracket device work only: device_ahead)
    device_ahead(args.steps)
    start.record()
    for _ in range(args.steps):
        step_device(record=True)
    stop.record()
    barrier(world)
    serial_ms = max_over_ranks(start.elapsed_time(stop) / args.steps, world)
    kern = statistics.mean(a.elapsed_time(b) for a, b in kernel_ms)
    kern = max_over_ranks(kern, world)
    evals = N_BATCH * GRID[2]

    # the headline: K batches through the batch pipeline, queued by one
    # library call (wfx_pipeline_run: batch k + 1's set-up on a second
    # stream during batch k's forward; each batch its own set-up and
    # forward); the strain of batch k goes to output slot k % 2
    from waveformx_b200.pipeline import SETUP_BINARIES, Pipeline, polarizations_batches

    pipe = Pipeline(device)

    def copies(k):
        batches = params.unsqueeze(0).expand(k, -1, -1).contiguous()
        torch.cuda.synchronize()
        return batches

    warm = copies(args.warmup)
    group = max(1, min(args.steps, SETUP_BINARIES // N_BATCH))
    ring = polarizations_batches("IMRPhenomXAS", warm, freqs, f_min=f_min, precision=_lib.FP32, ring=2,
                                 group=group, pipeline=pipe)[:2]
    timed_batches = copies(args.steps)
    # (the timed call's buffers, allocated beforehand)
    status_buf = torch.empty((args.steps, N_BATCH), dtype=torch.int32, device=device)
    tables_buf = torch.empty((2, group, N_BATCH, _lib.TABLE_STRIDE), dtype=torch.float32, device=device)
    with Clocks(device) as clocks:
        # (the warm-up batches again once the sampler is up, so that the timed
        # region follows a busy GPU rather than the sampler's start-up)
        polarizations_batches("IMRPhenomXAS", warm, freqs, f_min=f_min, precision=_lib.FP32, ring=2, group=group,
                              out=ring, pipeline=pipe)
        barrier(world)
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        polarizations_batches("IMRPhenomXAS", timed_batches, freqs, f_min=f_min, precision=_lib.FP32, ring=2,
                              group=group, out=ring, pipeline=pipe, status=status_buf, tables=tables_buf)
        stop.record()
        clocks.queued()
        barrier(world)
    ms = max_over_ranks(start.elapsed_time(stop) / args.steps, world)
    gpu_launches = 2 * args.steps  # each batch: the set-up kernel and the forward kernel
    value = evals * world / (ms * 1e-3)
    del warm, timed_batches, ring, status_buf, tables_buf
    pipe.close()

    # end to end through the torch drop-in with pinned host buffers
    fn = wt.polarizations_function("IMRPhenomXAS")
    host_params = torch.as_tensor(params_np).pin_memory()
    host_grid = torch.as_tensor(f_np).pin_memory()
    out_p = torch.empty((N_BATCH, GRID[2]), dtype=torch.complex64).pin_memory()
    out_c = torch.empty_like(out_p).pin_memory()

    def step_e2e():
        p = host_params.to(device, non_blocking=True)
        g = host_grid.to(device, non_blocking=True)
        binary = {"mass_1": p[:, 0], "mass_2": p[:, 1],
                  "spin_1": torch.stack([torch.zeros_like(p[:, 2]), torch.zeros_like(p[:, 2]), p[:, 2]], -1),
                  "spin_2": torch.stack([torch.zeros_like(p[:, 3]), torch.zeros_like(p[:, 3]), p[:, 3]], -1),
                  "luminosity_distance": p[:, 4], "inclination": p[:, 5], "phi_ref": p[:, 6], "f_ref": p[:, 7]}
        hp, hc = fn(binary, g)
        out_p.copy_(hp, non_blocking=True)
        out_c.copy_(hc, non_blocking=True)

    e2e_ms = timed(step_e2e, args.steps, args.warmup, world)
    h2d = host_params.numel() * 4 + host_grid.numel() * 4
    d2h = 2 * out_p.numel() * 8

    detail = {}
    if not args.quick:
        detail = details(args, device, world, rng)

    peaks = {}
    peaks_path = ROOT / "MEASURED_PEAKS.json"
    if peaks_path.exists():
        peaks = json.loads(peaks_path.read_text())
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    achieved = BYTES_PER_EVAL * evals / (kern * 1e-3) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s", "frac": achieved / hbm_peak,
                "traffic": traffic_from_profiles("k_fwd_f32_shared"), "kernel": "k_fwd_f32_shared<XAS>",
                "kernel_ms": kern, "algorithmic_bytes_per_launch": BYTES_PER_EVAL * evals,
                "peak_source": "MEASURED_PEAKS.json hbm_gbs (burst copy) of measured" if peaks else "fallback"}
    line = {
        "metric": METRIC, "value": value, "unit": "evals/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 (double-float phase; FP64 set-up)", "data": "synthetic (seeded draws of the batch config)",
        "config": {"workload": "IMRPhenomXAS batch 4096 x linspace(20,1024,4017), FP32-comp, complex64 out",
                   "global_batch": N_BATCH * world, "frequencies": GRID[2], "parallelism": f"binaries sharded x{world}",
                   "l2": "no flush: each step writes 263 MB of strain (> 126 MB L2)"},
        "e2e": {"value": evals * world / (e2e_ms * 1e-3), "unit": "evals/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "api": "waveformx_b200.torch.polarizations_function (pinned host in/out)"},
        "roofline": roofline,
        "gpu_launches": gpu_launches,
        "clocks": clocks.summary(),
        "step": {"pipeline": "waveformx_b200.pipeline.polarizations_batches (wfx_pipeline_run, one call for the "
                             "K batches): set-up of batch k+1 during the forward of batch k",
                 "serial_ms_per_step": serial_ms,
                 "serial_evals_per_s": evals * world / (serial_ms * 1e-3)},
        "detail": detail,
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(params_np, f_np, budget_s=args.cpu_seconds)
    return line


def traffic_from_profiles(kernel):
    """DRAM bytes per launch of ``kernel`` from the committed ncu summary
    (profiles/traffic.txt: ``kernel workload bytes``), or None."""
    path = ROOT / "profiles" / "traffic.txt"
    if not path.exists():
        return None
    for line in path.read_text().splitlines():
        parts = line.split()
        if len(parts) >= 3 and parts[0] == kernel:
            try:
                return float(parts[-1])
            except ValueError:
                return None
    return None


#: FP32 flops per evaluation of the fused likelihood and its gradient (the
#: forward's 128, the 8 tangent directions' 54 each, 40 for the residual, the
#: loss and the reduction; FMA = 2): the figure of the roofline of k_adj_f32.
FUSED_FLOPS_PER_EVAL = 600

#: The slot of an IMRPhenomXAS table that holds its amplitude cutoff (Hz):
#: above it the waveform is zero and the reverse pass evaluates the loss only.
XAS_F_CUT_SLOT = 53

#: The measurement kernel of the FMA issue peak: 8 independent FMA chains a
#: thread, 128 FMAs per loop trip, nothing stored in practice (the guard
#: never holds, but the compiler cannot drop the chains). REAL and FMA are
#: float and fmaf, or double and fma.
FMA_SOURCE = r"""
extern "C" __global__ void __launch_bounds__(256) fma_chains(REAL* out, int iters, REAL a, REAL b) {
  REAL x[8];
  for (int k = 0; k < 8; ++k) x[k] = threadIdx.x * (REAL)1e-3 + k;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int j = 0; j < 16; ++j) {
#pragma unroll
      for (int k = 0; k < 8; ++k) x[k] = FMA(x[k], a, b);
    }
  }
  REAL s = 0;
  for (int k = 0; k < 8; ++k) s += x[k];
  if (s == (REAL)123.456) out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}
"""


def fma_peak(device, iters=4096, blocks_per_sm=8, launches=10, real="float"):
    """The FP32 (``real`` "double": FP64) FMA issue rate of this GPU,
    measured: FMA_SOURCE compiled by NVRTC for sm_100a and launched on every
    SM (``blocks_per_sm`` blocks of 256 threads each), timed with CUDA events
    over ``launches`` launches after three warm-up ones; flops = 2 x FMAs.
    The SM clock is sampled meanwhile (the peak scales with it)."""
    import ctypes

    import torch
    from cuda.bindings import driver, nvrtc

    err, prog = nvrtc.nvrtcCreateProgram(FMA_SOURCE.encode(), b"fma_chains.cu", 0, [], [])
    opts = [b"--gpu-architecture=sm_100a", f"-DREAL={real}".encode(),
            b"-DFMA=fma" if real == "double" else b"-DFMA=fmaf"]
    (err,) = nvrtc.nvrtcCompileProgram(prog, len(opts), opts)
    if err != nvrtc.nvrtcResult.NVRTC_SUCCESS:
        raise RuntimeError(f"NVRTC failed: {err}")
    err, size = nvrtc.nvrtcGetCUBINSize(prog)
    cubin = b" " * size
    nvrtc.nvrtcGetCUBIN(prog, cubin)
    nvrtc.nvrtcDestroyProgram(prog)
    torch.cuda.synchronize(device)  # (the device's primary context is current)
    err, module = driver.cuModuleLoadData(cubin)
    if err != driver.CUresult.CUDA_SUCCESS:
        raise RuntimeError(f"cuModuleLoadData: {err}")
    err, fn = driver.cuModuleGetFunction(module, b"fma_chains")
    sms = torch.cuda.get_device_properties(device).multi_processor_count
    grid = sms * blocks_per_sm
    double = real == "double"
    sink = torch.empty(grid * 256, dtype=torch.float64 if double else torch.float32, device=device)
    stream = torch.cuda.current_stream(device)
    ct = ctypes.c_double if double else ctypes.c_float
    args = ((sink.data_ptr(), iters, 0.9999, 1e-3), (ctypes.c_void_p, ctypes.c_int, ct, ct))

    def launch():
        (e,) = driver.cuLaunchKernel(fn, grid, 1, 1, 256, 1, 1, 0, driver.CUstream(stream.cuda_stream), args, 0)
        if e != driver.CUresult.CUDA_SUCCESS:
            raise RuntimeError(f"cuLaunchKernel: {e}")

    for _ in range(3):
        launch()
    torch.cuda.synchronize(device)
    with Clocks(device) as clocks:
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        for _ in range(launches):
            launch()
        stop.record()
        clocks.queued()
        torch.cuda.synchronize(device)
    ms = start.elapsed_time(stop) / launches
    driver.cuModuleUnload(module)
    flops = 2.0 * grid * 256 * iters * 128
    summary = clocks.summary()
    return {"tflops": flops / (ms * 1e-3) / 1e12, "ms_per_launch": ms, "flops_per_launch": flops,
            "kernel": f"fma_chains<{real}> (8 FMA chains per thread, 256 threads, {blocks_per_sm} blocks per SM)",
            "clocks": summary,
            "fp32_nominal_tflops_at_sm_mhz": (sms * 128 * 2 * summary["sm_mhz"] * 1e6 / 1e12) if summary["sm_mhz"]
            else None}


def fused_kernel_ms(p, freqs, tc, d, w, steps, warm, world):
    """ms per launch of the FP32 fused reverse pass alone
    (wfx_fused_loss_partials: k_adj_f32 on the shared grid), CUDA events on
    the launching stream, max over ranks."""
    from waveformx_b200 import _lib, ops

    tables = ops.setup("IMRPhenomXAS", p, freqs[:1].double(), precision=_lib.FP32)
    batch, n = p.shape[0], freqs.numel()
    ws = ops.workspace(_lib.OP_FUSED, _lib.XAS, _lib.FP32, batch, n, False, p.device)
    data_stride = ops.check_per_frequency(d, "data", batch, n, False)
    lib = _lib.library()

    def launch():
        _lib.check("wfx_fused_loss_partials", lib.wfx_fused_loss_partials(
            _lib.XAS, ops._ptr(tables.table), ops._ptr(freqs), None, batch, n, ops._ptr(tc), ops._ptr(d),
            data_stride, ops._ptr(w), 0, 1.0, 0.0, -0.5, ops._ptr(ws), ws.numel(), ops._stream(p.device)))

    return timed(launch, steps, warm, world)


def likelihood_workload(label, nb, grid, device):
    """The likelihood configurations' inputs (float32-rounded parameters,
    t_c, the grid, the data, the weights w = 1 / S):
    * c3: 1024 binaries on linspace(20, 1024, 4017), t_c = 0; each binary's
      data d_b = h+ at its parameters times (1 + 0.01 N(0, 1)) (spins
      clipped to [-0.99, 0.99], f_ref kept) plus complex Gaussian noise of
      standard deviation 0.1 |h+| per component;
    * c4: 65536 binaries with t_c uniform [-0.1, 0.1] s on
      linspace(10, 2048, 8192); one data vector shared by all: an injected
      binary's h+ plus complex Gaussian noise of variance eps^2 S(f), eps
      set for an SNR of 20 with w = 1 / S.
    The waveforms of the data come from the FP64 path (pinned to the
    reference's own outputs by the tests)."""
    import torch

    from waveformx_b200 import _lib, ops

    rng = np.random.default_rng(5 if label == "c3" else 6)
    p_np = draw_batch(rng, nb).astype(np.float32).astype(np.float64)
    f_np = np.linspace(*grid).astype(np.float32)
    f64 = torch.as_tensor(f_np.astype(np.float64), device=device)
    w = 1.0 / psd(f_np.astype(np.float64))
    if label == "c3":
        t_c = np.zeros(nb, dtype=np.float32)
        shifted = p_np * (1.0 + 0.01 * rng.normal(size=p_np.shape))
        shifted[:, 2:4] = np.clip(shifted[:, 2:4], -0.99, 0.99)
        shifted[:, 7] = p_np[:, 7]
        t = ops.setup("IMRPhenomXAS", torch.as_tensor(shifted, device=device), f64[:1], precision=_lib.FP64)
        h = ops.polarizations("IMRPhenomXAS", t.table, f64)[0].cpu().numpy()
        sigma = 0.1 * np.abs(h)
        data = h + sigma * (rng.normal(size=h.shape) + 1j * rng.normal(size=h.shape))
    else:
        t_c = rng.uniform(-0.1, 0.1, nb).astype(np.float32)
        injection = draw_batch(rng, 1)
        t = ops.setup("IMRPhenomXAS", torch.as_tensor(injection, device=device), f64[:1], precision=_lib.FP64)
        h = ops.polarizations("IMRPhenomXAS", t.table, f64)[0][0].cpu().numpy()
        s = psd(f_np.astype(np.float64))
        eps = np.sqrt(np.sum(np.abs(h) ** 2 / s)) / 20.0
        data = h + eps * np.sqrt(s / 2.0) * (rng.normal(size=h.shape) + 1j * rng.normal(size=h.shape))
    return p_np, t_c, f_np, data, w


def loss_grad_accuracy(fp32, fp64):
    """The FP32 fused loss and gradient against the FP64 unfused ones: the
    largest relative loss error, and the largest |g32 - g64| over the
    reference's FP32 bound 1e-2 |g64| + 1e-3 max |g64| (per binary; <= 1
    passes)."""
    l32, g32 = fp32
    l64, g64 = fp64
    ok = np.isfinite(l64)
    rel = np.abs(l32[ok] - l64[ok]) / np.abs(l64[ok])
    bound = 1e-2 * np.abs(g64[ok]) + 1e-3 * np.max(np.abs(g64[ok]), axis=1, keepdims=True)
    ratio = np.abs(g32[ok] - g64[ok]) / np.where(bound > 0, bound, 1.0)
    return {"binaries": int(ok.sum()), "max_rel_loss_error": float(rel.max()),
            "max_grad_error_over_bound": float(ratio.max()),
            "median_grad_error_over_bound": float(np.median(ratio.max(axis=1)))}


def details(args, device, world, rng):
    """The other forms, each timed as the headline (device-resident)."""
    import torch

    from waveformx_b200 import _lib, ops

    out = {}
    f32 = np.linspace(*GRID).astype(np.float32)
    params_np = draw_batch(np.random.default_rng(77), N_BATCH).astype(np.float32).astype(np.float64)
    params = torch.as_tensor(params_np, device=device)
    steps, warm = max(3, args.steps // 2), max(3, args.warmup)
    evals = N_BATCH * GRID[2]
    for model in ("IMRPhenomXAS", "IMRPhenomD", "TaylorF2", "IMRPhenomXHM"):
        for name, precision, real in (("fp32", _lib.FP32, torch.float32), ("fp64", _lib.FP64, torch.float64)):
            freqs = torch.as_tensor(f32, dtype=real, device=device)

            def fwd():
                t = ops.setup(model, params, freqs[:1].double(), precision=precision)
                return ops.polarizations(model, t.table, freqs)

            ms = timed(fwd, steps, warm, world)
            out[f"{model}_{name}_fwd_evals_per_s"] = evals * world / (ms * 1e-3)
            # the same batches through the batch pipeline
            ms = timed_stream(model, params, freqs, precision, steps, warm, world)
            out[f"{model}_{name}_stream_evals_per_s"] = evals * world / (ms * 1e-3)
            # the same batches queued by one library call
            ms = timed_batches(model, params, freqs, precision, steps, warm, world)
            out[f"{model}_{name}_batches_evals_per_s"] = evals * world / (ms * 1e-3)
            # the frequency kernel alone (tables already set up)
            table = ops.setup(model, params, freqs[:1].double(), precision=precision).table
            ms = timed(lambda: ops.polarizations(model, table, freqs), steps, warm, world)
            out[f"{model}_{name}_fwd_kernel_ms"] = ms
            del table
        out[f"{model}_fwd_ratio_fp32_over_fp64"] = (out[f"{model}_fp32_fwd_evals_per_s"]
                                                    / out[f"{model}_fp64_fwd_evals_per_s"])
        out[f"{model}_stream_ratio_fp32_over_fp64"] = (out[f"{model}_fp32_stream_evals_per_s"]
                                                       / out[f"{model}_fp64_stream_evals_per_s"])
        out[f"{model}_batches_ratio_fp32_over_fp64"] = (out[f"{model}_fp32_batches_evals_per_s"]
                                                        / out[f"{model}_fp64_batches_evals_per_s"])
        out[f"{model}_fwd_kernel_ratio_fp32_over_fp64"] = (out[f"{model}_fp64_fwd_kernel_ms"]
                                                           / out[f"{model}_fp32_fwd_kernel_ms"])
    # a template bank matched against one signal, maximised over time and
    # phase: the templates evaluated into the overlap series (FP32, never
    # written as strain), cuFFT, FP64 refinement; vs the plain FP64 form
    # (strain written, then matched)
    from waveformx_b200 import match as wmatch

    f64 = np.linspace(*GRID)
    w64 = psd(f64)
    t0 = ops.setup("IMRPhenomXAS", params[:1], torch.as_tensor(f64[:1], device=device), precision=_lib.FP64)
    sig128 = ops.polarizations("IMRPhenomXAS", t0.table, torch.as_tensor(f64, device=device))[0][0]
    sig64 = sig128.to(torch.complex64).contiguous()
    w32_t = torch.as_tensor(w64, dtype=torch.float32, device=device)
    w64_t = torch.as_tensor(w64, device=device)
    f64_t = torch.as_tensor(f64, device=device)
    ms = timed(lambda: wmatch.template_match("IMRPhenomXAS", params, f64, sig64, w32_t), steps, warm, world)
    out["bank_fp32_fused_match_evals_per_s"] = evals * world / (ms * 1e-3)

    def bank64():
        t = ops.setup("IMRPhenomXAS", params, f64_t[:1], precision=_lib.FP64)
        hp, _ = ops.polarizations("IMRPhenomXAS", t.table, f64_t)
        return wmatch.match(hp, sig128, f64, w64_t)

    ms = timed(bank64, max(3, steps // 4), warm, world)
    out["bank_fp64_unfused_match_evals_per_s"] = evals * world / (ms * 1e-3)
    out["bank_match_ratio_fp32_fused_over_fp64_unfused"] = (out["bank_fp32_fused_match_evals_per_s"]
                                                            / out["bank_fp64_unfused_match_evals_per_s"])
    wmatch._SERIES.clear()
    torch.cuda.empty_cache()
    # forward + gradient: fused likelihood (FP32) vs unfused FP64 forward + backward
    peak = fma_peak(device)
    out["fp32_fma_peak"] = peak
    out["fp64_fma_peak"] = fma_peak(device, iters=1024, real="double")
    accuracy_lg = {}
    for label, nb, grid in (("c3", 1024, (20.0, 1024.0, 4017)), ("c4", 65536, (10.0, 2048.0, 8192))):
        p_np, t_c, f_np, data_np, w = likelihood_workload(label, nb, grid, device)
        p = torch.as_tensor(p_np, device=device)
        rows = nb * grid[2]
        results = {}
        for name, precision, real, cplx in (("fp32_fused", _lib.FP32, torch.float32, torch.complex64),
                                            ("fp64_fused", _lib.FP64, torch.float64, torch.complex128)):
            if label == "c4" and name == "fp64_fused":
                continue
            freqs = torch.as_tensor(f_np, dtype=real, device=device)
            tc = torch.as_tensor(t_c, dtype=real, device=device)
            d = torch.as_tensor(data_np, dtype=cplx, device=device)
            wt_ = torch.as_tensor(w, dtype=real, device=device)

            def fused():
                if precision == _lib.FP32:
                    # (the dual-number set-up on a second stream, overlapped
                    # with the value set-up and the reverse pass)
                    return ops.fused_loss_from_params("IMRPhenomXAS", p, freqs[:1].double(), freqs, None, tc, d,
                                                      wt_, scale=-0.5)
                t = ops.setup("IMRPhenomXAS", p, freqs[:1].double(), precision=precision, jvp=True)
                return ops.fused_loss("IMRPhenomXAS", t.table, t.dtable, freqs, None, tc, d, wt_, scale=-0.5)

            ms = timed(fused, steps, warm, world)
            out[f"{label}_{name}_loss_grad_evals_per_s"] = rows * world / (ms * 1e-3)
            if precision != _lib.FP32:
                continue
            loss, grad = fused()[:2]
            results["fp32"] = (loss.double().cpu().numpy(), grad.double().cpu().numpy())
            # the reverse kernel alone (k_adj_f32, fused): its roofline against
            # the measured FP32 FMA peak
            kernel_ms = fused_kernel_ms(p, freqs, tc, d, wt_, steps, warm, world)
            # (the 600 flops are those of an evaluation below the binary's
            # amplitude cutoff; above it the kernel adds w |d|^2 to the loss)
            f_cut = ops.setup("IMRPhenomXAS", p, freqs[:1].double(), precision=_lib.FP64).table[:, XAS_F_CUT_SLOT]
            in_band = int((freqs.double()[None, :] <= f_cut[:, None]).sum())
            achieved = FUSED_FLOPS_PER_EVAL * in_band / (kernel_ms * 1e-3) / 1e12
            out[f"{label}_fused_roofline"] = {
                "bound": "fp32", "kernel": "k_adj_f32<XAS, shared grid, fused>", "kernel_ms": kernel_ms,
                "flops_per_eval": FUSED_FLOPS_PER_EVAL, "in_band_evals": in_band, "evals": rows,
                "achieved": achieved, "peak": peak["tflops"], "unit": "TFLOP/s", "frac": achieved / peak["tflops"],
                "achieved_counting_every_eval": FUSED_FLOPS_PER_EVAL * rows / (kernel_ms * 1e-3) / 1e12,
                "peak_source": "FP32 FMA-chain kernel measured in this run (fp32_fma_peak)"}
            # K batches through the batch pipeline (pipeline.likelihood_stream:
            # the set-ups of batch k + 1 during batch k's fused likelihood)
            from waveformx_b200.pipeline import likelihood_stream

            def run_stream(k):
                for _ in likelihood_stream("IMRPhenomXAS", [(p, tc)] * k, freqs, d, wt_, scale=-0.5):
                    pass

            run_stream(warm)
            barrier(world)
            start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record()
            run_stream(steps)
            stop.record()
            barrier(world)
            ms = max_over_ranks(start.elapsed_time(stop) / steps, world)
            out[f"{label}_fp32_fused_stream_loss_grad_evals_per_s"] = rows * world / (ms * 1e-3)
            # the same step replayed from a CUDA graph (graphs.CapturedLikelihood:
            # parameters and t_c copied in, every kernel of the step replayed)
            from waveformx_b200.graphs import CapturedLikelihood

            captured = CapturedLikelihood("IMRPhenomXAS", nb, freqs, d, wt_, t_c=True, scale=-0.5)
            captured(p, tc)
            ms = timed(lambda: captured(p, tc), steps, warm, world)
            out[f"{label}_fp32_fused_graph_loss_grad_evals_per_s"] = rows * world / (ms * 1e-3)
            del captured
            # K batches in one library call (pipeline.likelihood_batches:
            # the dual-number set-ups of a group of batches, 4096 binaries, in
            # one launch during the previous group's fused likelihoods)
            from waveformx_b200.pipeline import LIKELIHOOD_SETUP_BINARIES, Pipeline, likelihood_batches

            kb = max(8, args.steps)
            group = max(1, min(kb, LIKELIHOOD_SETUP_BINARIES // nb))
            pk = p.unsqueeze(0).expand(kb, nb, 8).contiguous()
            tck = tc.unsqueeze(0).expand(kb, nb).contiguous()
            bufs = dict(out=(torch.empty((kb, nb), dtype=torch.float32, device=device),
                             torch.empty((kb, nb, _lib.GRAD_COLUMNS), dtype=torch.float32, device=device)),
                        status=torch.empty((kb, nb), dtype=torch.int32, device=device),
                        tables=(torch.empty((2, group, nb, _lib.TABLE_STRIDE), dtype=torch.float32, device=device),
                                torch.empty((2, group, nb, _lib.TABLE_STRIDE, 8), dtype=torch.float64,
                                            device=device)),
                        workspace=torch.empty(2 * int(_lib.library().wfx_workspace_bytes(
                            _lib.OP_FUSED, _lib.XAS, _lib.FP32, nb, grid[2], 0)), dtype=torch.uint8, device=device))
            with Pipeline(device) as pipe:
                def run_batches():
                    likelihood_batches("IMRPhenomXAS", pk, freqs, d, wt_, t_c=tck, scale=-0.5, group=group,
                                       pipeline=pipe, **bufs)

                run_batches()
                barrier(world)
                start.record()
                run_batches()
                stop.record()
                barrier(world)
                ms = max_over_ranks(start.elapsed_time(stop) / kb, world)
            out[f"{label}_fp32_fused_batches_loss_grad_evals_per_s"] = rows * world / (ms * 1e-3)
            out[f"{label}_fp32_fused_batches"] = {"batches": kb, "group": group, "ms_per_batch": ms}
            del pk, tck, bufs
        # plain FP64, unfused: forward to memory, residual and cotangent, backward
        freqs = torch.as_tensor(f_np, dtype=torch.float64, device=device)
        tc = torch.as_tensor(t_c.astype(np.float64), device=device)
        d = torch.as_tensor(data_np, dtype=torch.complex128, device=device)
        wt_ = torch.as_tensor(w, device=device)

        def unfused():
            t = ops.setup("IMRPhenomXAS", p, freqs[:1].double(), precision=_lib.FP64, jvp=True)
            hp, hc = ops.polarizations("IMRPhenomXAS", t.table, freqs, None, tc)
            r = hp - d
            loss = -0.5 * (wt_ * (r.real ** 2 + r.imag ** 2)).sum(-1)
            cot = (-wt_ * r).contiguous()
            grad = ops.vjp("IMRPhenomXAS", t.table, t.dtable, freqs, None, tc, cot, torch.zeros_like(hc))
            return loss, grad

        s = 2 if label == "c4" else steps
        ms = timed(unfused, s, 2 if label == "c4" else warm, world)
        out[f"{label}_fp64_unfused_loss_grad_evals_per_s"] = rows * world / (ms * 1e-3)
        loss64, grad64 = unfused()
        accuracy_lg[label] = loss_grad_accuracy(results["fp32"], (loss64.cpu().numpy(), grad64.cpu().numpy()))
        del loss64, grad64
        out[f"{label}_loss_grad_ratio_fp32_fused_over_fp64_unfused"] = (
            out[f"{label}_fp32_fused_loss_grad_evals_per_s"] / out[f"{label}_fp64_unfused_loss_grad_evals_per_s"])
        fp64_key = f"{label}_fp64_unfused_loss_grad_evals_per_s"
        if label == "c3":
            # the plain FP64 step replayed from a CUDA graph too (c4's is
            # bound by its kernels: its eager time stands)
            replay = graphed(unfused)
            ms = timed(replay, steps, warm, world)
            fp64_key = f"{label}_fp64_unfused_graph_loss_grad_evals_per_s"
            out[fp64_key] = rows * world / (ms * 1e-3)
            del replay
        out[f"{label}_loss_grad_ratio_graph_fp32_fused_over_fp64_unfused"] = (
            out[f"{label}_fp32_fused_graph_loss_grad_evals_per_s"] / out[fp64_key])
        out[f"{label}_loss_grad_ratio_stream_fp32_fused_over_fp64_unfused"] = (
            out[f"{label}_fp32_fused_stream_loss_grad_evals_per_s"] / out[fp64_key])
        out[f"{label}_loss_grad_ratio_batches_fp32_fused_over_fp64_unfused"] = (
            out[f"{label}_fp32_fused_batches_loss_grad_evals_per_s"] / out[fp64_key])
        del d, wt_, freqs
        torch.cuda.empty_cache()
    out["loss_grad_accuracy"] = accuracy_lg
    # ragged: 16384 binaries on their own grids
    nb = 16384
    p_np = draw_batch(np.random.default_rng(9), nb).astype(np.float32).astype(np.float64)
    r2 = np.random.default_rng(10)
    f_low = r2.uniform(10.0, 30.0, nb)
    duration = r2.choice([4.0, 8.0, 16.0, 32.0, 64.0], nb)
    f_high = np.minimum(2048.0, 0.3 / ((p_np[:, 0] + p_np[:, 1]) * MTSUN_SI))
    lengths = np.maximum(np.floor((f_high - f_low) * duration).astype(np.int64), 1)
    offsets_np = np.concatenate([[0], np.cumsum(lengths)])
    total = int(offsets_np[-1])
    idx = np.arange(total) - np.repeat(offsets_np[:-1], lengths)
    flat = (np.repeat(f_low, lengths) + idx / np.repeat(duration, lengths)).astype(np.float32)
    p = torch.as_tensor(p_np, device=device)
    freqs = torch.as_tensor(flat, device=device)
    offsets = torch.as_tensor(offsets_np, device=device)
    f_min = torch.as_tensor(f_low.astype(np.float32).astype(np.float64), device=device)

    def ragged():
        t = ops.setup("IMRPhenomXAS", p, f_min, precision=_lib.FP32)
        return ops.polarizations("IMRPhenomXAS", t.table, freqs, offsets)

    ms = timed(ragged, steps, warm, world)
    out["c2_ragged_fp32_fwd_evals_per_s"] = total * world / (ms * 1e-3)
    # the same, autotuned and replayed from a CUDA graph (one launch per step)
    from waveformx_b200.graphs import CapturedPolarizations
    from waveformx_b200.tuning import lookup

    captured = CapturedPolarizations("IMRPhenomXAS", nb, freqs, offsets)
    captured(p)
    ms = timed(lambda: captured(p), steps, warm, world)
    out["c2_ragged_graph_tuned_fp32_fwd_evals_per_s"] = total * world / (ms * 1e-3)
    out["c2_ragged_tuning"] = dict(zip(("item_length", "blocks_per_sm", "tuned"), lookup("IMRPhenomXAS", nb, total)))
    out["c2_ragged_total_evals"] = total
    out["c2_ragged_max_length"] = int(lengths.max())
    del captured, freqs, offsets
    torch.cuda.empty_cache()
    out["accuracy"] = accuracy(device)
    return out


def accuracy(device):
    """Noise-weighted mismatch, max phase error and max relative amplitude
    error of the FP32 kernels against the oracle on 64 binaries of the batch
    draw (float32-rounded inputs)."""
    import torch

    import oracle
    from oracle.api import amplitude_error
    from waveformx_b200 import _lib, ops

    out = {}
    p_np = draw_batch(np.random.default_rng(3), 64).astype(np.float32).astype(np.float64)
    for label, grid, t_c in (("c1", GRID, None), ("c4", (10.0, 2048.0, 8192), 0.1)):
        f = np.linspace(*grid).astype(np.float32).astype(np.float64)
        tc_np = None if t_c is None else np.random.default_rng(4).uniform(-t_c, t_c, 64).astype(np.float32)
        for model in ("IMRPhenomXAS", "IMRPhenomD", "TaylorF2"):
            p = torch.as_tensor(p_np, device=device)
            freqs = torch.as_tensor(f, dtype=torch.float32, device=device)
            t = ops.setup(model, p, freqs[:1].double(), precision=_lib.FP32)
            tc = None if tc_np is None else torch.as_tensor(tc_np, device=device)
            hp, _ = ops.polarizations(model, t.table, freqs, None, tc)
            ref, _ = oracle.polarizations(model, p_np, f, t_c=None if tc_np is None else tc_np.astype(np.float64))
            a = hp.cpu().numpy().astype(np.complex128)
            out[f"{label}_{model}"] = {"max_mismatch": float(np.max(oracle.mismatch(a, ref, 1.0 / psd(f)))),
                                       "max_phase_error_rad": float(np.max(oracle.phase_error(a, ref))),
                                       "max_rel_amplitude_error": float(np.max(amplitude_error(a, ref)))}
        # IMRPhenomXHM: FP32 against the FP64 form (which the tests pin to the
        # reference's own outputs to 1e-9)
        p = torch.as_tensor(p_np, device=device)
        tc32 = None if tc_np is None else torch.as_tensor(tc_np, device=device)
        hp32, _ = ops.polarizations("IMRPhenomXHM", ops.setup("IMRPhenomXHM", p, torch.as_tensor(f[:1], device=device),
                                                              precision=_lib.FP32).table,
                                    torch.as_tensor(f, dtype=torch.float32, device=device), None, tc32)
        tc64 = None if tc_np is None else torch.as_tensor(tc_np.astype(np.float64), device=device)
        hp64, _ = ops.polarizations("IMRPhenomXHM", ops.setup("IMRPhenomXHM", p, torch.as_tensor(f[:1], device=device),
                                                              precision=_lib.FP64).table,
                                    torch.as_tensor(f, device=device), None, tc64)
        a, ref = hp32.cpu().numpy().astype(np.complex128), hp64.cpu().numpy()
        out[f"{label}_IMRPhenomXHM_fp32_vs_fp64"] = {
            "max_mismatch": float(np.max(oracle.mismatch(a, ref, 1.0 / psd(f)))),
            "max_phase_error_rad": float(np.max(oracle.phase_error(a, ref))),
            "max_rel_amplitude_error": float(np.max(amplitude_error(a, ref)))}
    return out


# ---------------------------------------------------------------------------
# CPU baseline and the reference arm (the oracle on the host cores)


def cpu_baseline(params_np, f_np, budget_s=10.0, threads=0):
    """The oracle's C restatement (``oracle/xas_eval.c``, ``kind`` port) of
    the reference's CPU path on every host core: per step the NumPy
    oracle's tables of the batch (vectorised over binaries) and the C
    evaluation of every binary at every frequency (POSIX threads over
    binaries; the grid's powers once, as jax.vmap with the grid unbatched).
    The whole batch per step, repeated for about ``budget_s``; the median
    step."""
    from oracle import native, xas

    p = params_np.astype(np.float64)
    f = f_np.astype(np.float64)
    cores = threads if threads > 0 else native.cores()

    def step():
        tab = xas.flat(xas.table(p, f[0]))
        return native.xas_evaluate(tab, f, cores)

    step()  # warm-up (the library's first load, page faults of the outputs)
    times, t0 = [], time.perf_counter()
    while time.perf_counter() - t0 < budget_s or len(times) < 3:
        a = time.perf_counter()
        step()
        times.append(time.perf_counter() - a)
    seconds = statistics.median(times)
    evals = p.shape[0] * f.size
    return {"value": evals / seconds, "unit": "evals/s", "cores": cores, "kind": "port",
            "sample": f"the whole {p.shape[0]}-binary batch x {f.size} frequencies per step, {len(times)} steps "
                      f"(median {seconds * 1e3:.1f} ms): the oracle's tables (NumPy float64) and its C "
                      f"restatement of the evaluation on {cores} threads",
            "same_config": True}


def reference_arm(args, rank, world):
    """The reference's CPU path on the host cores: JAX, which the reference
    runs on, is absent, so its algorithm as the oracle restates it (the
    NumPy tables and the C evaluation, all host threads), one whole batch
    per step: ``--warmup`` untimed steps, then the median of ``--steps``."""
    if rank != 0:
        return None
    from oracle import native, xas

    params_np = draw_batch(np.random.default_rng(1234), N_BATCH).astype(np.float32).astype(np.float64)
    f_np = np.linspace(*GRID).astype(np.float32).astype(np.float64)
    cores = native.cores()

    def step():
        tab = xas.flat(xas.table(params_np, f_np[0]))
        return native.xas_evaluate(tab, f_np, cores)

    times = []
    for i in range(args.warmup + args.steps):
        a = time.perf_counter()
        step()
        if i >= args.warmup:
            times.append(time.perf_counter() - a)
    seconds = statistics.median(times)
    value = N_BATCH * GRID[2] / seconds
    return {
        "metric": METRIC, "value": value, "unit": "evals/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": seconds * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded draws of the batch config)",
        "config": {"workload": "IMRPhenomXAS batch 4096 x linspace(20,1024,4017), FP64, complex128 out",
                   "global_batch": N_BATCH, "frequencies": GRID[2], "parallelism": f"{cores} host threads"},
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": "evals/s", "cores": cores, "kind": "port",
                         "sample": f"the whole batch per step (median of {args.steps} steps after {args.warmup})",
                         "same_config": True},
        "e2e": {"value": value, "unit": "evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "reference JAX CPU: unavailable on this box (jax is not installed); the oracle restates its "
                "algorithm (NumPy float64 tables, C evaluation on POSIX threads)",
    }


def profile_case(args):
    """Run one family of kernels on its workload ``--steps + --warmup`` times
    and exit (a command for ncu): ``forward`` (the 4096 x 4017 batch, FP32),
    ``forward64`` (the same, plain FP64), ``fused`` (the fused likelihood
    with its gradient on 1024 x 4017; ``fused_large``: 8192 x linspace(10, 2048, 8192)), ``vjp`` (the FP32 backward on
    1024 x 4017), ``ragged`` (2048 binaries on their own grids), ``bank`` (the
    4096 XAS templates matched against one signal), ``xhm`` (IMRPhenomXHM's
    FP32 polarizations of 2048 binaries on the 4017 frequencies)."""
    import torch

    from waveformx_b200 import _lib, ops

    device = torch.device("cuda", 0)
    nb, grid = (1024, (20.0, 1024.0, 4017)) if args.profile_case in ("fused", "vjp") else (N_BATCH, GRID)
    if args.profile_case == "fused_large":
        nb, grid = 8192, (10.0, 2048.0, 8192)
    if args.profile_case == "xhm":
        nb = 2048
    p_np = draw_batch(np.random.default_rng(5), nb).astype(np.float32).astype(np.float64)
    p = torch.as_tensor(p_np, device=device)
    f_np = np.linspace(*grid).astype(np.float32)
    real = torch.float64 if args.profile_case == "forward64" else torch.float32
    precision = _lib.FP64 if args.profile_case == "forward64" else _lib.FP32
    freqs = torch.as_tensor(f_np, dtype=real, device=device)
    if args.profile_case in ("forward", "forward64"):
        def step():
            t = ops.setup("IMRPhenomXAS", p, freqs[:1].double(), precision=precision)
            ops.polarizations("IMRPhenomXAS", t.table, freqs)
    elif args.profile_case in ("fused", "fused_large", "vjp"):
        w = torch.as_tensor(1.0 / psd(f_np.astype(np.float64)), dtype=torch.float32, device=device)
        d = torch.zeros(grid[2], dtype=torch.complex64, device=device)
        tc = torch.zeros(nb, dtype=torch.float32, device=device)
        t = ops.setup("IMRPhenomXAS", p, freqs[:1].double(), precision=precision, jvp=True)
        cot = torch.ones((nb, grid[2]), dtype=torch.complex64, device=device)

        def step():
            if args.profile_case in ("fused", "fused_large"):
                ops.fused_loss("IMRPhenomXAS", t.table, t.dtable, freqs, None, tc, d, w)
            else:
                ops.vjp("IMRPhenomXAS", t.table, t.dtable, freqs, None, tc, cot, cot)
    elif args.profile_case == "xhm":
        t = ops.setup("IMRPhenomXHM", p, freqs[:1].double(), precision=precision)

        def step():
            ops.polarizations("IMRPhenomXHM", t.table, freqs)
    elif args.profile_case == "bank":
        from waveformx_b200 import match as wmatch

        f64 = np.linspace(*grid)
        w = torch.as_tensor(psd(f64), dtype=torch.float32, device=device)
        t0 = ops.setup("IMRPhenomXAS", p[:1], torch.as_tensor(f64[:1], device=device), precision=_lib.FP32)
        sig = ops.polarizations("IMRPhenomXAS", t0.table, freqs)[0][0].contiguous()

        def step():
            wmatch.template_match("IMRPhenomXAS", p, f64, sig, w)
    elif args.profile_case == "ragged":
        nb = 2048
        lengths = np.random.default_rng(1).integers(1000, 40000, nb)
        offsets_np = np.concatenate([[0], np.cumsum(lengths)])
        idx = np.arange(offsets_np[-1]) - np.repeat(offsets_np[:-1], lengths)
        flat = torch.as_tensor((20.0 + idx / 8.0).astype(np.float32), device=device)
        offsets = torch.as_tensor(offsets_np, device=device)
        pr = p[:nb]
        f_min = torch.full((nb,), 20.0, dtype=torch.float64, device=device)

        def step():
            t = ops.setup("IMRPhenomXAS", pr, f_min, precision=_lib.FP32)
            ops.polarizations("IMRPhenomXAS", t.table, flat, offsets)
    else:
        raise SystemExit(f"unknown profile case {args.profile_case!r}")
    for _ in range(args.warmup + args.steps):
        step()
    torch.cuda.synchronize()
    print(f"profile case {args.profile_case}: {args.warmup + args.steps} steps done")


def main():
    parser = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    parser.add_argument("--gpus", type=int, default=1)
    parser.add_argument("--steps", type=int, default=400)
    parser.add_argument("--warmup", type=int, default=5)
    parser.add_argument("--impl", choices=["b200", "reference"], default="b200")
    parser.add_argument("--quick", action="store_true", help="the headline only (no detail block)")
    parser.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    parser.add_argument("--cpu-seconds", type=float, default=10.0)
    parser.add_argument("--profile-case", default=None,
                        help="run one kernel family for a profiler and exit (forward, forward64, fused, fused_large, vjp, ragged, bank, xhm)")
    args = parser.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.profile_case:
        profile_case(args)
        return
    if args.impl == "reference":
        rank = int(os.environ.get("RANK", "0"))
        world = int(os.environ.get("WORLD_SIZE", "1"))
        line = reference_arm(args, rank, world)
        if line is not None:
            print(json.dumps(line), flush=True)
        return
    rank, world, local = init_dist()
    try:
        line = b200_arm(args, rank, world, local)
        if rank == 0:
            print(json.dumps(line), flush=True)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
