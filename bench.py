"""Benchmark: fwd+VJP events/s of the batched LOITS sampler on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload ragged|uniform|single|precision|tuple|gan] [--events E]

One step = forward (normalise, CDF, Philox, inverse-CDF search +
interpolation, stable compaction) + VJP of the whole density batch.  The
default workload is the ragged batch: 512 densities with knot counts
log-uniform in [64, 8192] and event counts log-uniform in [1e4, 1e6] (about
1.0e8 events per step), a per-density acceptance cut x > x_cut; seeded
synthetic densities (sums of 1-3 x^a (1-x)^b components), no dataset.

Arms:
  --impl b200       (default) the persistent form captured in one CUDA graph
                    (``value``); beside it the plain form -- one forward and
                    one backward launch per density, no graph -- with its own
                    tuned launch geometry, the saved-state form, and ``e2e``:
                    LOITS(backend="cuda")(DensityBatch, event_counts) +
                    autograd backward with host buffers.
  --impl reference  the reference's own openmp core (oracle/_ref, compiled
                    from the reference sources) on the host cores, on the exact
                    embedding of the same workload, a bounded sample per step.

Before timing, the launch geometry (threads per CTA, Philox blocks per thread,
CDF scan width) of each form is tuned on the workload itself by timing each
of its candidates (quantom_loits_b200.tuning; untimed, reported as
tuning_ms_per_step); --no-tune keeps the plan's default (CTA size by
occupancy); --threads/--blocks and --plain-threads/--plain-blocks fix them.

--workload uniform (64 x 1024 knots, 1e6 events each), single (1 x 256 knots,
1e5 events) and precision (16 x 2^20 knots, 1e7 events each) run the other
batch shapes; --workload gan runs batched GAN steps (generator MLP ->
power-law theory on 2048 knots -> 256 x 2e5 events binned into 64-bin
histograms in the sampler's kernels -> discriminator), the sampler's share of
the step reported; --workload tuple runs the reference's own 2-D theory tuple
at the scale of its GPU benchmark (99 x 99 cells, K = 10, 1e7 events; fp64,
bit-exact with the reference) through LOITS(backend="cuda"); its reference
arm is the reference's openmp core on the identical tuple.

--eager-steps K only runs K eager forward + backward launches of a batched
workload at a given geometry (the launches a profiler attaches to).

Under torchrun each rank (one GPU) samples its own copy-shaped share of a
global batch (density_base = rank * B, same Philox slot stride): weak
scaling, no collective on the data path; the step time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "fwd+VJP events/s on 1 B200 (batched vs plain), %HBM peak, CDF err vs FP64"
PEAKS = ROOT / "MEASURED_PEAKS.json"
TRAFFIC = ROOT / "profiles" / "traffic.json"
FALLBACK_HBM_GBS = 6650.0
# algorithmic bytes per kept event: the forward writes the event (4 B), the VJP
# reads its cotangent (4 B); the saved-state form (the default) also writes,
# and its VJP reads, the row's interval and offset (8 B); per knot the forward
# reads grid + value (8 B), the VJP reads them again and writes the gradient
# (12 B)
FWD_B_PER_EVENT, BWD_B_PER_EVENT, STATE_B_PER_EVENT = 4, 4, 8
FWD_B_PER_KNOT, BWD_B_PER_KNOT = 8, 12


def max_over_ranks(ms: float) -> float:
    from quantom_loits_b200.sharding import max_over_ranks as _max

    return _max(ms)


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def workload_spec(name: str, events: int = 0):
    from quantom_loits_b200 import workloads

    if name == "tuple":
        return workloads.theory_tuple(n_events=events or 10_000_000)
    return workloads.WORKLOADS[name]()


def describe(spec) -> dict:
    g = np.diff(spec.knot_offsets)
    return {"workload": spec.name, "densities": spec.n_densities,
            "knots_min": int(g.min()), "knots_max": int(g.max()),
            "events_per_step": spec.total_events,
            "x_cut": spec.x_cut is not None}


class ClockSampler:
    """SM clocks and throttle reasons sampled every ~2 ms during the timed
    region through NVML (read-only queries), nvidia-smi when NVML is absent.
    The device is found by its PCI address, so it is the GPU torch uses."""

    REASONS = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.samples: list[tuple[float, float, set]] = []
        self._stop = None
        self._thread = None
        self._proc = None
        self._path = None

    def _nvml_handle(self):
        import pynvml
        import torch

        pynvml.nvmlInit()
        p = torch.cuda.get_device_properties(self.index)
        bus = f"{p.pci_domain_id:08X}:{p.pci_bus_id:02X}:{p.pci_device_id:02X}.0"
        try:
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def __enter__(self):
        import threading

        try:
            nv, h = self._nvml_handle()
            bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                    "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                    "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                    "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
            mx = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self._stop = threading.Event()

            def poll():
                while not self._stop.is_set():
                    sm = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                    r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                    self.samples.append((sm, mx, {k for k, b in bits.items() if r & b}))
                    time.sleep(0.002)

            self._thread = threading.Thread(target=poll, daemon=True)
            self._thread.start()
            time.sleep(0.01)
        except Exception:
            self._start_smi()
        return self

    def _start_smi(self):
        import tempfile

        self._path = os.path.join(tempfile.gettempdir(), f"loits_bench_clocks_{os.getpid()}.csv")
        try:
            self._out = open(self._path, "w")
            self._proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self._out, stderr=subprocess.DEVNULL)
        except Exception:
            self._proc = None
        time.sleep(0.3)

    def __exit__(self, *exc):
        if self._thread is not None:
            self._stop.set()
            self._thread.join(timeout=5)
        if self._proc is not None:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except Exception:
                self._proc.kill()
            self._out.close()
            for line in open(self._path):
                f = line.split(",")
                if len(f) < 9 or not f[1].strip().replace(".", "").isdigit():
                    continue
                reasons = {self.REASONS[i] for i in range(4)
                           if "Active" in f[5 + i] and "Not" not in f[5 + i]}
                self.samples.append((float(f[1]), float(f[2]), reasons))

    def summary(self) -> dict:
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        reasons = sorted(set().union(*(r for _, _, r in self.samples)))
        return {"sm_mhz": statistics.median(s for s, _, _ in self.samples),
                "sm_max_mhz": max(m for _, m, _ in self.samples), "reasons": reasons,
                "samples": len(self.samples),
                "source": "nvml" if self._thread is not None else "nvidia-smi"}


def hbm_peak() -> tuple[float, str]:
    try:
        return float(json.loads(PEAKS.read_text())["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def cpu_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


# --------------------------------------------------------------- reference

def reference_sample(spec, n_dens: int):
    """The reference openmp core on the exact embedding of the first n_dens
    densities (full event counts).  Returns (events, seconds fwd+bwd)."""
    from oracle import oracle as O

    ref = O.Reference("openmp")
    ref.set_threads(cpu_cores())
    koff = spec.knot_offsets[:n_dens + 1]
    grid = spec.grid[:koff[-1]]
    values = spec.values[:koff[-1]]
    counts = spec.event_counts[:n_dens]
    *arrs, n_events = O.embed_densities(koff, grid, values, counts)
    t0 = time.perf_counter()
    st = ref.forward(*arrs, n_events, spec.seed, spec.sequence)
    g = np.zeros_like(st["events"])
    g[:, 0] = 1.0
    ref.backward(g, st, arrs[0], arrs[1], arrs[2], arrs[3], arrs[5])
    dt = time.perf_counter() - t0
    return int(counts.sum()), dt


# The reference's intervals are int16 (cpp/loits_core.cpp:12-18) and its
# search counts every knot per event: a 2^20-knot density is out of its range.
REFERENCE_INFEASIBLE = {
    "precision": "reference infeasible on this workload: its int16 intervals overflow at 2^20 "
                 "knots and its search is O(knots) per event (cpp/loits_core.cpp:12-18)",
}


def reference_timing(spec, seconds: float, warmup: int, repeats: int):
    """The one method both CPU legs use: calibrate on one density, take the
    first n densities that make about `seconds` of reference work, run that
    sample `warmup` times untimed and `repeats` times timed.  Returns
    (events/s of the mean timed run, n densities, events per run, mean s).
    The reference's search counts every knot, so a density's work is taken
    as its events times its knots."""
    _, t1 = reference_sample(spec, 1)
    knots = np.diff(np.asarray(spec.knot_offsets, np.int64)).astype(np.float64)
    work = np.cumsum(np.asarray(spec.event_counts, np.float64) * knots)

    def pick(target_work):
        return int(max(1, min(spec.n_densities, np.searchsorted(work, target_work, "right"))))

    n_dens = pick(seconds * work[0] / max(t1, 1e-6))
    # the untimed runs also refine the sample toward `seconds`
    for _ in range(max(warmup, 1)):
        _, t = reference_sample(spec, n_dens)
        n_dens = pick(work[n_dens - 1] * seconds / max(t, 1e-6))
    times, evs = [], 0
    for _ in range(max(repeats, 1)):
        ev, dt = reference_sample(spec, n_dens)
        times.append(dt)
        evs = ev
    t = float(np.mean(times))
    return evs / t, n_dens, evs, t


def reference_sample_text(spec, n_dens: int, evs: int, warmup: int, repeats: int) -> str:
    return (f"first {n_dens} of {spec.n_densities} densities ({evs} events) per run, exact "
            f"embedding into the reference tuple, reference openmp core on {cpu_cores()} "
            f"threads; forward + backward wall clock, mean of {repeats} runs after {warmup} "
            f"untimed")


def run_reference(args, spec) -> dict:
    if spec.name in REFERENCE_INFEASIBLE:
        return {"impl": "reference", "unavailable": REFERENCE_INFEASIBLE[spec.name],
                "metric": METRIC, "config": describe(spec)}
    warm = 1
    value, n_dens, evs, t = reference_timing(spec, args.ref_seconds, warm, args.steps)
    sample = reference_sample_text(spec, n_dens, evs, warm, args.steps)
    return {"metric": METRIC, "value": value, "unit": "events/s", "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": describe(spec),
            "cpu_baseline": {"value": value, "unit": "events/s", "cores": cpu_cores(),
                             "kind": "reference", "sample": sample},
            "e2e": {"value": value, "unit": "events/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


# ------------------------------------------------------------------- b200

def tune(spec, dev, args, plain: bool):
    """Launch geometry of the persistent form (plain=False) or of the
    one-launch-per-density form (plain=True), each timed on this rank's batch
    on its own candidates (untimed by the bench).  Returns (config dict,
    {candidate: ms})."""
    from quantom_loits_b200 import batched as B
    from quantom_loits_b200.tuning import CANDIDATES, PLAIN_CANDIDATES, Autotuner

    threads, blocks = (args.plain_threads, args.plain_blocks) if plain else (args.threads,
                                                                              args.blocks)
    base = {"guide_ratio": args.guide_ratio}
    if plain:
        base["plain"] = 1
    if threads or blocks or args.no_tune:
        return dict(base, threads=threads, blocks_per_item=blocks, scan_knots=0), None
    tbatch = B.DensityBatch.from_spec(spec, dev)
    tuner = Autotuner(dev, candidates=PLAIN_CANDIDATES if plain else CANDIDATES, base=base,
                      saved_state=True, buckets=not args.no_bucket_tune)
    best, times = tuner.tune(tbatch, spec.event_counts, spec.seed, 0)
    return best, times


def make_step(spec, dev, geom, rank, saved_state=False):
    from quantom_loits_b200 import batched as B
    from quantom_loits_b200.tuning import density_tables, plain_config

    nmax = int(spec.event_counts.max())
    cfg = B.make_config(**plain_config(geom), density_base=rank * spec.n_densities,
                        slot_stride=nmax)
    blocks, scan = density_tables(spec.knot_offsets, geom)
    plan = B.BatchPlan(spec.knot_offsets, spec.event_counts, cfg, dev, density_blocks=blocks,
                       density_scan=scan)
    step = B.BatchStep(plan, seed=spec.seed, with_cut=spec.x_cut is not None,
                       saved_state=saved_state)
    step.grid.copy_(torch_from(spec.grid))
    step.values.copy_(torch_from(spec.values))
    if spec.x_cut is not None:
        step.x_cut.copy_(torch_from(spec.x_cut))
    return plan, step


def torch_from(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a))


def time_steps(step, steps, barrier, stream) -> float:
    """ms per step of `steps` back-to-back steps (graph replays when
    captured), device-timed with CUDA events between barriers."""
    import torch

    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    t0.record(stream)
    for _ in range(steps):
        step.step()
    t1.record(stream)
    barrier()
    return t0.elapsed_time(t1) / steps


def time_kernels(step, steps, stream) -> tuple[float, float]:
    """Mean device time of the forward launch and of the backward launch."""
    import torch

    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    fwd, bwd = [], []
    for _ in range(steps):
        ev[0].record(stream)
        step.forward()
        ev[1].record(stream)
        step.backward()
        ev[2].record(stream)
        ev[2].synchronize()
        fwd.append(ev[0].elapsed_time(ev[1]))
        bwd.append(ev[1].elapsed_time(ev[2]))
    return float(np.mean(fwd)), float(np.mean(bwd))


def run_b200(args, spec, rank, world, dist) -> dict:
    import torch

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream(dev)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(dev)

    # ---- launch geometries: each form tuned on its own candidates
    geom, tune_ms = tune(spec, dev, args, plain=False)
    pgeom, ptune_ms = tune(spec, dev, args, plain=True)
    args.geom = geom
    # the measured form: saved state (the forward keeps each kept row's
    # interval and offset, the backward reads them), persistent kernels
    plan, step = make_step(spec, dev, geom, rank, saved_state=True)
    gen = torch.Generator(device=dev).manual_seed(1000 + rank)
    step.grad_events.normal_(generator=gen)

    # ---- per-kernel durations (forward and backward launches, eager)
    for _ in range(max(args.warmup, 3)):
        step.forward()
        step.backward()
    torch.cuda.synchronize(dev)
    step.check_status()
    f_ms, b_ms = time_kernels(step, args.steps, stream)

    # ---- batched form: persistent kernels, forward + backward in one graph
    step.capture()
    for _ in range(args.warmup):
        step.step()
    with ClockSampler(dev.index) as clocks:
        ms = time_steps(step, args.steps, barrier, stream)
    step.check_status()
    if dist is not None:
        ms = max_over_ranks(ms)
    events_step = spec.total_events * world
    value = events_step / (ms * 1e-3)
    valid = int(step.row_offsets[-1].item())

    # ---- plain form: one forward and one backward launch per density, its
    # own tuned geometry, saved state, no graph
    pplan, pstep = make_step(spec, dev, pgeom, rank, saved_state=True)
    pstep.grad_events.copy_(step.grad_events)
    for _ in range(args.warmup):
        pstep.step()
    plain_ms = time_steps(pstep, args.steps, barrier, stream)
    pstep.check_status()
    if dist is not None:
        plain_ms = max_over_ranks(plain_ms)
    same = torch.equal(pstep.events[:valid], step.events[:valid])
    plain_rows_same = torch.equal(pstep.row_offsets, step.row_offsets)
    plain_launch = pplan.config
    del pstep, pplan

    # ---- replay form: no per-row state; the backward regenerates the
    # uniforms, intervals and compaction ranks
    rplan, rstep = make_step(spec, dev, geom, rank, saved_state=False)
    rstep.grad_events.copy_(step.grad_events)
    for _ in range(max(args.warmup, 3)):
        rstep.step()
    torch.cuda.synchronize(dev)
    rstep.check_status()
    r_fwd, r_bwd = time_kernels(rstep, args.steps, stream)
    rstep.capture()
    for _ in range(args.warmup):
        rstep.step()
    replay_ms = time_steps(rstep, args.steps, barrier, stream)
    rstep.check_status()
    if dist is not None:
        replay_ms = max_over_ranks(replay_ms)
    gscale = float(step.grad_values.abs().max().item()) or 1.0
    replay = {
        "value": events_step / (replay_ms * 1e-3), "ms_per_step": replay_ms,
        "kernels_ms": {"batch_forward_kernel": r_fwd, "batch_backward_kernel": r_bwd},
        "form": "no per-row state: the backward regenerates uniforms, intervals and "
                "compaction ranks from (seed, sequence); one CUDA graph",
        "events_identical": bool(torch.equal(rstep.events[:valid], step.events[:valid])),
        "grad_max_diff_over_scale": float((rstep.grad_values - step.grad_values).abs().max()
                                          .item()) / gscale,
    }
    rstep.graph = None
    del rstep, rplan

    # ---- end to end through LOITS(backend="cuda") with host buffers
    e2e = run_e2e(args, spec, dev, rank, world, dist)

    # ---- roofline of the dominant kernel
    knots = spec.total_knots
    fwd_bytes = (FWD_B_PER_EVENT + STATE_B_PER_EVENT) * valid + FWD_B_PER_KNOT * knots
    bwd_bytes = (BWD_B_PER_EVENT + STATE_B_PER_EVENT) * valid + BWD_B_PER_KNOT * knots
    kname, k_ms, k_bytes = (("batch_forward_kernel", f_ms, fwd_bytes) if f_ms >= b_ms
                            else ("batch_backward_kernel", b_ms, bwd_bytes))
    peak, peak_kind = hbm_peak()
    achieved = k_bytes / (k_ms * 1e-3) / 1e9
    traffic = None
    try:
        t = json.loads(TRAFFIC.read_text())
        entry = t.get(spec.name + "_state", {}).get(kname)
        if entry:
            # measured on this workload; scaled by kept events if they differ
            traffic = entry["bytes_per_launch"] * valid / entry["kept_events"]
    except Exception:
        pass
    precision = precision_report(plan, step, spec) if rank == 0 else None
    step.graph = None

    out = {
        "metric": METRIC, "value": value, "unit": "events/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {**describe(spec),
                   "form": "persistent forward + backward, saved state (interval and offset "
                           "per kept row, 8 B), one CUDA graph",
                   "parallelism": f"density-sharded x{world} (no collective on the data path)",
                   "l2": f"per step {12 * valid / 1e6:.0f} MB of events and state written "
                         f"and {12 * valid / 1e6:.0f} MB of cotangents and state read, each "
                         "larger than the 126 MB L2 (no flush)" if 4 * valid > 126e6 else
                         "inputs smaller than L2: not a valid roofline case",
                   "launch": plan.config, "accepted_events_per_step": valid * world,
                   "bucket_tables": {k: geom.get(k) for k in ("bucket_blocks", "bucket_scan")},
                   "tuning_ms_per_step": tune_ms},
        "plain": {"value": events_step / (plain_ms * 1e-3), "ms_per_step": plain_ms,
                  "form": "one forward + one backward launch per density, saved state, "
                          "no graph",
                  "launch": plain_launch, "tuning_ms_per_step": ptune_ms,
                  "batched_over_plain": plain_ms / ms, "events_identical": bool(same),
                  "row_offsets_identical": bool(plain_rows_same)},
        "kernels_ms": {"batch_forward_kernel": f_ms, "batch_backward_kernel": b_ms},
        "replay": replay,
        "roofline": {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic,
                     "algorithmic_bytes": k_bytes},
        "step_hbm_frac": (fwd_bytes + bwd_bytes) / (ms * 1e-3) / 1e9 / peak,
        "cdf_err_vs_fp64": None if precision is None else precision.get("cdf_err"),
        "precision": precision,
        "e2e": e2e,
        "gpu_launches": 2 * args.steps,
        "clocks": clocks.summary(),
    }
    return out


def run_eager(args, spec) -> dict:
    """--eager-steps K: K eager forward + backward launches of the persistent
    form on one GPU at a given geometry, untimed -- the launches a profiler
    attaches to.  Prints the kept-row count and the resolved launch."""
    import torch

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    geom = dict(threads=args.threads, blocks_per_item=args.blocks, scan_knots=args.scan_knots,
                guide_ratio=args.guide_ratio, plain=1 if args.plain else 0)
    plan, step = make_step(spec, dev, geom, 0, saved_state=args.saved_state)
    step.grad_events.normal_(generator=torch.Generator(device=dev).manual_seed(0))
    for _ in range(args.eager_steps):
        step.forward()
        step.backward()
    torch.cuda.synchronize(dev)
    step.check_status()
    return {"workload": spec.name, "eager_steps": args.eager_steps,
            "events": spec.total_events, "knots": spec.total_knots,
            "kept": int(step.row_offsets[-1].item()), "launch": plan.config}


def precision_report(plan, step, spec, n_check: int = 2) -> dict:
    """Accuracy against the fp64 oracle, outside the timed region:
    max |CDF - oracle CDF| over every knot; max relative event-quantile error
    at p = 1e-6, 0.5, 1 - 1e-6 over every density; and, over the first
    n_check densities' events, the intervals that differ from the oracle's
    (bin flips) and how many of those lie farther than 2 ulp from a knot."""
    import torch

    try:
        from oracle import oracle as O

        ora = O.Oracle()
        cdf, _ = plan.cdf(step.workspace)
        _, ocdf, _ = ora.d_cdf(spec.knot_offsets, spec.grid, spec.values)
        rep = {"cdf_err": float(np.abs(cdf.cpu().numpy() - ocdf).max())}
        p = np.array([1e-6, 0.5, 1 - 1e-6], dtype=np.float32)
        qerr = np.zeros(3)
        for b in range(spec.n_densities):
            x, _ = plan.quantile(step.workspace, b, torch.from_numpy(p))
            xo, _ = ora.d_quantile(b, spec.knot_offsets, spec.grid, ocdf, p.astype(np.float64))
            qerr = np.maximum(qerr, np.abs(x.cpu().numpy() - xo) / np.maximum(np.abs(xo), 1e-30))
        rep["quantile_rel_err"] = {"1e-6": float(qerr[0]), "0.5": float(qerr[1]),
                                   "1-1e-6": float(qerr[2])}
        # intervals of the first n_check densities against the oracle's
        nd = min(n_check, spec.n_densities)
        ints = torch.full((max(plan.capacity, 1),), -1, dtype=torch.int32, device=step.events.device)
        plan.forward(step.grid, step.values, step.x_cut, step.seed, step.sequence, step.events,
                     step.row_offsets, step.workspace, ints)
        rows = step.row_offsets.cpu().numpy()
        koff = spec.knot_offsets[:nd + 1]
        counts = spec.event_counts[:nd]
        ref = ora.d_forward(koff, np.concatenate([[0], np.cumsum(counts)]),
                            spec.grid[:koff[-1]], spec.values[:koff[-1]],
                            None if spec.x_cut is None else spec.x_cut[:nd], step.seed,
                            step.sequence, 0, int(spec.event_counts.max()))
        mine = ints[:rows[nd]].cpu().numpy()
        diff = np.flatnonzero(mine != ref["intervals"])
        far = 0
        for r in diff:
            b = int(np.searchsorted(ref["row_offsets"], r, side="right") - 1)
            c = ref["cdf"][koff[b]:koff[b + 1]]
            u = np.float32(ref["u"][r])
            i = int(np.searchsorted(c, float(u)))
            gap = min(abs(float(u) - c[max(i - 1, 0)]), abs(float(u) - c[min(i, len(c) - 1)]))
            far += gap > 2 * max(float(np.spacing(u)), 2.0 ** -24)
        rep.update({"flips": int(len(diff)), "flips_far_from_knot": int(far),
                    "checked_events": int(len(mine)), "checked_densities": nd})
        return rep
    except Exception as exc:  # pragma: no cover
        return {"unavailable": str(exc)}


def run_e2e(args, spec, dev, rank, world, dist) -> dict:
    """The user-facing call with host data: pinned host -> device copies of the
    step's inputs (density values, grid, cut, cotangent),
    ``LOITS(backend="cuda")(DensityBatch, event_counts)`` + autograd backward,
    device -> host copies of the events and the gradient.  The cotangent's copy
    in and the events' copy out run on their own streams (opposite PCIe
    directions) beside the forward; the backward waits for the cotangent and
    the step ends when events and gradient are on the host."""
    import torch

    from quantom_loits_b200 import batched as B
    from quantom_loits_b200.loits import LOITS

    nmax = int(spec.event_counts.max())
    # the tuned geometry (with its per-bucket tables) as the sampler's config
    cfg = dict(args.geom, density_base=rank * spec.n_densities, slot_stride=nmax)
    sampler = LOITS(backend="cuda", device=dev, batch_config=cfg)
    h_vals = torch_from(spec.values).pin_memory()
    h_grid = torch_from(spec.grid).pin_memory()
    h_cut = None if spec.x_cut is None else torch_from(spec.x_cut).pin_memory()
    h_cot = torch.randn(spec.total_events, generator=torch.Generator().manual_seed(5)).pin_memory()
    h_events = torch.empty(spec.total_events, dtype=torch.float32).pin_memory()
    h_grad = torch.empty(spec.total_knots, dtype=torch.float32).pin_memory()
    stream = torch.cuda.current_stream(dev)
    s_in, s_out = torch.cuda.Stream(dev), torch.cuda.Stream(dev)

    def one():
        s_in.wait_stream(stream)
        with torch.cuda.stream(s_in):
            cot = h_cot.to(dev, non_blocking=True)
        cot.record_stream(stream)
        values = h_vals.to(dev, non_blocking=True).requires_grad_(True)
        grid = h_grid.to(dev, non_blocking=True)
        cut = None if h_cut is None else h_cut.to(dev, non_blocking=True)
        batch = B.DensityBatch(grid, values, spec.knot_offsets, spec.event_counts, cut)
        events, rows = sampler(batch, spec.event_counts)
        n = events.shape[0]
        s_out.wait_stream(stream)
        with torch.cuda.stream(s_out):
            h_events[:n].copy_(events.detach(), non_blocking=True)
        events.record_stream(s_out)
        stream.wait_stream(s_in)
        events.backward(cot[:n])
        h_grad.copy_(values.grad, non_blocking=True)
        stream.wait_stream(s_out)
        return n

    for _ in range(max(2, args.warmup // 2)):
        one()
    torch.cuda.synchronize(dev)
    if dist is not None:
        dist.barrier()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    steps = max(3, args.steps // 2)
    t0.record(stream)
    n = 0
    for _ in range(steps):
        n = one()
    t1.record(stream)
    torch.cuda.synchronize(dev)
    ms = t0.elapsed_time(t1) / steps
    if dist is not None:
        ms = max_over_ranks(ms)
    h2d = 4 * (spec.total_knots * 2 + spec.total_events + (spec.n_densities if h_cut is not None else 0))
    d2h = 4 * (n + spec.total_knots)
    return {"value": spec.total_events * world / (ms * 1e-3), "unit": "events/s",
            "ms_per_step": ms, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
            "api": "LOITS(backend='cuda')(DensityBatch, event_counts) + autograd backward"}


def tuple_cpu_baseline(args, spec) -> dict:
    """The reference openmp core on the same tuple, rank 0 / N=1 only."""
    try:
        from oracle import oracle as O

        ref = O.Reference("openmp")
        ref.set_threads(cpu_cores())
        reference_tuple_step(ref, spec)
        dt = float(np.mean([reference_tuple_step(ref, spec) for _ in range(3)]))
        return {"value": spec.n_events / dt, "unit": "events/s", "cores": cpu_cores(),
                "kind": "reference",
                "sample": f"the whole tuple workload ({spec.n_events} events), reference openmp "
                          "core, forward + backward wall clock, mean of 3"}
    except Exception as exc:
        return {"value": None, "unit": "events/s", "cores": cpu_cores(), "kind": "reference",
                "sample": f"unavailable: {exc}"}


def cpu_baseline_leg(args, spec) -> dict:
    """The reference openmp core on a bounded sample, rank 0 / N=1 only: the
    reference arm's own method (reference_timing), three timed runs."""
    if spec.name in REFERENCE_INFEASIBLE:
        return {"value": None, "unit": "events/s", "cores": cpu_cores(), "kind": "reference",
                "sample": REFERENCE_INFEASIBLE[spec.name]}
    try:
        warm, reps = 1, 3
        value, n_dens, evs, _ = reference_timing(spec, args.ref_seconds, warm, reps)
        return {"value": value, "unit": "events/s", "cores": cpu_cores(), "kind": "reference",
                "sample": reference_sample_text(spec, n_dens, evs, warm, reps)}
    except Exception as exc:
        return {"value": None, "unit": "events/s", "cores": cpu_cores(), "kind": "reference",
                "sample": f"unavailable: {exc}"}


# ------------------------------------------------------------------ tuple

TUPLE_B_PER_EVENT = 24  # events (2 x fp64) + packed slot (int64) out; cotangent + slot in


def describe_tuple(spec) -> dict:
    B, nx, kx = spec.x_bins.shape
    return {"workload": "tuple", "batch": B, "cells": spec.cells, "knots": kx,
            "n_events": spec.n_events, "layout": "reference theory tuple, fp64"}


def reference_tuple_step(ref, spec):
    t0 = time.perf_counter()
    st = ref.forward(*spec.arrays, spec.n_events, spec.seed, spec.sequence)
    g = np.ones_like(st["events"])
    ref.backward(g, st, spec.x_bins, spec.xsec_x, spec.q_bins, spec.xsec_q, spec.acceptance)
    return time.perf_counter() - t0


def run_tuple_reference(args, spec) -> dict:
    from oracle import oracle as O

    ref = O.Reference("openmp")
    ref.set_threads(cpu_cores())
    for _ in range(args.warmup):
        reference_tuple_step(ref, spec)
    t = float(np.mean([reference_tuple_step(ref, spec) for _ in range(args.steps)]))
    value = spec.n_events / t
    sample = (f"the whole tuple workload ({spec.cells} cells, {spec.n_events} events) per step, "
              "reference openmp core, forward + backward wall clock")
    return {"metric": METRIC, "value": value, "unit": "events/s", "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": describe_tuple(spec),
            "cpu_baseline": {"value": value, "unit": "events/s", "cores": cpu_cores(),
                             "kind": "reference", "sample": sample},
            "e2e": {"value": value, "unit": "events/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def run_tuple_b200(args, spec, rank, world, dist) -> dict:
    """The reference tuple through the CUDA backend (replicas under torchrun:
    rank r samples sequence r, no collective on the data path)."""
    import torch

    from quantom_loits_b200 import backend as BK
    from quantom_loits_b200.loits import LOITS

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    seq = spec.sequence + rank
    t = [torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in spec.arrays]
    stream = torch.cuda.current_stream(dev)
    gen = torch.Generator(device=dev).manual_seed(7)

    def step():
        ev, st = BK.tuple_forward(*t, spec.n_events, spec.seed, seq)
        g = torch.randn(ev.shape, generator=gen, device=dev, dtype=torch.float64)
        BK.tuple_backward(g, t[0], t[1], t[2], t[3], t[5], st, spec.seed, seq)
        return ev

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    ev3 = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    f_ms, b_ms = [], []
    for _ in range(args.steps):
        ev3[0].record(stream)
        ev, st = BK.tuple_forward(*t, spec.n_events, spec.seed, seq)
        ev3[1].record(stream)
        g = torch.ones(ev.shape, device=dev, dtype=torch.float64)
        BK.tuple_backward(g, t[0], t[1], t[2], t[3], t[5], st, spec.seed, seq)
        ev3[2].record(stream)
        ev3[2].synchronize()
        f_ms.append(ev3[0].elapsed_time(ev3[1]))
        b_ms.append(ev3[1].elapsed_time(ev3[2]))
    valid = int(ev.shape[0])
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize(dev)
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # eager form: the reference call's shape, two host round trips per forward
    t0.record(stream)
    for _ in range(args.steps):
        step()
    t1.record(stream)
    torch.cuda.synchronize(dev)
    eager_ms = t0.elapsed_time(t1) / args.steps
    if dist is not None:
        eager_ms = max_over_ranks(eager_ms)
    # measured form: forward + backward captured in one CUDA graph, counts
    # kept on the device (TupleStep)
    tstep = BK.TupleStep(*t, spec.n_events, spec.seed, seq)
    tstep.grad_events.normal_(generator=gen)
    tstep.capture()
    for _ in range(args.warmup):
        tstep.step()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize(dev)
    with ClockSampler(dev.index) as clocks:
        t0.record(stream)
        for _ in range(args.steps):
            tstep.step()
        t1.record(stream)
        torch.cuda.synchronize(dev)
    tstep.check_status()
    ms = t0.elapsed_time(t1) / args.steps
    if dist is not None:
        ms = max_over_ranks(ms)
    graph_same = bool(torch.equal(tstep.result()[0], ev))
    tstep.graph = None
    del tstep
    value = spec.n_events * world / (ms * 1e-3)

    # end to end through LOITS(backend="cuda") with host buffers
    h = [torch.from_numpy(np.ascontiguousarray(a)).pin_memory() for a in spec.arrays]
    h_cot = torch.randn((spec.n_events, 2), dtype=torch.float64,
                        generator=torch.Generator().manual_seed(3)).pin_memory()
    h_events = torch.empty((spec.n_events, 2), dtype=torch.float64).pin_memory()
    h_gx = torch.empty(spec.xsec_x.shape, dtype=torch.float64).pin_memory()
    h_gq = torch.empty(spec.xsec_q.shape, dtype=torch.float64).pin_memory()
    sampler = LOITS(backend="cuda", device=dev)
    s_in = torch.cuda.Stream(dev)

    def one():
        s_in.wait_stream(stream)
        with torch.cuda.stream(s_in):
            cot = h_cot.to(dev, non_blocking=True)
        cot.record_stream(stream)
        d = [x.to(dev, non_blocking=True) for x in h]
        d[1].requires_grad_(True)
        d[3].requires_grad_(True)
        events = sampler(tuple(d), spec.n_events)
        n = events.shape[0]
        h_events[:n].copy_(events.detach(), non_blocking=True)
        stream.wait_stream(s_in)
        events.backward(cot[:n])
        h_gx.copy_(d[1].grad, non_blocking=True)
        h_gq.copy_(d[3].grad, non_blocking=True)
        return n

    for _ in range(max(2, args.warmup // 2)):
        one()
    torch.cuda.synchronize(dev)
    e_steps = max(3, args.steps // 2)
    t0.record(stream)
    for _ in range(e_steps):
        n = one()
    t1.record(stream)
    torch.cuda.synchronize(dev)
    e_ms = t0.elapsed_time(t1) / e_steps
    if dist is not None:
        e_ms = max_over_ranks(e_ms)
    h2d = sum(int(a.nbytes) for a in spec.arrays) + n * 16
    d2h = n * 16 + int(spec.xsec_x.nbytes + spec.xsec_q.nbytes)

    fm, bm = float(np.mean(f_ms)), float(np.mean(b_ms))
    kname, k_ms = (("tuple_prepare+tuple_sample", fm) if fm >= bm else ("tuple_backward", bm))
    peak, peak_kind = hbm_peak()
    k_bytes = TUPLE_B_PER_EVENT * valid
    achieved = k_bytes / (k_ms * 1e-3) / 1e9
    traffic = None
    try:
        entry = json.loads(TRAFFIC.read_text()).get("tuple", {}).get(kname)
        if entry:
            traffic = entry["bytes_per_launch"] * valid / entry["kept_events"]
    except Exception:
        pass
    out = {
        "metric": METRIC, "value": value, "unit": "events/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {**describe_tuple(spec), "accepted_events_per_step": valid * world,
                   "parallelism": f"replicas x{world} (sequence = rank)",
                   "l2": "events + cotangent " + ("larger" if 32 * valid > 126e6 else "smaller")
                         + " than the 126 MB L2 (no flush)"},
        "kernels_ms": {"forward (prepare + sample)": fm, "backward": bm},
        "form": "TupleStep: prepare + bounded sample + backward in one CUDA graph, counts on "
                "the device",
        "eager": {"value": spec.n_events * world / (eager_ms * 1e-3), "ms_per_step": eager_ms,
                  "form": "tuple_forward + tuple_backward, two host round trips per forward",
                  "graph_events_identical": graph_same},
        "roofline": {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "algorithmic_bytes": k_bytes},
        "e2e": {"value": spec.n_events * world / (e_ms * 1e-3), "unit": "events/s",
                "ms_per_step": e_ms, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "api": "LOITS(backend='cuda')(theory_outputs, n_events) + autograd backward"},
        # per step: prepare (2 kernels), sample (1), backward (4)
        "gpu_launches": 7 * args.steps,
        "clocks": clocks.summary(),
    }
    if rank == 0:
        out["parity"] = tuple_parity(spec, t, dev)
    return out


def tuple_parity(spec, t, dev) -> dict:
    """The sampler's events against the oracle's restatement of the reference
    core on the same tuple, seed and sequence (bit-exact expected)."""
    try:
        from oracle import oracle as O
        from quantom_loits_b200 import backend as BK

        ev, st = BK.tuple_forward(*t, spec.n_events, spec.seed, spec.sequence)
        ref = O.Oracle().r_forward(*spec.arrays, spec.n_events, spec.seed, spec.sequence)
        mine = ev.cpu().numpy()
        same = mine.shape == ref["events"].shape and bool(np.array_equal(mine, ref["events"]))
        return {"events_bit_exact": same, "valid": int(mine.shape[0]),
                "packed_equal": bool(np.array_equal(st["packed"].cpu().numpy(), ref["packed"]))}
    except Exception as exc:  # pragma: no cover
        return {"unavailable": str(exc)}


# -------------------------------------------------------------------- gan

def describe_gan(tr) -> dict:
    return {"workload": "gan", "densities": tr.batch, "knots": int(tr.theory.grid.numel()),
            "events_per_density": tr.n_events, "bins": tr.bins, "latent": tr.latent,
            "sampler_calls_per_step": "2 forward (discriminator + generator step) + 1 VJP",
            "generator": "64-256-256-6 SiLU bf16", "discriminator": "64-256-1 SiLU"}


def run_gan_b200(args, rank, world, dist) -> dict:
    """Config 4: batched GAN steps (replicas under torchrun: rank r seeds r)."""
    import torch

    from quantom_loits_b200.gan import BatchedGANTrainer

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    # the sampler's launch geometry: tuned on the batch (config="auto") unless
    # --threads / --blocks name one
    if args.threads or args.blocks:
        from quantom_loits_b200.batched import make_config

        config = make_config(threads=args.threads, blocks_per_item=args.blocks)
    else:
        config = "auto"
    tr = BatchedGANTrainer(dev, seed=rank, config=config)
    tr.capture()  # the whole step as one CUDA graph
    stream = torch.cuda.current_stream(dev)
    for _ in range(args.warmup):
        tr.step()
    torch.cuda.synchronize(dev)
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev.index) as clocks:
        if dist is not None:
            dist.barrier()
        t0.record(stream)
        for _ in range(args.steps):
            d_loss, g_loss = tr.step()
        t1.record(stream)
        torch.cuda.synchronize(dev)
    ms = t0.elapsed_time(t1) / args.steps
    if dist is not None:
        ms = max_over_ranks(ms)
    # the sampler alone on the same shapes: 2 histogram forwards + 1 VJP (with
    # the theory evaluated inside it, as the step runs it)
    params = tr.generator(tr.latent_noise()).detach().requires_grad_(True)
    w = torch.randn((tr.batch, tr.bins), device=dev)

    def sampler_only():
        with torch.no_grad():
            tr.generate_from(params)
        (tr.generate_from(params) * w).sum().backward()

    for _ in range(3):
        sampler_only()
    torch.cuda.synchronize(dev)
    t0.record(stream)
    for _ in range(args.steps):
        sampler_only()
    t1.record(stream)
    torch.cuda.synchronize(dev)
    s_ms = t0.elapsed_time(t1) / args.steps
    # end to end: latent noise from pinned host memory, losses read back
    h_z = torch.randn((2, tr.batch, tr.latent), generator=torch.Generator().manual_seed(1)).pin_memory()
    h_loss = torch.empty(2).pin_memory()

    def one():
        z = h_z.to(dev, non_blocking=True)
        d_l, g_l = tr.step(z[0], z[1])
        h_loss.copy_(torch.stack([d_l, g_l]), non_blocking=True)

    for _ in range(2):
        one()
    torch.cuda.synchronize(dev)
    t0.record(stream)
    for _ in range(args.steps):
        one()
    t1.record(stream)
    torch.cuda.synchronize(dev)
    e_ms = t0.elapsed_time(t1) / args.steps
    if dist is not None:
        e_ms = max_over_ranks(e_ms)
    ev_step = 2 * tr.batch * tr.n_events
    return {
        "metric": METRIC, "value": ev_step * world / (ms * 1e-3), "unit": "events/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {**describe_gan(tr), "events_per_step": ev_step,
                   "parallelism": f"replicas x{world}", "form": "whole step in one CUDA graph",
                   "launch": next(iter(tr.sampler._plans.values())).config
                   if tr.sampler._plans else None},
        "gan": {"steps_per_s": 1e3 / ms, "sampler_ms_per_step": s_ms,
                "sampler_share": s_ms / ms, "d_loss": float(d_loss), "g_loss": float(g_loss)},
        "e2e": {"value": ev_step * world / (e_ms * 1e-3), "unit": "events/s", "ms_per_step": e_ms,
                "h2d_bytes_per_step": int(h_z.nbytes), "d2h_bytes_per_step": int(h_loss.nbytes),
                "api": "BatchedGANTrainer.step"},
        # per step: theory x2, theory VJP, histogram forward x2, histogram VJP
        "gpu_launches": 6 * args.steps,
        "clocks": clocks.summary(),
        "cpu_baseline": {"value": None, "unit": "events/s", "cores": cpu_cores(),
                         "kind": "reference", "sample": GAN_NO_REFERENCE},
    }


GAN_NO_REFERENCE = ("no reference counterpart: the reference GAN (pytorch/gan.py) trains one "
                    "2-D theory on raw events; the batched histogram GAN step has no CPU path "
                    "in the reference")


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--workload",
                    choices=["ragged", "uniform", "single", "precision", "tuple", "gan"],
                    default="ragged")
    ap.add_argument("--events", type=int, default=0,
                    help="events per step of the tuple workload (default 1e7)")
    ap.add_argument("--threads", type=int, default=0,
                    help="threads per CTA of the persistent form (0: tuned)")
    ap.add_argument("--blocks", type=int, default=0,
                    help="Philox blocks per thread per tile of the persistent form (0: tuned)")
    ap.add_argument("--plain-threads", type=int, default=0,
                    help="threads per CTA of the one-launch-per-density form (0: tuned)")
    ap.add_argument("--plain-blocks", type=int, default=0,
                    help="Philox blocks per thread per tile of that form (0: tuned)")
    ap.add_argument("--scan-knots", type=int, default=0)
    ap.add_argument("--guide-ratio", type=int, default=0,
                    help="log2 guide buckets per knot of small densities (0: default)")
    ap.add_argument("--eager-steps", type=int, default=0,
                    help="only run this many eager forward + backward launches (for a profiler)")
    ap.add_argument("--plain", action="store_true", help="--eager-steps: the plain form")
    ap.add_argument("--saved-state", action="store_true", help="--eager-steps: saved-state form")
    ap.add_argument("--ref-seconds", type=float, default=3.0,
                    help="CPU seconds per reference step (bounded sample)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-tune", action="store_true",
                    help="use the plan's default launch geometry instead of tuning it")
    ap.add_argument("--no-bucket-tune", action="store_true",
                    help="tune one launch geometry for the whole batch, not per grid-size bucket")
    args = ap.parse_args(argv)
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    world, rank, local = dist_env()
    is_tuple, is_gan = args.workload == "tuple", args.workload == "gan"
    spec = None if is_gan else workload_spec(args.workload, args.events)
    if args.eager_steps:
        if is_tuple or is_gan:
            ap.error("--eager-steps runs the batched workloads")
        print(json.dumps(run_eager(args, spec)), flush=True)
        return 0

    if args.impl == "reference":
        if rank != 0:
            return 0
        if is_gan:
            out = {"impl": "reference", "unavailable": GAN_NO_REFERENCE, "metric": METRIC,
                   "config": {"workload": "gan"}}
        else:
            out = run_tuple_reference(args, spec) if is_tuple else run_reference(args, spec)
        print(json.dumps(out), flush=True)
        return 0

    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as tdist

        torch.cuda.set_device(local)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                 device_id=torch.device("cuda", local))
        dist = tdist
    try:
        if is_gan:
            out = run_gan_b200(args, rank, world, dist)
        elif is_tuple:
            out = run_tuple_b200(args, spec, rank, world, dist)
        else:
            out = run_b200(args, spec, rank, world, dist)
        if rank == 0:
            if world == 1 and not args.no_cpu_baseline and not is_gan:
                out["cpu_baseline"] = (tuple_cpu_baseline(args, spec) if is_tuple
                                       else cpu_baseline_leg(args, spec))
            print(json.dumps(out), flush=True)
    finally:
        if dist is not None:
            dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
