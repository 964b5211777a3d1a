#!/usr/bin/env python3
"""Benchmark of the streamline-tracking hot path on B200.

Workload (single GPU): the plain Diffusion configuration -- a synthetic
145 x 174 x 145 spherical-harmonic FOD (lmax 8, 45 float32 coefficients,
1.25 mm voxels, about 660 MB), seeds drawn by ``seeds.from_fod`` with a
fixed NumPy seed, Diffusion with step 0.001 mm, gamma 1, noise variance 0.1,
save_at 0.25 mm, maximum length 300 mm, 1 000 000 seeds in batches of
50 000.  One benchmark step is the whole job, i.e. one
``tg.tractogram(fod, seeds, algorithm=..., batch_size=50000)`` call: every
batch keeps its own reference RNG seed and stream ids, and all batches run
in one persistent launch (a 50 000-seed batch alone cannot fill the ~95 000
resident lanes of a B200).

Metric: streamline-steps/s, where a step is one iteration of the tracking
loop that passed both the domain and the field check (tracking.py:121-147).

Reported:
  value     device-resident throughput: seeds already in HBM, one
            persistent-tracker run per job, packed output left on the
            device, one job at a time; CUDA events on the run's stream, max
            over ranks.  ``--in-flight N`` keeps N jobs in flight instead,
            each slot with its own stream and tracker (events spanning every
            stream); the one-at-a-time figure is then reported as
            single_job.  (Measured: a second job in flight overlaps one
            job's copies with the other's tracking, but the finished job's
            offsets scan and gather wait for the next job's persistent warps
            to leave, and the device-resident rate varied from equal to 7 %
            below the one-at-a-time rate.)
  e2e       the same metric through the C ABI with host buffers, jobs in
            flight as for value: the host-to-device copy of the job's seeds,
            tracking, and the device-to-host copy of lengths, offsets and
            packed points are all inside the timed region.
  roofline  the tracking kernel's algorithmic bytes per step
            (4 C + 4 + 16 step/save_at = 184.064 B at C = 45) times the
            steps of a launch over its event-timed duration (the
            one-at-a-time leg), against the measured HBM copy bandwidth.
  cpu_baseline  the CPU oracle (plain-C restatement of the reference
            kernel, OpenMP over seeds) on a bounded sample of the same
            workload on this host's cores.

``--impl reference`` times the reference's CPU path instead (the compiled
reference kernels under oracle/_ref when present, else the oracle) and
prints the same JSON line with "impl": "reference".
"""

from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import subprocess
import sys
import threading
import time
import types
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "streamline-steps/s"
UNIT = "steps/s"
C = 45
STEP = 0.001
SAVE_AT = 0.25
MAX_LENGTH = 300.0
GAMMA = 1.0
NOISE = 0.1
BYTES_PER_STEP = 4 * C + 4 + 16 * STEP / SAVE_AT
WORKLOAD = ("config1 Diffusion: SH lmax 8 (45 f32 coefficients) 145x174x145 at 1.25 mm, 3 bundles; "
            "seeds from seeds.from_fod; step 0.001 mm, gamma 1, noise_variance 0.1; save_at 0.25, "
            "max length 300 mm; 1M seeds per step in reference batches of 50000")


def parse_args():
    p = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--seeds", type=int, default=1000000, help="seeds per step (one tg.tractogram job)")
    p.add_argument("--batch", type=int, default=50000, help="reference batch_size inside a job")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--in-flight", type=int, default=1,
                   help="config1: jobs in flight (each on its own stream and tracker); one job's copies and "
                        "host work overlap the other's tracking")
    p.add_argument("--compact-lanes", type=int, default=0,
                   help="config1: tail compaction (tg_tracker_set_tuning): warps left with at most this many "
                        "live streamlines after the queue drains hand them to a follow-up round; 0 = off")
    p.add_argument("--compact-rounds", type=int, default=4, help="config1: follow-up rounds of tail compaction")
    p.add_argument("--slice", type=int, default=None,
                   help="config1: time slicing (tg_tracker_set_slicing): a streamline yields its lane every this "
                        "many steps while other work waits; 0 = off; default: the library's")
    p.add_argument("--workload", choices=["config1", "config0", "mixed", "config2", "serve", "tod", "connectome"],
                   default="config1",
                   help="config1 (default headline), the 64-job mixed workload, the DTI + mesh workload, or "
                        "serving under Poisson load")
    p.add_argument("--rates", default="5,20,50,100,200", help="serving: arrival rates (requests/s)")
    p.add_argument("--duration", type=float, default=6.0, help="serving: seconds of arrivals per rate")
    p.add_argument("--epoch-steps", type=int, default=65536, help="serving: step cap of an epoch")
    p.add_argument("--epoch-ms", type=float, default=6.0, help="serving: device-clock budget of an epoch (ms)")
    p.add_argument("--burst", action="store_true",
                   help="serving: submit the mixed workload's jobs at once and compare with one batched run")
    p.add_argument("--jobs", type=int, default=64, help="jobs of the mixed workload")
    p.add_argument("--per-class", action="store_true",
                   help="mixed: also time each code path's jobs alone (persistent and plain)")
    return p.parse_args()


def measured_peaks():
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        data = json.loads(path.read_text())
        return float(data["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_constant(key):
    """A per-step constant recorded in the committed ncu summary of the tracking kernel."""
    path = ROOT / "profiles" / "track_persistent_config1.md"
    if not path.exists():
        return None
    for line in path.read_text().splitlines():
        if line.startswith(key + ":"):
            return float(line.split(":", 1)[1].split()[0])
    return None


def fp32_peak_tflops():
    """FP32 FMA peak from the device properties: SMs x 128 lanes x 2 FLOP x SM clock."""
    import torch

    props = torch.cuda.get_device_properties(0)
    clock_khz = getattr(props, "clock_rate", 0) or 1965000
    return props.multi_processor_count * 128 * 2 * clock_khz * 1e3 / 1e12


def traffic_per_step(profile="track_persistent_config1.md"):
    """DRAM bytes per accepted step of the tracking kernel from the committed ncu summary."""
    path = ROOT / "profiles" / profile
    if not path.exists():
        return None
    for line in path.read_text().splitlines():
        if line.startswith("dram_bytes_per_step:"):
            return float(line.split(":", 1)[1].split()[0])
    return None


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.device_index = device_index
        self.proc = None
        self.lines = []
        self.thread = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.device_index)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # nvidia-smi's start-up takes host CPU: let it deliver its first
            # sample before the caller starts timing
            t0 = time.perf_counter()
            while not self.lines and time.perf_counter() - t0 < 5.0:
                time.sleep(0.02)
        except (OSError, ValueError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread is not None:
            self.thread.join(timeout=2)

    def summary(self):
        rows = []
        for line in self.lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), parts[4:9]))
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = np.array([r[0] for r in rows])
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for _, _, flags in rows:
            for name, flag in zip(names, flags[1:]):
                if flag.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(rows[0][1]), "reasons": sorted(reasons),
                "samples": len(rows)}


def combine_ranks(dist, times, counts, device):
    """Whole-job figures of independent replicas: the slowest rank's times
    (max) and the work of all ranks (sum).  No data-path collective: the
    ranks track disjoint seed sets and only these scalars are exchanged."""
    import torch

    t = torch.tensor(times, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    c = torch.tensor(counts, dtype=torch.float64, device=device)
    dist.all_reduce(c, op=dist.ReduceOp.SUM)
    return [float(x) for x in t.tolist()], [int(x) for x in c.tolist()]


def replica_seed(rank: int) -> int:
    """NumPy seed of a replica's seeds.from_fod draw (distinct per rank)."""
    return 2024 + rank


def setup_workload(rank: int, n_seeds: int, runtime):
    from tractography_b200 import synthetic

    return synthetic.config1_workload(n_seeds, runtime, numpy_seed=replica_seed(rank), algorithm_seed=1234 + rank)


def run_ours(args):
    import torch

    import tractography_b200 as tg
    from tractography_b200 import _lib
    from tractography_b200.algorithm import to_struct

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local_rank)
    n_job = args.seeds
    n_steps = int(math.floor(MAX_LENGTH / SAVE_AT))
    # every streamline fits a pool of n_job x n_steps points: no retry waves,
    # and each slot's tracker takes only its own share of the device
    pool = n_job * n_steps
    runtime = tg.CudaRuntime(local_rank, pool_points=pool)
    lib = runtime.lib
    fod, field, domain, seeds, algorithm = setup_workload(rank, n_job, runtime)
    n_batches = (n_job + args.batch - 1) // args.batch
    # one reference RNG seed per batch, drawn in batch order for every job
    rng_seeds = [np.array([algorithm.get_rng_seed() for _ in range(n_batches)], dtype=np.uint32)
                 for _ in range(args.warmup + args.steps)]
    in_flight = max(1, args.in_flight)
    with runtime.device_scope():
        d_handle = domain.device(runtime)
        f_handle = field.device(runtime, _lib.MODEL_SH)
        a = to_struct(algorithm)
        dev_seeds = runtime.to_device(seeds)
        host_seeds = runtime.pinned(seeds.shape, np.float32)
        host_seeds[...] = seeds

        class Slot:
            """One job in flight: a stream, its tracker and its host buffers."""

            def __init__(self, rt):
                self.rt = rt
                self.stream = rt.stream
                self.sh = ctypes.c_void_p(rt.stream_handle)
                self.tracker = rt.tracker()
                if args.compact_lanes > 0:
                    rt.set_tuning(0, args.compact_lanes, args.compact_rounds)
                if args.slice is not None:
                    rt.set_slicing(args.slice)
                self.lengths = np.empty(n_job, np.uint32)
                self.offsets = np.empty(n_job, np.uint64)
                self.out_host = None

        slots = [Slot(runtime)] + [Slot(tg.CudaRuntime(local_rank, stream=torch.cuda.Stream(local_rank),
                                                       pool_points=pool)) for _ in range(in_flight - 1)]
        torch.cuda.synchronize()

        def run(slot, i, on_host):
            total, steps = ctypes.c_uint64(), ctypes.c_uint64()
            kms, waves, launches = ctypes.c_float(), ctypes.c_uint32(), ctypes.c_uint32()
            ptr = host_seeds.ctypes.data_as(ctypes.c_void_p) if on_host else ctypes.c_void_p(dev_seeds.data_ptr())
            _lib.check(lib.tg_tracker_run(
                slot.tracker, ctypes.byref(a), d_handle, f_handle, ptr, 1 if on_host else 0, n_job, args.batch,
                rng_seeds[i].ctypes.data_as(ctypes.c_void_p), SAVE_AT, n_steps,
                slot.lengths.ctypes.data_as(ctypes.c_void_p), slot.offsets.ctypes.data_as(ctypes.c_void_p),
                ctypes.byref(total), ctypes.byref(steps), slot.sh))
            _lib.check(lib.tg_tracker_stats(slot.tracker, ctypes.byref(kms), ctypes.byref(waves),
                                            ctypes.byref(launches)))
            return int(steps.value), int(total.value), float(kms.value), int(launches.value), int(waves.value)

        def leg(on_host, width):
            """Time jobs warmup .. warmup+steps-1 with `width` of them in flight.

            Slot k runs jobs k, k+width, ... one after another from its own host
            thread (its first job queued 20 ms after the previous slot's), so
            that the next job is queued while the previous one runs.  The
            start event is recorded before any job is queued and every other
            stream waits for it; the end event waits for every stream."""
            ev_start, ev_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            ev_start.record(slots[0].stream)
            for sl in slots[1:width]:
                sl.stream.wait_event(ev_start)
            results = [None] * args.steps
            errors = []

            def worker(k):
                slot = slots[k]
                try:
                    with slot.rt.device_scope():
                        # the first job takes every SM slot; the next one, queued a
                        # moment later, starts as the first one's blocks retire
                        if k > 0:
                            time.sleep(0.02 * k)
                        for j in range(k, args.steps, width):
                            i = args.warmup + j
                            st, pts, km, nl, nw = run(slot, i, on_host)
                            if on_host:
                                if slot.out_host is None or pts > slot.out_host.shape[0]:
                                    slot.out_host = slot.rt.pinned((int(pts * 1.1) + 1024, 3), np.float32)
                                _lib.check(lib.tg_tracker_copy_points(
                                    slot.tracker, slot.out_host.ctypes.data_as(ctypes.c_void_p), 0, pts, 1,
                                    slot.sh))
                            results[j] = (st, pts, km, nl, nw)
                except Exception as exc:  # re-raised by the caller after every worker ends
                    errors.append(exc)

            threads = [threading.Thread(target=worker, args=(k,)) for k in range(width)]
            for t in threads:
                t.start()
            for t in threads:
                t.join()
            if errors:
                raise errors[0]
            for sl in slots[1:width]:
                ev = torch.cuda.Event()
                ev.record(sl.stream)
                slots[0].stream.wait_event(ev)
            ev_end.record(slots[0].stream)
            torch.cuda.synchronize()
            return ev_start.elapsed_time(ev_end), results

        # warm-up from host seeds: each slot's tracker allocates its seed copy too
        warm_points = 0
        for i in range(max(args.warmup, in_flight)):
            warm_points = max(warm_points, run(slots[i % in_flight], i % max(1, args.warmup), on_host=True)[1])
        # page-locked result buffers exist before any timed region
        for sl in slots:
            sl.out_host = sl.rt.pinned((int(warm_points * 1.25) + 1024, 3), np.float32)

        sampler = ClockSampler(local_rank)
        with sampler:
            # one job at a time: the tracking kernel's launches alone (roofline)
            if dist is not None:
                dist.barrier()
            single_ms, single = leg(False, 1)
            kernel_ms = sum(r[2] for r in single)
            single_steps = sum(r[0] for r in single)
            n_launch = sum(r[3] for r in single)
            n_waves = sum(r[4] for r in single)
            if dist is not None:
                dist.barrier()
            # device-resident leg, jobs overlapped (one at a time: the leg above)
            dev_ms, dev = leg(False, in_flight) if in_flight > 1 else (single_ms, single)
            dev_steps = sum(r[0] for r in dev)
            dev_points = sum(r[1] for r in dev)
            if dist is not None:
                dist.barrier()
            # end-to-end leg through the C ABI with host buffers, jobs overlapped
            e2e_ms, e2e = leg(True, in_flight)
            e2e_steps = sum(r[0] for r in e2e)
            h2d = sum(seeds.nbytes + rng_seeds[args.warmup + j].nbytes for j in range(args.steps))
            d2h = sum(r[1] * 12 + n_job * (4 + 8) for r in e2e)
            if dist is not None:
                dist.barrier()

        # outside the timed region: the last job of the end-to-end leg against the oracle
        parity = None
        last = slots[(args.steps - 1) % in_flight]
        if not args.no_cpu_baseline and world == 1:
            parity = parity_sample(lib, last.tracker, last.sh, algorithm, field, domain, seeds, args.batch,
                                   rng_seeds[args.warmup + args.steps - 1], last.lengths, last.offsets)

    if dist is not None:
        (dev_ms, e2e_ms, kernel_ms, single_ms), (dev_steps, e2e_steps, dev_points, n_launch, n_waves,
                                                 single_steps) = combine_ranks(
            dist, [dev_ms, e2e_ms, kernel_ms, single_ms],
            [dev_steps, e2e_steps, dev_points, n_launch, n_waves, single_steps], "cuda")
    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return

    peak, peak_kind = measured_peaks()
    value = dev_steps / (dev_ms / 1e3)
    # the tracking kernel's own rate, from the leg that runs one job at a time
    kernel_steps_per_s = single_steps / max(1, world) / (kernel_ms / 1e3)
    achieved = kernel_steps_per_s * BYTES_PER_STEP / 1e9
    tps = traffic_per_step()
    line = {
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": dev_ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded generator; no dataset)",
        "config": {
            "workload": WORKLOAD,
            "seeds_per_step": n_job,
            "batch_size": args.batch,
            "max_points_per_streamline": n_steps,
            "cache": "inputs larger than L2: 660 MB FOD volume, 126 MB L2",
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
            "rng": "MWC64X reference stream per batch",
            "jobs_in_flight": in_flight,
            "compact_lanes": args.compact_lanes,
            "slice_steps": runtime.slicing(),
        },
        "streamlines_per_s": n_job * args.steps * world / (dev_ms / 1e3),
        "points_per_step": dev_points / args.steps / max(1, world),
        "e2e": {
            "value": e2e_steps / (e2e_ms / 1e3),
            "unit": UNIT,
            "h2d_bytes_per_step": int(h2d / args.steps),
            "d2h_bytes_per_step": int(d2h / args.steps),
        },
        "gpu_launches": n_launch,
        "roofline": {
            "bound": "hbm",
            "achieved": achieved,
            "peak": peak,
            "unit": "GB/s",
            "frac": achieved / peak,
            "traffic": (tps * single_steps / max(1, n_waves)) if tps is not None else None,
            "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
            "bytes_per_step": BYTES_PER_STEP,
            "kernel_ms_per_step": kernel_ms / args.steps / max(1, world),
            "launches_from": "the one-job-at-a-time leg",
        },
        "clocks": sampler.summary(),
    }
    if in_flight > 1:
        line["single_job"] = {
            "value": single_steps / (single_ms / 1e3),
            "ms_per_step": single_ms / args.steps,
            "note": "the same jobs one at a time: each tg_tracker_run returns before the next starts",
        }
    line["roofline"]["note"] = ("algorithmic bytes: the 184 B gather of a step; a voxel's coefficients stay in "
                                "registers for the ~1250 steps a streamline spends in it, so DRAM carries ~0.3 B "
                                "per step (traffic) and frac above 1 is that reuse, not DRAM; the kernel is bound "
                                "by instruction issue (issue)")
    inst = profile_constant("thread_inst_per_step")
    issue = profile_constant("issue_active_pct")
    if inst is not None and issue is not None:
        line["issue"] = {"thread_instructions_per_step": inst, "issue_active": issue / 100.0,
                         "source": "full-size ncu counters of the tracking kernel "
                                   "(profiles/track_persistent_config1.md)"}
    flop = profile_constant("fp32_flop_per_step")
    if flop is not None:
        tflops = kernel_steps_per_s * flop / 1e12
        peak_fp32 = fp32_peak_tflops()
        line["fp32"] = {"flop_per_step": flop, "achieved_tflops": tflops, "peak_tflops": peak_fp32,
                        "frac": tflops / peak_fp32,
                        "note": "FP32 FLOP per step from the ncu instruction mix of the tracking kernel "
                                "(FFMA = 2); peak = SMs x 128 x 2 x SM clock"}
    if not args.no_cpu_baseline and world == 1:
        line["cpu_baseline"] = cpu_baseline(field, domain, seeds)
    if parity is not None:
        line["parity"] = parity
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def _reference_lib():
    """The compiled reference kernels (oracle/_ref), or None."""
    path = ROOT / "oracle" / "_ref" / "libtgref.so"
    if not path.exists():
        return None
    try:
        from oracle import reference

        return reference
    except ImportError:
        return None


def _cpu_track(field, domain, seeds, rng_seed, threads):
    """Track `seeds` on the CPU; returns (accepted steps, seconds, kind, description)."""
    from oracle import oracle as O

    n_steps = int(math.floor(MAX_LENGTH / SAVE_AT))
    ref = _reference_lib()
    if ref is not None:
        t0 = time.perf_counter()
        steps = ref.tractogram_steps(domain, field, "diffusion", STEP, GAMMA, NOISE, seeds, rng_seed, SAVE_AT,
                                     n_steps, threads)
        return steps, time.perf_counter() - t0, "reference", \
            "reference OpenCL kernel source compiled as C++ (oracle/_ref), OpenMP over seeds"
    case = O.Case(mask=domain.values, mask_inv_affine=domain.inverse_affine, field=field.values,
                  field_inv_affine=field.inverse_affine, model=O.MODEL_SH, algorithm=O.ALGO_DIFFUSION,
                  step_size=STEP, gamma=GAMMA, noise_variance=NOISE, rng_seed=rng_seed, save_at=SAVE_AT,
                  n_steps=n_steps)
    t0 = time.perf_counter()
    _, _, steps = case.tractogram(seeds, n_threads=threads, return_steps=True)
    return steps, time.perf_counter() - t0, "port", "plain-C oracle restating the reference kernel, OpenMP over seeds"


def cpu_baseline(field, domain, seeds, threads=None):
    """CPU throughput on a bounded sample (about 120 seeds per core) of the workload."""
    threads = threads or os.cpu_count() or 1
    n_sample = min(len(seeds), 120 * threads)
    sample = np.ascontiguousarray(seeds[:n_sample])
    steps, dt, kind, what = _cpu_track(field, domain, sample, 77, threads)
    return {"value": steps / dt, "unit": UNIT, "cores": threads, "kind": kind,
            "sample": f"first {n_sample} seeds of the timed batches ({steps} steps, {dt:.1f} s); {what}; "
                      "pocl unavailable here"}


def parity_sample(lib, tracker, stream, algorithm, field, domain, seeds, batch, rng_seeds, lengths, offsets,
                  n_sample=256, threads=None):
    """Outside the timed region: the last timed run's streamlines of a spread
    sample of seeds against the CPU oracle with the same batch RNG seeds and
    batch-local stream ids (tracking.py:103-148); bit for bit."""
    from oracle import oracle as O
    from tractography_b200 import _lib

    threads = threads or os.cpu_count() or 1
    n = len(seeds)
    n_steps = int(math.floor(MAX_LENGTH / SAVE_AT))
    ids = np.unique(np.linspace(0, n - 1, n_sample).astype(np.int64))
    identical = True
    mismatches = 0
    for b in np.unique(ids // batch):
        sel = ids[ids // batch == b]
        local = (sel - b * batch).astype(np.uint32)
        case = O.Case(mask=domain.values, mask_inv_affine=domain.inverse_affine, field=field.values,
                      field_inv_affine=field.inverse_affine, model=O.MODEL_SH, algorithm=O.ALGO_DIFFUSION,
                      step_size=algorithm.step_size, gamma=algorithm.gamma,
                      noise_variance=algorithm.noise_variance, rng_seed=int(rng_seeds[b]), save_at=SAVE_AT,
                      n_steps=n_steps)
        want, want_len = case.tractogram_ids(seeds[sel], local, n_threads=threads)
        for k, i in enumerate(sel):
            got = np.zeros((int(lengths[i]), 3), np.float32)
            if len(got):
                _lib.check(lib.tg_tracker_copy_points(tracker, got.ctypes.data_as(ctypes.c_void_p), int(offsets[i]),
                                                      int(lengths[i]), 1, stream))
            same = int(lengths[i]) == int(want_len[k]) and np.array_equal(got, want[k, : want_len[k], :3],
                                                                          equal_nan=True)
            if not same:
                identical = False
                mismatches += 1
    return {"seeds": int(len(ids)), "identical": identical, "mismatches": mismatches,
            "against": "CPU oracle, bit for bit (lengths and every point), last timed run"}


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import tractography_b200 as tg
    from oracle import oracle as O
    from tractography_b200 import synthetic

    fod = synthetic.config1(seed=0)
    field = tg.field.Image(fod)
    mask = np.any(field.values != 0, axis=-1).astype(np.uint8)
    domain = tg.domain.Image(tg.Nifti1Image(mask, fod.affine))
    threads = os.cpu_count() or 1
    per_step = max(8, 16 * threads)
    inline, voxels, affine = tg.seeds.sparse_fod(fod)
    np.random.seed(2024)
    states = np.random.randint(4294967295, size=(per_step * (args.warmup + args.steps), 2)).astype(np.uint32)
    seeds = O.seeds_from_fod(O.MODEL_SH, inline, voxels, affine, states, n_threads=threads)
    algorithm = tg.algorithm.Diffusion(tg.local.RealSymmetricSphericalHarmonics(C), step_size=STEP, gamma=GAMMA,
                                       noise_variance=NOISE, seed=1234)
    total_steps, total_t = 0, 0.0
    kind = what = ""
    for i in range(args.warmup + args.steps):
        chunk = np.ascontiguousarray(seeds[i * per_step:(i + 1) * per_step])
        steps, dt, kind, what = _cpu_track(field, domain, chunk, algorithm.get_rng_seed(), threads)
        if i >= args.warmup:
            total_steps += steps
            total_t += dt
    value = total_steps / total_t if total_t > 0 else 0.0
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * total_t / max(1, args.steps), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator; no dataset)",
        "impl": "reference",
        "config": {"workload": WORKLOAD, "batch_seeds": per_step,
                   "note": "each step is a bounded sample of the workload on the host cores"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                         "sample": f"{per_step} seeds per step, {args.steps} timed steps; {what}"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def build_mixed_jobs(n_jobs, seed=0):
    """Config-3 jobs (see synthetic.mixed_job_specs); volumes shared per (size, lmax)."""
    import tractography_b200 as tg
    from tractography_b200 import jobs as jobs_module
    from tractography_b200 import synthetic

    cache = {}
    out = []
    for sp in synthetic.mixed_job_specs(n_jobs=n_jobs, seed=seed):
        key = (sp["shape"], sp["lmax"])
        if key not in cache:
            fod, mask = synthetic.bundle_field(sp["shape"], lmax=sp["lmax"], seed=len(cache))
            cache[key] = (tg.field.Image(fod), tg.domain.Image(mask), mask)
        field, domain, mask = cache[key]
        C = (sp["lmax"] + 1) * (sp["lmax"] + 2) // 2
        model = tg.local.RealSymmetricSphericalHarmonics(C)
        step = 0.2   # 0.1 voxel at 2 mm
        if sp["algorithm"] == "transport":
            alg = tg.algorithm.Transport(model, step_size=step, gamma=1.0)
        else:
            alg = tg.algorithm.Diffusion(model, step_size=step, gamma=1.0, noise_variance=sp["noise_variance"],
                                         seed=sp["seed"])
        seeds = synthetic.uniform_seeds(mask, sp["n_seeds"], seed=sp["seed"])
        batch = 50000
        n_batches = (len(seeds) + batch - 1) // batch
        rng = np.array([alg.get_rng_seed() for _ in range(n_batches)], dtype=np.uint32)
        out.append(jobs_module.Job(field=field, domain=domain, algorithm=alg, seeds=seeds, save_at=SAVE_AT,
                                   n_steps=int(math.floor(sp["max_length"] / SAVE_AT)), min_points=0,
                                   batch_size=batch, batch_rng_seeds=rng))
    return out


def run_mixed(args):
    """Config 3: 64 uneven jobs, persistent multi-job run vs plain one launch per batch."""
    import torch

    import tractography_b200 as tg
    from tractography_b200 import _lib, tracking
    from tractography_b200.algorithm import to_struct

    torch.cuda.set_device(0)
    runtime = tg.CudaRuntime(0)
    lib = runtime.lib
    sh = ctypes.c_void_p(runtime.stream_handle)
    jobs = build_mixed_jobs(args.jobs)
    n_total = sum(j.n_seeds for j in jobs)
    with runtime.device_scope():
        structs = (_lib.Job * len(jobs))()
        dev_seeds = []
        for k, job in enumerate(jobs):
            d_h, f_h = tracking._handles(job.algorithm, job.domain, job.field, runtime)
            ds = runtime.to_device(job.seeds)
            dev_seeds.append(ds)
            s = structs[k]
            s.domain, s.field = d_h, f_h
            s.algorithm = to_struct(job.algorithm)
            s.seeds = ds.data_ptr()
            s.n_seeds = job.n_seeds
            s.batch_size = job.batch_size
            s.batch_rng_seeds = job.batch_rng_seeds.ctypes.data
            s.save_at = job.save_at
            s.n_steps = job.n_steps
        lengths = np.empty(n_total, np.uint32)
        offsets = np.empty(n_total, np.uint64)
        total, steps = ctypes.c_uint64(), ctypes.c_uint64()
        kms, waves, launches = ctypes.c_float(), ctypes.c_uint32(), ctypes.c_uint32()

        def persistent(subset=None):
            table, n = (structs, len(jobs)) if subset is None else subset
            _lib.check(lib.tg_tracker_run_jobs(runtime.tracker(), table, n, 0,
                                               lengths.ctypes.data_as(ctypes.c_void_p),
                                               offsets.ctypes.data_as(ctypes.c_void_p), ctypes.byref(total),
                                               ctypes.byref(steps), sh))
            _lib.check(lib.tg_tracker_stats(runtime.tracker(), ctypes.byref(kms), ctypes.byref(waves),
                                            ctypes.byref(launches)))

        max_batch = max(min(j.batch_size, j.n_seeds) for j in jobs)
        max_steps = max(j.n_steps for j in jobs)
        d_out = torch.empty((max_batch * max_steps * 4,), dtype=torch.float32, device=runtime.device)
        d_len = torch.empty((n_total,), dtype=torch.int32, device=runtime.device)

        def plain(only=None):
            n_launch = 0
            base = 0
            for k, job in enumerate(jobs):
                if only is not None and k not in only:
                    base += job.n_seeds
                    continue
                d_h, f_h = tracking._handles(job.algorithm, job.domain, job.field, runtime)
                for b in range(len(job.batch_rng_seeds)):
                    lo = b * job.batch_size
                    n = min(job.batch_size, job.n_seeds - lo)
                    a = to_struct(job.algorithm, int(job.batch_rng_seeds[b]))
                    _lib.check(lib.tg_tractogram(ctypes.byref(a), d_h, f_h,
                                                 ctypes.c_void_p(dev_seeds[k].data_ptr() + lo * 32), n,
                                                 job.save_at, job.n_steps, ctypes.c_void_p(d_out.data_ptr()),
                                                 ctypes.c_void_p(d_len.data_ptr() + 4 * (base + lo)), sh))
                    n_launch += 1
                base += job.n_seeds
            return n_launch

        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        for _ in range(args.warmup):
            persistent()
            plain()
        torch.cuda.synchronize()
        p_ms = q_ms = 0.0
        n_plain = 0
        per_step = []
        sampler = ClockSampler(0)
        with sampler:
            for _ in range(args.steps):
                ev0.record(runtime.stream)
                persistent()
                ev1.record(runtime.stream)
                torch.cuda.synchronize()
                p = ev0.elapsed_time(ev1)
                ev0.record(runtime.stream)
                n_plain = plain()
                ev1.record(runtime.stream)
                torch.cuda.synchronize()
                q = ev0.elapsed_time(ev1)
                p_ms, q_ms = p_ms + p, q_ms + q
                per_step.append(q / p)
        plain_len = d_len.cpu().numpy().view(np.uint32)
        same_lengths = bool(np.array_equal(plain_len, lengths))
        work = int(steps.value)
        persistent_kernel_ms = float(kms.value)
        persistent_launches = int(launches.value)
        classes = []
        if args.per_class:
            # each code path's jobs alone: the multi-job run restricted to them, and their plain launches
            groups = {}
            for k, job in enumerate(jobs):
                key = (type(job.algorithm.local_model).__name__, job.algorithm.local_model.n_parameters,
                       type(job.algorithm).__name__)
                groups.setdefault(key, []).append(k)
            for key, members in sorted(groups.items()):
                sub = (_lib.Job * len(members))(*[structs[k] for k in members])
                persistent((sub, len(members)))
                torch.cuda.synchronize()
                ev0.record(runtime.stream)
                persistent((sub, len(members)))
                ev1.record(runtime.stream)
                torch.cuda.synchronize()
                c_ms, c_kernel, c_steps = ev0.elapsed_time(ev1), float(kms.value), int(steps.value)
                plain(set(members))
                torch.cuda.synchronize()
                ev0.record(runtime.stream)
                plain(set(members))
                ev1.record(runtime.stream)
                torch.cuda.synchronize()
                q = ev0.elapsed_time(ev1)
                classes.append({"model": key[0], "coefficients": key[1], "algorithm": key[2], "jobs": len(members),
                                "seeds": int(sum(jobs[k].n_seeds for k in members)), "steps": c_steps,
                                "persistent_ms": c_ms, "persistent_kernel_ms": c_kernel, "plain_ms": q,
                                "persistent_kernel_steps_per_s": c_steps / (c_kernel / 1e3),
                                "plain_steps_per_s": c_steps / (q / 1e3), "speedup_kernel_vs_plain": q / c_kernel})
    line = {
        "metric": METRIC, "workload": "mixed", "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "higher_is_better": True, "dtype": "f32",
        "data": "synthetic (seeded generator; no dataset)",
        "value": work / (p_ms / args.steps / 1e3),
        "plain_value": work / (q_ms / args.steps / 1e3),
        "speedup_vs_plain": q_ms / p_ms,
        "speedup_per_step": per_step,
        "speedup_median": float(np.median(per_step)),
        "speedup_spread": float((max(per_step) - min(per_step)) / np.median(per_step)),
        "ms_per_step": p_ms / args.steps,
        "plain_ms_per_step": q_ms / args.steps,
        "gpu_launches_per_step": persistent_launches,
        "kernel_ms_per_step": persistent_kernel_ms,
        "plain_launches_per_step": n_plain,
        "identical_lengths": same_lengths,
        "config": {
            "workload": ("64 jobs: volume 64^3 / 96x96x60 / 128^3 / 145x174x145, SH lmax 4/6/8, seeds "
                         "log-U[1k, 500k], Transport or Diffusion (noise U[0.05, 0.2]), max length "
                         "U[50, 300] mm, step 0.2 mm (0.1 voxel), save_at 0.25, batch 50000"),
            "jobs": len(jobs), "seeds": n_total, "steps_per_run": work,
            "plain": "one tg_tractogram launch per 50000-seed batch, jobs in order, dense output",
        },
        "clocks": sampler.summary(),
    }
    if classes:
        line["classes"] = classes
    print(json.dumps(line), flush=True)


PRODUCT_SEEDS = 100000
PRODUCT_WORKLOAD = ("{kind} on the config-1 volume: SH lmax 8 (45 f32 coefficients) 145x174x145 at 1.25 mm, 3 "
                    "bundles; domain = nonzero voxels (the whole box); {n} boundary seeds (domain.seed's sampler) "
                    "per step; the reference's default algorithm for tg.{kind} (Transport, step 0.001 mm, gamma 1); "
                    "maximum length 300 mm{extra}")


def run_product(args):
    """TOD or connectome (tracking.py:181-385, :388-602) on the config-1 volume."""
    import torch

    import tractography_b200 as tg
    from tractography_b200 import _lib, synthetic, tracking
    from tractography_b200.algorithm import to_struct

    kind = args.workload
    torch.cuda.set_device(0)
    runtime = tg.CudaRuntime(0)
    lib = runtime.lib
    sh = ctypes.c_void_p(runtime.stream_handle)
    fod = synthetic.config1(seed=0)
    field = tg.field.Image(fod)
    mask = np.any(field.values != 0, axis=-1).astype(np.uint8)
    domain = tg.domain.Image(tg.Nifti1Image(mask, fod.affine))
    n_seeds = args.seeds if args.seeds != 1000000 else PRODUCT_SEEDS
    model = tg.local.RealSymmetricSphericalHarmonics(C)
    algorithm = tg.algorithm.Transport(model)                 # step 0.001, gamma 1 (the reference defaults)
    n_steps = int(math.floor(MAX_LENGTH / algorithm.step_size))
    v4, f4, cumulative = domain.boundary_arrays()
    shape = fod.shape[:3]
    inv = np.ascontiguousarray(np.linalg.inv(np.asarray(fod.affine, np.float64)), dtype=np.float32)
    with runtime.device_scope():
        d_h, f_h = tracking._handles(algorithm, domain, field, runtime)
        b_h = domain.boundary_bvh().device(runtime) if kind == "connectome" else None
        dv, df, dc = runtime.to_device(v4), runtime.to_device(f4), runtime.to_device(cumulative)
        steps = torch.zeros((1,), dtype=torch.int64, device=runtime.device)
        if kind == "tod":
            out = torch.zeros(tuple(shape) + (45,), dtype=torch.float32, device=runtime.device)
            dims = np.asarray(shape, dtype=np.uint32)
        else:
            rows = runtime.empty((9 * n_seeds,), torch.int32)
            cols = runtime.empty((9 * n_seeds,), torch.int32)
            weights = runtime.empty((9 * n_seeds,), torch.float32)

        def run(rng_seed):
            a = to_struct(algorithm, rng_seed)
            if kind == "tod":
                out.zero_()
                _lib.check(lib.tg_tod(ctypes.byref(a), d_h, f_h, ctypes.c_void_p(dv.data_ptr()), len(v4),
                                      ctypes.c_void_p(df.data_ptr()), ctypes.c_void_p(dc.data_ptr()), len(f4),
                                      n_seeds, n_steps, dims.ctypes.data_as(ctypes.c_void_p),
                                      inv.ctypes.data_as(ctypes.c_void_p), ctypes.c_void_p(out.data_ptr()),
                                      ctypes.c_void_p(steps.data_ptr()), sh))
            else:
                _lib.check(lib.tg_connectome(ctypes.byref(a), d_h, f_h, b_h, ctypes.c_void_p(dv.data_ptr()), len(v4),
                                             ctypes.c_void_p(df.data_ptr()), ctypes.c_void_p(dc.data_ptr()), len(f4),
                                             n_seeds, n_steps, 0.0, ctypes.c_void_p(rows.data_ptr()),
                                             ctypes.c_void_p(cols.data_ptr()), ctypes.c_void_p(weights.data_ptr()),
                                             ctypes.c_void_p(steps.data_ptr()), sh))

        for w in range(args.warmup):
            run(1000 + w)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        sampler = ClockSampler(0)
        with sampler:
            torch.cuda.synchronize()
            steps.zero_()
            ev0.record(runtime.stream)
            for k in range(args.steps):
                run(k)
            ev1.record(runtime.stream)
            torch.cuda.synchronize()
            dev_ms = ev0.elapsed_time(ev1)
            dev_steps = int(steps.item())
            # end to end: the public call (host arrays out: the TOD image / the CSR matrix)
            e2e_steps, t0 = 0, time.perf_counter()
            for k in range(args.steps):
                st = {}
                if kind == "tod":
                    grid = types.SimpleNamespace(shape=tuple(shape), affine=np.asarray(fod.affine), header=None)
                    tracking.tod(algorithm, domain, field, grid, n_seeds, runtime=runtime, stats=st)
                else:
                    tracking.connectome(algorithm, domain, field, n_seeds, runtime=runtime, stats=st)
                e2e_steps += st["steps"]
            torch.cuda.synchronize()
            e2e_s = time.perf_counter() - t0
    out_bytes = int(np.prod(shape)) * 45 * 4 if kind == "tod" else 9 * n_seeds * 12
    line = {"metric": METRIC, "value": dev_steps / (dev_ms / 1e3), "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dev_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator; no dataset)",
            "workload": kind,
            "config": {"workload": PRODUCT_WORKLOAD.format(
                kind=kind, n=n_seeds,
                extra="; output: the (145, 174, 145, 45) raw TOD on the field grid" if kind == "tod" else
                "; output: 9 weighted contributions per track (end segment hit on the boundary BVH)"),
                "boundary_triangles": len(f4)},
            "tracks_per_s": n_seeds * args.steps / (dev_ms / 1e3),
            "e2e": {"value": e2e_steps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": out_bytes,
                    "note": "wall clock of the public tracking call; boundary arrays resident"},
            "gpu_launches": args.steps, "clocks": sampler.summary()}
    if not args.no_cpu_baseline:
        from oracle import oracle as O

        threads = os.cpu_count() or 1
        n_cpu = max(8 * threads, 64)
        case = O.Case(mask=domain.values, mask_inv_affine=domain.inverse_affine, field=field.values,
                      field_inv_affine=field.inverse_affine, step_size=algorithm.step_size, gamma=1.0, rng_seed=7)
        t0 = time.perf_counter()
        if kind == "tod":
            case.tod((v4, f4, cumulative), n_cpu, n_steps, shape, inv)
        else:
            bvh = O.BoundaryBvh.build(domain.boundary.vertices, domain.boundary.faces)
            t0 = time.perf_counter()
            case.connectome(bvh, (v4, f4, cumulative), n_cpu, n_steps)
        dt = time.perf_counter() - t0
        # steps of the sample: the same tracks on the GPU (bit-identical loop)
        with runtime.device_scope():
            a = to_struct(algorithm, 7)
            steps.zero_()
            n_save = n_seeds
            n_seeds = n_cpu
            run(7)
            n_seeds = n_save
            torch.cuda.synchronize()
            cpu_steps = int(steps.item())
        line["cpu_baseline"] = {"value": cpu_steps / dt, "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": f"{n_cpu} tracks ({cpu_steps} steps, {dt:.1f} s); plain-C oracle, "
                                          f"OpenMP over tracks"}
    print(json.dumps(line), flush=True)


C0_WORKLOAD = ("config0 Transport: SH lmax 8 (45 f32 coefficients) 32^3 at 2 mm, bundle along x and y-z arcs, "
               "ellipsoid mask 14/12/12 voxels; 10000 seeds uniform in the mask; step 0.2 mm (0.1 voxel), gamma 1; "
               "save_at 0.25, max length 300 mm")


def run_config0(args):
    """Config 0: the reference's CPU-runnable Transport case, GPU vs the reference kernel on the host."""
    import torch

    import tractography_b200 as tg
    from tractography_b200 import _lib, synthetic
    from tractography_b200.algorithm import to_struct

    torch.cuda.set_device(0)
    runtime = tg.CudaRuntime(0)
    lib = runtime.lib
    sh = ctypes.c_void_p(runtime.stream_handle)
    fod, mask = synthetic.config0()
    field, domain = tg.field.Image(fod), tg.domain.Image(mask)
    n_job = args.seeds if args.seeds != 1000000 else 10000
    seeds = synthetic.seeds_in_mask(mask, n_job, seed=0)
    algorithm = tg.algorithm.Transport(tg.local.RealSymmetricSphericalHarmonics(45), step_size=0.2, gamma=1.0)
    n_steps = int(math.floor(MAX_LENGTH / SAVE_AT))
    rng = np.zeros((n_job + args.batch - 1) // args.batch, np.uint32)
    with runtime.device_scope():
        d_h, f_h = domain.device(runtime), field.device(runtime, _lib.MODEL_SH)
        a = to_struct(algorithm)
        dev_seeds = runtime.to_device(seeds)
        lengths = np.empty(n_job, np.uint32)
        offsets = np.empty(n_job, np.uint64)
        total, steps = ctypes.c_uint64(), ctypes.c_uint64()
        kms, waves, launches = ctypes.c_float(), ctypes.c_uint32(), ctypes.c_uint32()

        host_seeds = runtime.pinned(seeds.shape, np.float32)
        host_seeds[...] = seeds

        def run(on_host=False):
            ptr = host_seeds.ctypes.data_as(ctypes.c_void_p) if on_host else ctypes.c_void_p(dev_seeds.data_ptr())
            _lib.check(lib.tg_tracker_run(runtime.tracker(), ctypes.byref(a), d_h, f_h,
                                          ptr, 1 if on_host else 0, n_job, args.batch,
                                          rng.ctypes.data_as(ctypes.c_void_p), SAVE_AT, n_steps,
                                          lengths.ctypes.data_as(ctypes.c_void_p),
                                          offsets.ctypes.data_as(ctypes.c_void_p), ctypes.byref(total),
                                          ctypes.byref(steps), sh))
            _lib.check(lib.tg_tracker_stats(runtime.tracker(), ctypes.byref(kms), ctypes.byref(waves),
                                            ctypes.byref(launches)))
            return int(steps.value), float(kms.value), int(launches.value), int(total.value)

        t_warm = time.perf_counter()
        for _ in range(args.warmup):
            run()
        per_job = (time.perf_counter() - t_warm) / max(1, args.warmup)
        # one job takes a few ms: repeat it until the timed region lasts about a
        # second, so that the clock sampler sees it
        n_timed = max(args.steps, int(math.ceil(1.0 / max(per_job, 1e-4))))
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        out_host = runtime.pinned((n_job * n_steps // 4 + 1024, 3), np.float32)
        sampler = ClockSampler(0)
        with sampler:
            # A job lasts a few ms, most of it host bookkeeping, so the two
            # legs alternate job by job: anything else on the host slows both
            # alike.  Each job is bracketed by its own events.
            dev_steps = n_launch = 0
            kernel_ms = dev_ms = e2e_ms = 0.0
            e2e_steps = d2h = 0
            for _ in range(n_timed):
                torch.cuda.synchronize()
                ev0.record(runtime.stream)
                st, k, nl, _ = run()
                ev1.record(runtime.stream)
                torch.cuda.synchronize()
                dev_ms += ev0.elapsed_time(ev1)
                dev_steps, kernel_ms, n_launch = dev_steps + st, kernel_ms + k, n_launch + nl
                # end to end: seeds from pinned host memory, points back to it
                ev0.record(runtime.stream)
                st, _, _, pts = run(True)
                if pts > out_host.shape[0]:
                    out_host = runtime.pinned((pts, 3), np.float32)
                _lib.check(lib.tg_tracker_copy_points(runtime.tracker(), out_host.ctypes.data_as(ctypes.c_void_p), 0,
                                                      pts, 1, sh))
                ev1.record(runtime.stream)
                torch.cuda.synchronize()
                e2e_ms += ev0.elapsed_time(ev1)
                e2e_steps += st
                d2h += pts * 12 + n_job * 12
    peak, peak_kind = measured_peaks()
    bps = 4 * 45 + 4 + 16 * 0.2 / SAVE_AT
    kernel_sps = dev_steps / (kernel_ms / 1e3)
    line = {"metric": METRIC, "value": dev_steps / (dev_ms / 1e3), "unit": UNIT, "n_gpus": 1, "steps": n_timed,
            "warmup": args.warmup, "ms_per_step": dev_ms / n_timed, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator; no dataset)",
            "workload": "config0",
            "e2e": {"value": e2e_steps / (e2e_ms / 1e3), "unit": UNIT,
                    "h2d_bytes_per_step": int(seeds.nbytes + rng.nbytes), "d2h_bytes_per_step": int(d2h / n_timed)},
            "config": {"workload": C0_WORKLOAD, "seeds_per_step": n_job,
                       "cache": "volume (5.9 MB) L2-resident; one job is far below one GPU's lanes"},
            "streamlines_per_s": n_job * n_timed / (dev_ms / 1e3), "gpu_launches": n_launch,
            "roofline": {"bound": "hbm", "achieved": kernel_sps * bps / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": kernel_sps * bps / 1e9 / peak, "bytes_per_step": bps,
                         "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"},
            "clocks": sampler.summary()}
    if not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        ref = _reference_lib()
        t0 = time.perf_counter()
        if ref is not None:
            st = ref.tractogram_steps(domain, field, "transport", 0.2, 1.0, 0.0, seeds, 0, SAVE_AT, n_steps, threads)
            kind, what = "reference", "reference OpenCL kernel source compiled as C++ (oracle/_ref)"
        else:
            from oracle import oracle as O

            case = O.Case(mask=domain.values, mask_inv_affine=domain.inverse_affine, field=field.values,
                          field_inv_affine=field.inverse_affine, step_size=0.2, gamma=1.0, save_at=SAVE_AT,
                          n_steps=n_steps)
            st = case.tractogram(seeds, n_threads=threads, return_steps=True)[2]
            kind, what = "port", "plain-C oracle"
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": st / dt, "unit": UNIT, "cores": threads, "kind": kind,
                                "sample": f"all {n_job} seeds ({st} steps, {dt:.1f} s); {what}, OpenMP over seeds"}
    print(json.dumps(line), flush=True)


C2_STEP = 0.2           # 0.1 voxel at 2 mm
C2_SEEDS = 2_000_000
C2_BYTES_PER_STEP = 4 * 6 + 1 + 16 * C2_STEP / SAVE_AT
C2_WORKLOAD = ("config2 DTI + mesh: 96x96x60 tensors (6 f32) at 2 mm along the config-0 field with 5% "
               "log-normal eigenvalue jitter; closed surface of 499280 triangles (geodesic sphere, "
               "r = 1 + 0.1 Y21 + 0.05 Y40, scaled to the volume) terminating streamlines through its BVH; "
               "2M seeds uniform inside; Transport, step 0.2 mm (0.1 voxel), gamma 1; save_at 0.25, "
               "max length 300 mm; batches of 50000")


def setup_config2(runtime, n_seeds):
    from tractography_b200 import synthetic

    return synthetic.config2_workload(n_seeds, runtime, step_size=C2_STEP)


def run_config2(args):
    """Config 2: DTI Transport in a closed-surface (BVH) domain, 2M seeds."""
    import torch

    import tractography_b200 as tg
    from tractography_b200 import _lib
    from tractography_b200.algorithm import to_struct

    torch.cuda.set_device(0)
    runtime = tg.CudaRuntime(0)
    lib = runtime.lib
    sh = ctypes.c_void_p(runtime.stream_handle)
    n_job = args.seeds if args.seeds != 1000000 else C2_SEEDS
    field, mesh, seeds, algorithm = setup_config2(runtime, n_job)
    n_steps = int(math.floor(MAX_LENGTH / SAVE_AT))
    n_batches = (n_job + args.batch - 1) // args.batch
    rng = np.zeros(n_batches, np.uint32)
    with runtime.device_scope():
        d_handle = mesh.device(runtime)
        f_handle = field.device(runtime, _lib.MODEL_DTI)
        tracker = runtime.tracker()
        a = to_struct(algorithm)
        dev_seeds = runtime.to_device(seeds)
        host_seeds = runtime.pinned(seeds.shape, np.float32)
        host_seeds[...] = seeds
        lengths = np.empty(n_job, np.uint32)
        offsets = np.empty(n_job, np.uint64)
        total, steps = ctypes.c_uint64(), ctypes.c_uint64()
        kms, waves, launches = ctypes.c_float(), ctypes.c_uint32(), ctypes.c_uint32()

        def run(on_host):
            ptr = host_seeds.ctypes.data_as(ctypes.c_void_p) if on_host else ctypes.c_void_p(dev_seeds.data_ptr())
            _lib.check(lib.tg_tracker_run(tracker, ctypes.byref(a), d_handle, f_handle, ptr, 1 if on_host else 0,
                                          n_job, args.batch, rng.ctypes.data_as(ctypes.c_void_p), SAVE_AT, n_steps,
                                          lengths.ctypes.data_as(ctypes.c_void_p),
                                          offsets.ctypes.data_as(ctypes.c_void_p), ctypes.byref(total),
                                          ctypes.byref(steps), sh))
            _lib.check(lib.tg_tracker_stats(tracker, ctypes.byref(kms), ctypes.byref(waves), ctypes.byref(launches)))
            return int(steps.value), int(total.value), float(kms.value), int(launches.value)

        warm = 0
        for _ in range(args.warmup):
            warm = max(warm, run(False)[1])
        out_host = runtime.pinned((int(warm * 1.25) + 1024, 3), np.float32)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        sampler = ClockSampler(0)
        with sampler:
            torch.cuda.synchronize()
            ev0.record(runtime.stream)
            dev_steps = dev_points = n_launch = 0
            kernel_ms = 0.0
            for _ in range(args.steps):
                st, pts, k, nl = run(False)
                dev_steps, dev_points, kernel_ms, n_launch = dev_steps + st, dev_points + pts, kernel_ms + k, \
                    n_launch + nl
            ev1.record(runtime.stream)
            torch.cuda.synchronize()
            dev_ms = ev0.elapsed_time(ev1)
            ev0.record(runtime.stream)
            e2e_steps = h2d = d2h = 0
            for _ in range(args.steps):
                st, pts, _, _ = run(True)
                if pts > out_host.shape[0]:
                    out_host = runtime.pinned((pts, 3), np.float32)
                _lib.check(lib.tg_tracker_copy_points(tracker, out_host.ctypes.data_as(ctypes.c_void_p), 0, pts, 1,
                                                      sh))
                e2e_steps += st
                h2d += seeds.nbytes + rng.nbytes
                d2h += pts * 12 + n_job * 12
            ev1.record(runtime.stream)
            torch.cuda.synchronize()
            e2e_ms = ev0.elapsed_time(ev1)
    peak, peak_kind = measured_peaks()
    kernel_sps = dev_steps / (kernel_ms / 1e3)
    c2_tps = traffic_per_step("track_persistent_config2.md")
    info = mesh.info(runtime)
    line = {
        "metric": METRIC, "value": dev_steps / (dev_ms / 1e3), "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dev_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator; no dataset)",
        "workload": "config2",
        "config": {"workload": C2_WORKLOAD, "seeds_per_step": n_job, "batch_size": args.batch,
                   "mesh": info, "cache": "BVH (34 MB) and tensor volume (13 MB) are L2-resident by design"},
        "streamlines_per_s": n_job * args.steps / (dev_ms / 1e3),
        "points_per_step": dev_points / args.steps,
        "e2e": {"value": e2e_steps / (e2e_ms / 1e3), "unit": UNIT, "h2d_bytes_per_step": int(h2d / args.steps),
                "d2h_bytes_per_step": int(d2h / args.steps)},
        "gpu_launches": n_launch,
        "roofline": {"bound": "hbm", "achieved": kernel_sps * C2_BYTES_PER_STEP / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": kernel_sps * C2_BYTES_PER_STEP / 1e9 / peak,
                     "traffic": (c2_tps * dev_steps / args.steps) if c2_tps is not None else None,
                     "traffic_source": "DRAM bytes per accepted step of the 200k-seed ncu capture "
                                       "(profiles/track_persistent_config2.md) x the steps of one launch",
                     "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                     "bytes_per_step": C2_BYTES_PER_STEP,
                     "note": "bytes exclude the BVH nodes and triangles read near the surface",
                     "kernel_ms_per_step": kernel_ms / args.steps},
        "clocks": sampler.summary(),
    }
    if not args.no_cpu_baseline:
        from oracle import oracle as O

        threads = os.cpu_count() or 1
        n_sample = min(n_job, 200 * threads)
        case = O.Case(field=field.values, field_inv_affine=field.inverse_affine, model=O.MODEL_DTI,
                      algorithm=O.ALGO_TRANSPORT, step_size=C2_STEP, gamma=1.0, save_at=SAVE_AT, n_steps=n_steps,
                      mesh=O.BoundaryBvh.build(mesh.vertices, mesh.faces))
        t0 = time.perf_counter()
        _, _, st = case.tractogram(seeds[:n_sample], n_threads=threads, return_steps=True)
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": st / dt, "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": f"first {n_sample} seeds ({st} steps, {dt:.1f} s); plain-C oracle with "
                                          "the reference's BVH traversal, OpenMP over seeds"}
    print(json.dumps(line), flush=True)


SERVE_WORKLOAD = ("config4 serving: 8 resident SH lmax 8 volumes (64^3, 96x96x60, 128^3, 145x174x145, two "
                  "each, 2 mm) and 2 resident mesh boundaries (199k-triangle surfaces on the two 96x96x60 volumes); "
                  "Poisson arrivals; each request picks a volume uniformly, seeds log-U[1k, 2M], 70% Transport / "
                  "30% Diffusion (noise_variance U[0.05, 0.2]), step 0.2 mm, save_at 1 and maximum length 300 mm "
                  "(the reference defaults), batches of 50000; server HBM budget 150 GB minus the resident "
                  "volumes")


def setup_serving(runtime, pool_seeds=2_000_000):
    import tractography_b200 as tg
    from tractography_b200 import synthetic

    volumes = []
    shapes = list(synthetic.MIXED_SHAPES) * 2
    for i, shape in enumerate(shapes):
        fod, mask = synthetic.bundle_field(shape, lmax=8, seed=100 + i)
        field = tg.field.Image(fod)
        if i in (1, 5):
            v, f = synthetic.config2_surface(shape=shape, frequency=100)
            domain = tg.domain.Mesh(v, f)
            seeds = synthetic.seeds_inside(lambda q, d=domain: tg.domain.contains(d, q, runtime), v.min(axis=0),
                                           v.max(axis=0), pool_seeds, seed=i)
        else:
            domain = tg.domain.Image(mask)
            seeds = synthetic.uniform_seeds(mask, pool_seeds, seed=i)
        field.device(runtime, 0)
        domain.device(runtime)
        volumes.append((field, domain, seeds, field.values.nbytes))
    return volumes


def make_request(volumes, rng):
    import tractography_b200 as tg
    from tractography_b200 import jobs as jobs_module

    field, domain, pool, _ = volumes[int(rng.integers(0, len(volumes)))]
    n = int(np.exp(rng.uniform(np.log(1e3), np.log(2e6))))
    start = int(rng.integers(0, len(pool) - n + 1))
    model = tg.local.RealSymmetricSphericalHarmonics(45)
    if rng.uniform() < 0.7:
        alg = tg.algorithm.Transport(model, step_size=0.2, gamma=1.0)
    else:
        alg = tg.algorithm.Diffusion(model, step_size=0.2, gamma=1.0, noise_variance=float(rng.uniform(0.05, 0.2)),
                                     seed=int(rng.integers(1 << 31)))
    return jobs_module.prepare(field, pool[start:start + n], domain, alg, save_at=1.0,
                               maximum_streamline_length=300.0, batch_size=50000)


def run_serve_burst(args):
    """The mixed workload's jobs submitted to the server at once, against one batched run of them."""
    import torch

    import tractography_b200 as tg
    from tractography_b200 import _lib
    from tractography_b200 import jobs as jobs_module
    from tractography_b200.serve import Server

    torch.cuda.set_device(0)
    runtime = tg.CudaRuntime(0)
    jobs = build_mixed_jobs(args.jobs)
    kms, waves, launches = ctypes.c_float(), ctypes.c_uint32(), ctypes.c_uint32()
    for _ in range(2):                          # the second run is the one reported
        work = jobs_module.run_jobs_packed(jobs, runtime).steps
        _lib.check(runtime.lib.tg_tracker_stats(runtime.tracker(), ctypes.byref(kms), ctypes.byref(waves),
                                                ctypes.byref(launches)))
    batched_kernel_ms = float(kms.value)
    runs = []
    sampler = ClockSampler(0)
    with sampler:
        for _ in range(2):
            with Server(runtime, hbm_budget_bytes=150e9, pool_points=256 << 20, epoch_steps=args.epoch_steps,
                        epoch_seconds=args.epoch_ms * 1e-3, max_requests=128) as server:
                t0 = time.perf_counter()
                for job in jobs:
                    server.submit(job)
                done, polls = 0, 0
                while done < len(jobs):
                    done += len([server.take(rid, points=False) for rid in server.poll()])
                    polls += 1
                    if polls > 200000:
                        raise RuntimeError("burst did not finish")
                wall = time.perf_counter() - t0
                st = server.stats()
            runs.append({"wall_s": wall, "busy_s": st.busy_seconds, "kernel_s": st.kernel_seconds,
                         "between_s": st.between_seconds, "harvest_s": st.harvest_seconds, "epochs": st.epochs,
                         "steps": st.steps})
        for _ in range(3):                      # the batched run again, under the same clock record
            work = jobs_module.run_jobs_packed(jobs, runtime).steps
            _lib.check(runtime.lib.tg_tracker_stats(runtime.tracker(), ctypes.byref(kms), ctypes.byref(waves),
                                                    ctypes.byref(launches)))
            batched_kernel_ms = min(batched_kernel_ms, float(kms.value))
    r = runs[-1]
    line = {"metric": METRIC, "value": r["steps"] / r["busy_s"], "unit": UNIT, "n_gpus": 1, "steps": 1,
            "warmup": 1, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded generator; no dataset)", "workload": "serve-burst",
            "config": {"workload": "the 64 mixed jobs submitted at once to the server",
                       "epoch_steps": args.epoch_steps, "epoch_ms": args.epoch_ms},
            "server": r, "server_kernel_steps_per_s": r["steps"] / r["kernel_s"],
            "batched_kernel_ms": batched_kernel_ms, "batched_steps": work,
            "batched_kernel_steps_per_s": work / (batched_kernel_ms / 1e3), "clocks": sampler.summary()}
    print(json.dumps(line), flush=True)


def run_serve(args):
    """Config 4: continuous-batching server under Poisson arrivals; p50/p99 latency per rate."""
    import torch

    import tractography_b200 as tg
    from tractography_b200.serve import Server

    if args.burst:
        return run_serve_burst(args)
    torch.cuda.set_device(0)
    runtime = tg.CudaRuntime(0)
    volumes = setup_serving(runtime)
    resident = sum(v[3] for v in volumes)
    rates = [float(r) for r in args.rates.split(",")]
    sweep = []
    sampler = ClockSampler(0)
    with sampler:
        for rate in rates:
            rng = np.random.default_rng(int(rate * 1000))
            n_req = max(5, int(rate * args.duration))
            arrivals = np.cumsum(rng.exponential(1.0 / rate, n_req))
            offered = 0
            server = Server(runtime, hbm_budget_bytes=150e9 - resident, pool_points=256 << 20,
                            epoch_steps=args.epoch_steps, epoch_seconds=args.epoch_ms * 1e-3, max_requests=128)
            latency, seeds_done = [], 0
            client = {"prepare_s": 0.0, "submit_s": 0.0, "poll_s": 0.0, "take_s": 0.0, "idle_s": 0.0}
            t0 = time.perf_counter()
            submitted = 0
            while len(latency) < n_req:
                now = time.perf_counter() - t0
                while submitted < n_req and arrivals[submitted] <= now:
                    c0 = time.perf_counter()
                    job = make_request(volumes, rng)
                    c1 = time.perf_counter()
                    offered += job.n_seeds
                    server.submit(job)
                    client["prepare_s"] += c1 - c0
                    client["submit_s"] += time.perf_counter() - c1
                    submitted += 1
                c0 = time.perf_counter()
                finished = server.poll()
                c1 = time.perf_counter()
                client["poll_s"] += c1 - c0
                for rid in finished:
                    _, _, lengths, seconds = server.take(rid, points=False)
                    latency.append(seconds)
                    seeds_done += len(lengths)
                client["take_s"] += time.perf_counter() - c1
                if not finished and server.active == 0 and server.pending == 0:
                    if submitted == n_req:
                        raise RuntimeError("the server holds no work but requests are unfinished")
                    c0 = time.perf_counter()
                    time.sleep(max(0.0, min(0.002, arrivals[submitted] - (time.perf_counter() - t0))))
                    client["idle_s"] += time.perf_counter() - c0
                if time.perf_counter() - t0 > 600.0:
                    raise RuntimeError(f"rate {rate}: requests still unfinished after 600 s")
            wall = time.perf_counter() - t0
            st = server.stats()
            server.close()
            lat = np.array(latency)
            sweep.append({"rate_per_s": rate, "requests": n_req, "p50_s": float(np.percentile(lat, 50)),
                          "p99_s": float(np.percentile(lat, 99)), "mean_s": float(lat.mean()),
                          "steps": st.steps, "epochs": st.epochs, "busy_s": st.busy_seconds, "wall_s": wall,
                          "client": client,
                          "kernel_s": st.kernel_seconds, "between_s": st.between_seconds,
                          "harvest_s": st.harvest_seconds,
                          "steps_per_s": st.steps / max(1e-9, st.busy_seconds),
                          "streamlines_per_s": seeds_done / max(1e-9, st.busy_seconds),
                          "offered_seeds_per_s": float(offered / arrivals[-1])})
            print(json.dumps({"rate": rate, **sweep[-1]}), file=sys.stderr, flush=True)
    best = max(x["steps_per_s"] for x in sweep)
    line = {"metric": METRIC, "value": best, "unit": UNIT, "n_gpus": 1, "steps": len(rates), "warmup": 0,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded generator; no dataset)", "workload": "serve",
            "config": {"workload": SERVE_WORKLOAD, "rates_per_s": rates, "arrival_seconds": args.duration,
                       "epoch_steps": args.epoch_steps, "epoch_ms": args.epoch_ms,
                       "latency": "submission to completion on the device (all streamlines "
                                                       "harvested into the request's result buffer)"},
            "sweep": sweep, "clocks": sampler.summary()}
    print(json.dumps(line), flush=True)


def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "mixed":
        run_mixed(args)
    elif args.workload == "config2":
        run_config2(args)
    elif args.workload == "config0":
        run_config0(args)
    elif args.workload in ("tod", "connectome"):
        run_product(args)
    elif args.workload == "serve":
        run_serve(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
