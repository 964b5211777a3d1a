"""Autotuner for the tracker's launch shape and tail compaction.

No reference counterpart.  The knobs (``tg_tracker_set_tuning``) never
change a result, only the time: resident blocks of 128 lanes per SM, and
tail compaction (warps left with at most ``compact_lanes`` live streamlines
after the queue drains hand them to ``compact_rounds`` follow-up launches).
``tune`` times a bounded sample of the caller's own job under each candidate
with CUDA events (device time of the tracking launches) and keeps the
fastest; results are cached per device and code path in a JSON file.

``tune_server_epoch`` picks the server's epoch length the same way from a
latency/throughput objective.
"""

from __future__ import annotations

import ctypes
import json
import os
from pathlib import Path

import numpy as np

from . import _lib, tracking
from .algorithm import to_struct

DEFAULT_CANDIDATES = ((0, 0, 0), (4, 0, 0), (3, 0, 0), (0, 8, 2), (0, 16, 4))
CACHE_ENV = "TG_B200_TUNE_CACHE"


def _cache_path() -> Path:
    return Path(os.environ.get(CACHE_ENV, Path.home() / ".cache" / "tractography_b200" / "tuning.json"))


def _key(runtime, job) -> str:
    import torch

    name = torch.cuda.get_device_name(runtime.device)
    model = type(job.algorithm.local_model).__name__
    return "|".join([name, model, str(job.algorithm.local_model.n_parameters), type(job.algorithm).__name__,
                     type(job.domain).__name__])


def load_cache() -> dict:
    path = _cache_path()
    try:
        return json.loads(path.read_text())
    except (OSError, ValueError):
        return {}


def _store(key: str, value: dict) -> None:
    path = _cache_path()
    data = load_cache()
    data[key] = value
    try:
        path.parent.mkdir(parents=True, exist_ok=True)
        path.write_text(json.dumps(data, indent=1, sort_keys=True))
    except OSError:
        pass


def time_job(runtime, job, seeds: np.ndarray, repeats: int = 2) -> tuple[float, int]:
    """Device milliseconds of the tracking launches and accepted steps of one run."""
    n = len(seeds)
    lengths = np.empty(max(1, n), np.uint32)
    offsets = np.empty(max(1, n), np.uint64)
    total, steps = ctypes.c_uint64(), ctypes.c_uint64()
    kms, waves, launches = ctypes.c_float(), ctypes.c_uint32(), ctypes.c_uint32()
    n_batches = (n + job.batch_size - 1) // job.batch_size
    rng = np.ascontiguousarray(job.batch_rng_seeds[:n_batches], dtype=np.uint32)
    with runtime.device_scope():
        d_h, f_h = tracking._handles(job.algorithm, job.domain, job.field, runtime)
        a = to_struct(job.algorithm, 0, job.philox_key, 0)
        d_seeds = runtime.to_device(seeds)
        best = float("inf")
        for _ in range(repeats):
            _lib.check(runtime.lib.tg_tracker_run(
                runtime.tracker(), ctypes.byref(a), d_h, f_h, ctypes.c_void_p(d_seeds.data_ptr()), 0, n,
                job.batch_size, rng.ctypes.data_as(ctypes.c_void_p), job.save_at, job.n_steps,
                lengths.ctypes.data_as(ctypes.c_void_p), offsets.ctypes.data_as(ctypes.c_void_p), ctypes.byref(total),
                ctypes.byref(steps), ctypes.c_void_p(runtime.stream_handle)))
            _lib.check(runtime.lib.tg_tracker_stats(runtime.tracker(), ctypes.byref(kms), ctypes.byref(waves),
                                                    ctypes.byref(launches)))
            best = min(best, kms.value)
    return best, int(steps.value)


def tune(runtime, job, candidates=DEFAULT_CANDIDATES, sample_seeds: int = 200_000, use_cache: bool = True,
         apply: bool = True) -> dict:
    """Pick the fastest tuning for `job`'s code path on this device.

    Times ``sample_seeds`` seeds of the job (the whole job when smaller)
    under every candidate (blocks_per_sm, compact_lanes, compact_rounds) and
    returns {"tuning": best, "steps_per_s": {candidate: rate}}; with
    ``apply`` the runtime's tracker keeps the best tuning.
    """
    key = _key(runtime, job)
    if use_cache:
        hit = load_cache().get(key)
        if hit is not None:
            if apply:
                runtime.set_tuning(*hit["tuning"])
            return hit
    seeds = np.ascontiguousarray(job.seeds[:sample_seeds], dtype=np.float32)
    before = runtime.tuning()
    rates = {}
    try:
        for cand in candidates:
            runtime.set_tuning(*cand)
            ms, steps = time_job(runtime, job, seeds)
            rates[str(tuple(cand))] = steps / (ms / 1e3) if ms > 0 else 0.0
    finally:
        runtime.set_tuning(before["blocks_per_sm"], before["compact_lanes"], before["compact_rounds"])
    best = max(candidates, key=lambda c: rates[str(tuple(c))])
    result = {"tuning": list(best), "steps_per_s": rates, "sample_seeds": len(seeds)}
    _store(key, result)
    if apply:
        runtime.set_tuning(*best)
    return result


def tune_server_epoch(make_server, jobs, candidates=(256, 1024, 4096), latency_weight: float = 1.0) -> dict:
    """Pick the server's epoch length: run the same burst of `jobs` through a
    server made by ``make_server(epoch_steps)`` for each candidate and keep
    the one minimising total busy time x (mean latency) ^ latency_weight."""
    scores = {}
    for epoch_steps in candidates:
        server = make_server(epoch_steps)
        try:
            for job in jobs:
                server.submit(job)
            latencies = []
            while len(latencies) < len(jobs):
                for rid in server.poll():
                    latencies.append(server.take(rid, points=False)[3])
            st = server.stats()
        finally:
            server.close()
        scores[epoch_steps] = {"busy_s": st.busy_seconds, "mean_latency_s": float(np.mean(latencies)),
                               "score": st.busy_seconds * float(np.mean(latencies)) ** latency_weight}
    best = min(candidates, key=lambda e: scores[e]["score"])
    return {"epoch_steps": best, "scores": scores}
