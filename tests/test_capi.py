"""The C ABI library loads and exports every function include/*.h declares (no GPU needed)."""

import ctypes
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from tractography_b200 import _lib

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    names = set()
    for header in (ROOT / "include").glob("*.h"):
        text = header.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(tg_[a-z_0-9]+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


def test_header_declares_the_abi():
    names = declared_functions()
    assert "tg_tractogram" in names and "tg_tracker_run" in names
    assert names == set(_lib.EXPORTS)


def test_library_loads_and_exports_every_declared_symbol():
    lib = _lib.load()
    for name in declared_functions():
        assert hasattr(lib, name), name
    assert lib.tg_abi_version() == 1
    assert lib.tg_status_string(0) == b"ok"
    assert lib.tg_status_string(5) == b"point pool exhausted"


def test_exports_are_c_symbols():
    out = subprocess.run(["nm", "-D", "--defined-only", str(_lib.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    assert declared_functions() <= exported


def test_invalid_arguments_fail_without_a_device():
    lib = _lib.load()
    out = ctypes.c_void_p()
    # null values are rejected before any CUDA call
    status = lib.tg_field_create(0, None, 1, 1, 1, 1, None, None, ctypes.byref(out))
    assert status == _lib.TG_ERR_INVALID_ARGUMENT
    assert b"null" in lib.tg_last_error()
    with pytest.raises(ValueError):
        _lib.check(status)
    assert lib.tg_tracker_set_slicing(None, 16) == _lib.TG_ERR_INVALID_ARGUMENT
    assert lib.tg_tracker_get_slicing(None, None) == _lib.TG_ERR_INVALID_ARGUMENT


def test_missing_library_fails_loudly(tmp_path, monkeypatch):
    """No CPU fallback: without libtg_b200.so the package raises instead of tracking on the host."""
    monkeypatch.setattr(_lib, "LIB_PATH", tmp_path / "absent.so")
    monkeypatch.setattr(_lib, "_lib", None)
    with pytest.raises(RuntimeError, match="not built"):
        _lib.load()


def _iterations_between_saves(step, save_at, n_points):
    """The reference loop's time accumulation (tracking.py:140-145) in binary32:
    iterations between consecutive saved points."""
    step, save_at = np.float32(step), np.float32(save_at)
    t, k, counts = np.float32(0.0), 0, []
    while len(counts) < n_points:
        t = np.float32(t + step)
        k += 1
        if t >= save_at:
            t = np.float32(t - save_at)
            counts.append(k)
            k = 0
    return counts


@pytest.mark.parametrize("step,save_at", [(0.001, 0.25), (0.0013, 0.25), (0.2, 0.25), (3e-6, 0.25),
                                          (0.37, 0.25), (0.001, 1.0), (7e-5, 0.3), (2.5e-6, 0.001)])
def test_step_bound_covers_the_reference_loop(step, save_at):
    lib = _lib.load()
    out = ctypes.c_uint64()
    assert lib.tg_step_bound(step, save_at, 1, ctypes.byref(out)) == 0
    per_point = out.value
    counts = _iterations_between_saves(step, save_at, 6)
    assert max(counts) <= per_point
    # tight enough to stop a runaway lane soon after the reference would have stopped
    assert per_point <= 2 * max(counts) + 64
    assert lib.tg_step_bound(step, save_at, 1200, ctypes.byref(out)) == 0
    assert out.value == 1200 * per_point


def test_non_terminating_step_sizes_are_rejected_without_a_device():
    """time + step == time below save_at: the reference loop would never end (tracking.py:140-145)."""
    lib = _lib.load()
    out = ctypes.c_uint64()
    half_ulp = np.float32(2.0 ** -27)   # half the spacing of binary32 values in [0.125, 0.25)
    # ties round to even: time 0.125 (an even multiple of the spacing) never moves
    assert np.float32(np.float32(0.125) + half_ulp) == np.float32(0.125)
    for step in (1e-9, float(half_ulp)):
        assert lib.tg_step_bound(step, 0.25, 1, ctypes.byref(out)) == _lib.TG_ERR_INVALID_ARGUMENT
        assert b"never end" in lib.tg_last_error()
    just_above = float(np.nextafter(half_ulp, np.float32(1.0)))
    assert lib.tg_step_bound(just_above, 0.25, 1, ctypes.byref(out)) == 0
    # a finite but absurd count is refused too (the per-lane step counter is 32-bit)
    assert lib.tg_step_bound(1e-8, 0.25, 1200, ctypes.byref(out)) == _lib.TG_ERR_INVALID_ARGUMENT
    assert b"2^32" in lib.tg_last_error()
    # every tracking entry point applies the rule before it looks at its handles
    algo = _lib.Algorithm(algorithm=0, step_size=1e-9, gamma=1.0, noise_variance=0.0, rng_mode=0, rng_seed=0)
    status = lib.tg_tractogram(ctypes.byref(algo), None, None, None, 1, 0.25, 1200, None, None, None)
    assert status == _lib.TG_ERR_INVALID_ARGUMENT and b"never end" in lib.tg_last_error()
    status = lib.tg_tractogram_noalloc(ctypes.byref(algo), None, None, None, 1, 1, None, 0.25, 1200, None, None,
                                       None)
    assert status == _lib.TG_ERR_INVALID_ARGUMENT and b"never end" in lib.tg_last_error()
    job = _lib.Job(algorithm=algo, n_seeds=1, batch_size=1, save_at=0.25, n_steps=1200)
    status = lib.tg_tracker_run_jobs(None, ctypes.byref(job), 1, 0, None, None, None, None, None)
    assert status == _lib.TG_ERR_INVALID_ARGUMENT
    with pytest.raises(ValueError, match="never end"):
        _lib.check(lib.tg_tractogram(ctypes.byref(algo), None, None, None, 1, 0.25, 1200, None, None, None))
    algo.step_size = 0.001
    status = lib.tg_tractogram(ctypes.byref(algo), None, None, None, 1, 0.25, 1200, None, None, None)
    assert status == _lib.TG_ERR_INVALID_ARGUMENT and b"domain and field" in lib.tg_last_error()
