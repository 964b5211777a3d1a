"""Autotuner on the GPU: it times real candidates and leaves the best applied."""

import pytest

import tractography_b200 as tg
from tractography_b200 import autotune
from tractography_b200 import jobs as jobs_module

from helpers import small_config0

pytestmark = pytest.mark.gpu


def test_tune_on_device(monkeypatch, tmp_path):
    monkeypatch.setenv(autotune.CACHE_ENV, str(tmp_path / "tune.json"))
    field, domain, seeds = small_config0(n_voxels=16, n_seeds=4000, seed=2)
    alg = tg.algorithm.Transport(tg.local.RealSymmetricSphericalHarmonics(45), step_size=0.1)
    job = jobs_module.prepare(field, seeds, domain, alg, save_at=0.25, maximum_streamline_length=30.0)
    runtime = tg.CudaRuntime()
    cands = [(0, 0, 0), (2, 0, 0), (0, 8, 2)]
    res = autotune.tune(runtime, job, candidates=cands, sample_seeds=4000)
    assert tuple(res["tuning"]) in cands
    assert all(v > 0 for v in res["steps_per_s"].values())
    t = runtime.tuning()
    assert (t["blocks_per_sm"], t["compact_lanes"], t["compact_rounds"]) == tuple(res["tuning"])
