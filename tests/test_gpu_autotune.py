"""The autotuner: timed trials on a small island set, a tuning file section
for this GPU, and pfsf_init picking that section up (pfsf_get_tuning reports
the values and that they came from the file)."""
import os

import numpy as np
import pytest

from pfsf_b200 import autotune, capi

pytestmark = pytest.mark.gpu

ENV = ("PFSF_CLUSTER", "PFSF_CLUSTER_MIN_VOXELS", "PFSF_GRID_MIN_VOXELS", "PFSF_WARP_MAX_VOXELS", "PFSF_CHEB_K",
       "PFSF_CHEB_LOWER", "PFSF_COARSE_WEIGHT", "PFSF_TAIL_CELLS", "PFSF_COARSE_SWEEPS", "PFSF_INNER_ETA")


def _same(t, best):
    """Engine values equal the tuner's (float parameters to FP32 rounding)."""
    return all(abs(getattr(t, k) - best[k]) <= 1e-6 * max(1.0, abs(best[k])) if k in autotune.FLOAT_KEYS
               else getattr(t, k) == best[k] for k in autotune.KEYS)


def test_autotune_cache_is_read_at_init(lib_built, tmp_path, monkeypatch):
    for k in ENV:
        monkeypatch.delenv(k, raising=False)
    cfg = capi.default_config(max_island_size=1 << 26, tick_budget_ms=1 << 30)
    eng = capi.Engine(cfg)
    assert eng.init() == capi.PFSF_OK, "CUDA device required"
    best, trials = autotune.tune(eng, islands=48, target_active=3e5, big_dims=None, reps=1, budget_s=60.0,
                                 candidates={"cluster": [1, 4], "cheb_k": [2, 3], "coarse_weight": [1.4, 1.8],
                                             "tail_cells": [64, 512]})
    assert len(trials) >= 2 and np.isfinite(trials[0]["ms"])
    # the tuner leaves the winner set on its engine
    rc, t = eng.tuning()
    assert rc == capi.PFSF_OK and _same(t, best)
    eng.close()
    path = tmp_path / "pfsf_tune.txt"
    key = autotune.device_key()
    autotune.write_section(str(path), "Another GPU 7", dict(best, cluster=8, cheb_k=1))
    autotune.write_section(str(path), key, best, note="test")
    monkeypatch.setenv("PFSF_TUNE_FILE", str(path))
    e2 = capi.Engine(cfg)
    assert e2.init() == capi.PFSF_OK
    rc, t2 = e2.tuning()
    assert rc == capi.PFSF_OK and t2.source == 1, t2.as_dict()
    assert _same(t2, best), (t2.as_dict(), best)
    # out-of-range values are refused and change nothing
    assert e2.set_tuning(cluster=3) == capi.PFSF_ERROR_INVALID_ARG
    assert e2.set_tuning(cheb_k=0) == capi.PFSF_ERROR_INVALID_ARG
    assert e2.set_tuning(coarse_weight=2.0) == capi.PFSF_ERROR_INVALID_ARG
    assert e2.set_tuning(cheb_lower=0.0) == capi.PFSF_ERROR_INVALID_ARG
    assert e2.set_tuning(tail_cells=-1) == capi.PFSF_ERROR_INVALID_ARG
    assert e2.set_tuning(coarse_sweeps=0) == capi.PFSF_ERROR_INVALID_ARG
    assert e2.set_tuning(inner_eta=1.0) == capi.PFSF_ERROR_INVALID_ARG
    rc, t3 = e2.tuning()
    assert t3.cluster == best["cluster"] and t3.cheb_k == best["cheb_k"]
    # an environment override wins over the file
    e2.close()
    monkeypatch.setenv("PFSF_CHEB_K", "4")
    e3 = capi.Engine(cfg)
    assert e3.init() == capi.PFSF_OK
    rc, t4 = e3.tuning()
    assert t4.cheb_k == 4 and t4.source == 2
    e3.close()
