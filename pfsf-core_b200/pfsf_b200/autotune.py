"""Autotuner of the batched tolerance solve's launch shapes.

    python -m pfsf_b200.autotune [--out FILE] [--islands N] [--budget S]

Parameters tuned (pfsf_tuning, include/pfsf/pfsf_b200.h): the cluster size
for big islands (1, 4, 8 CTAs), the island size from which clusters take
over from single CTAs, the size below which single warps take islands, the
Chebyshev smoothing degree and the lower end of its interval, the V-cycle's
coarse-correction weight, the coarse-level size from which one warp runs the
rest of the cycle, the smoothing steps on the coarsest level, the inner
PCG's stopping floor, and the size from which one island takes the whole GPU.  Method: timed trials -- the device time of a resident solve to
the benchmark tolerance (median of `reps`) -- by coordinate descent from the
current values, on a size-bucketed island set drawn like the benchmark's
(per-axis log-uniform sides scaled to the set's active-voxel target); the
whole-GPU threshold is decided on one island above 2^21 voxels, solved by
the whole GPU and by a cluster.  The winner is written as the section of the
tuning file for this GPU model and SM count; pfsf_init reads it from there
(PFSF_TUNE_FILE, else tune/pfsf_tune.txt beside the library's lib/ directory).
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import capi, synth

DEFAULT_FILE = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "tune", "pfsf_tune.txt")
KEYS = ("cluster", "cluster_min_voxels", "grid_min_voxels", "warp_max_voxels", "cheb_k", "cheb_lower",
        "coarse_weight", "tail_cells", "coarse_sweeps", "inner_eta")
FLOAT_KEYS = ("cheb_lower", "coarse_weight", "inner_eta")
CANDIDATES = {
    "cluster": [1, 4, 8],
    "cluster_min_voxels": [32768, 65536, 131072, 262144, 524288],
    "warp_max_voxels": [0, 1024, 2048],
    "cheb_k": [2, 3, 4],
    "cheb_lower": [0.05, 0.1, 0.15, 0.2, 0.3],
    # above 1.8 the preconditioner's SPD margin gets thin once the coarse
    # operator is rounded and solved inexactly: 1.9 measured 1.2 % faster on
    # the benchmark set, not enough to trade robustness on other islands
    "coarse_weight": [1.0, 1.4, 1.6, 1.8],
    "tail_cells": [0, 64, 128, 256, 512, 2048],
    "coarse_sweeps": [1, 2, 3, 4, 6],
    "inner_eta": [3e-5, 1e-4, 3e-4, 1e-3],
}


def device_key():
    """'<device name> <SM count>' as the engine matches tuning sections."""
    import torch
    p = torch.cuda.get_device_properties(torch.cuda.current_device())
    return f"{p.name} {p.multi_processor_count}"


def _register(eng, isls, first_id):
    ids, keep = [], []
    for k, isl in enumerate(isls):
        iid = first_id + k
        if eng.add_island(iid, isl.dims) != capi.PFSF_OK:
            raise RuntimeError("pfsf_add_island failed")
        phi = np.zeros(isl.n, np.float32)
        keep.append(phi)
        if eng.register_kappa(iid, phi, isl.source, isl.kappa, isl.vtype) != capi.PFSF_OK:
            raise RuntimeError("pfsf_register_island_kappa failed")
        ids.append(iid)
    return ids, keep


def _time(eng, ids, tol, reps):
    """Median device ms of resident cold-start solves (all islands must converge)."""
    flags = capi.SOLVE_NO_UPLOAD | capi.SOLVE_NO_READBACK | capi.SOLVE_COLD_START
    ms = []
    for _ in range(reps):
        rc, st = eng.solve(ids, tol=tol, flags=flags)
        if rc != capi.PFSF_OK or st.islands_converged != len(ids):
            return float("inf")
        ms.append(st.device_ms)
    return float(np.median(ms))


def tune(eng, islands=4096, target_active=6.0e7, big_dims=(160, 160, 96), tol=1e-6, reps=3, budget_s=300.0,
         seed=17, candidates=None, log=None):
    """Coordinate descent over the launch-shape parameters on engine `eng`
    (initialised, batched mode, BF16 storage).  Returns (best tuning dict,
    trial log)."""
    cands = dict(CANDIDATES if candidates is None else candidates)
    t_end = time.monotonic() + budget_s
    trials = []
    rc, t0 = eng.tuning()
    best = {k: (round(float(getattr(t0, k)), 6) if k in FLOAT_KEYS else getattr(t0, k)) for k in KEYS}
    eng.set_solve_mode(capi.SOLVE_BATCHED)
    eng.set_precision(capi.PREC_BF16)
    isls, _ = synth.batch(islands, seed=seed, target_active=target_active)
    ids, keep = _register(eng, isls, 1)
    eng.solve(ids, tol=tol, flags=capi.SOLVE_COLD_START)  # arena built and uploaded once

    def trial(params):
        if eng.set_tuning(**params) != capi.PFSF_OK:
            return float("inf")
        ms = _time(eng, ids, tol, reps)
        trials.append({"params": dict(params), "ms": ms})
        if log:
            log(json.dumps(trials[-1]))
        return ms

    best_ms = trial(best)
    for key in ("cluster", "cluster_min_voxels", "tail_cells", "cheb_k", "cheb_lower", "coarse_weight",
                "coarse_sweeps", "inner_eta", "warp_max_voxels"):
        for v in cands.get(key, []):
            if time.monotonic() > t_end:
                break
            if v == best[key]:
                continue
            p = dict(best, **{key: v})
            ms = trial(p)
            if ms < best_ms:
                best, best_ms = p, ms
    # whole-GPU tier threshold, on one island above 2^21 voxels
    if big_dims and time.monotonic() < t_end:
        big = synth.noise_island(tuple(big_dims), seed=seed + 1)
        bid, bkeep = _register(eng, [big], 100000)
        eng.solve(bid, tol=tol, flags=capi.SOLVE_COLD_START)
        res = {}
        for thr in (big.n, big.n + 1):  # the island on the whole GPU / on a cluster
            eng.set_tuning(**dict(best, grid_min_voxels=thr))
            res[thr] = _time(eng, bid, tol, reps)
            trials.append({"params": dict(best, grid_min_voxels=thr), "ms": res[thr], "island": list(big.dims)})
            if log:
                log(json.dumps(trials[-1]))
        if res[big.n] > res[big.n + 1]:
            # a cluster beat the whole GPU at this size: raise the threshold above it
            best["grid_min_voxels"] = max(best["grid_min_voxels"], 2 * big.n)
        else:
            best["grid_min_voxels"] = min(best["grid_min_voxels"], big.n)
        eng.L.pfsf_remove_island(eng.h, bid[0])
        del bkeep
    eng.set_tuning(**best)
    for iid in ids:
        eng.L.pfsf_remove_island(eng.h, iid)
    del keep
    return best, trials


def write_section(path, key, params, note=""):
    """Writes (or replaces) the [key] section of a tuning file."""
    lines = []
    if os.path.exists(path):
        with open(path) as f:
            lines = f.read().splitlines()
    out, skip = [], False
    for ln in lines:
        s = ln.strip()
        if s.startswith("[") and s.endswith("]"):
            skip = s[1:-1].strip() == key
        if not skip:
            out.append(ln)
    while out and not out[-1].strip():
        out.pop()
    if not out:
        out = ["# Launch shapes of the batched tolerance solve, one section per GPU model and SM count,",
               "# written by pfsf_b200/autotune.py (timed trials) and read by pfsf_init."]
    out.append("")
    out.append(f"[{key}]")
    if note:
        out.append(f"# {note}")
    for k in KEYS:
        if k in params:
            out.append(f"{k} = {float(params[k]):g}" if k in FLOAT_KEYS else f"{k} = {int(params[k])}")
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=DEFAULT_FILE)
    ap.add_argument("--islands", type=int, default=4096)
    ap.add_argument("--target-active", type=float, default=6.0e7)
    ap.add_argument("--budget", type=float, default=300.0)
    ap.add_argument("--reps", type=int, default=3)
    a = ap.parse_args()
    eng = capi.Engine(capi.default_config(max_island_size=1 << 28, tick_budget_ms=1 << 30, vram=180 << 30))
    if eng.init() != capi.PFSF_OK:
        raise SystemExit("pfsf_init failed (CUDA device required)")
    t0 = time.monotonic()
    best, trials = tune(eng, islands=a.islands, target_active=a.target_active, budget_s=a.budget, reps=a.reps,
                        log=print)
    key = device_key()
    batch = [t for t in trials if "island" not in t]  # trials on the island set (not the large island)
    base = batch[0]["ms"]
    bm = min(t["ms"] for t in batch)
    write_section(a.out, key, best, note=(f"{len(trials)} trials in {time.monotonic() - t0:.0f} s on {a.islands} "
                                          f"islands: {base:.1f} ms -> {bm:.1f} ms per solve"))
    print(json.dumps({"device": key, "best": best, "trials": len(trials), "file": a.out}))
    eng.close()


if __name__ == "__main__":
    main()
