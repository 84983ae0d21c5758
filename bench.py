#!/usr/bin/env python
"""Benchmark: ms per tick to a 1e-6 relative residual, batched mixed precision
vs plain FP32 per-island kernels, on one B200 (or N, one process per GPU).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (default "batch"): 4096 seeded islands, per-axis log-uniform sides
scaled to ~6e7 active voxels, value-noise occupancy 60 % kept to the anchored
26-connected component, three-material mix, point loads on 0.1 % of the top
surface (pfsf_b200.synth).  A tick solves every island from phi = 0 to
||s - A phi||_2 / ||s||_2 <= 1e-6 (FP64-evaluated) through the libpfsf C ABI:
one persistent launch, BF16 kappa / coarse operators in the preconditioner,
FP32 inner PCG, FP64 inner products and outer residual.

value     device ms per tick with inputs resident in HBM (CUDA events on the
          engine stream; the arena is far larger than L2, so nothing is cached
          between steps).
e2e       the same tick through pfsf_solve_to_tolerance with host buffers:
          H2D of kappa, source, type and phi0 from pinned memory, D2H of phi.
plain     the same islands solved one at a time with plain FP32 kernels
          (one grid-wide launch per operation), timed on a size-stratified
          sample and scaled by island count.
Multi-GPU: islands are independent, each rank solves its own workload
(weak scaling), no collective on the data path; the tick time is the max
over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "pfsf-core_b200"))

METRIC = "ms/tick to 1e-6 rel. residual: batched mixed-prec vs plain FP32, same B200"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["batch", "single", "adjoint", "fracture", "tick_dbb"], default="batch")
    ap.add_argument("--ticks", type=int, default=200, help="fracture workload: ticks")
    ap.add_argument("--fd-voxels", type=int, default=32)
    ap.add_argument("--dims", default="256,256,128", help="single workload: island sides x,y,z")
    ap.add_argument("--scaling", choices=["weak", "strong"], default="weak",
                    help="batch workload with N GPUs: every rank its own 4096 islands (weak) or one 4096-island "
                         "workload partitioned by active voxels (strong)")
    ap.add_argument("--islands", type=int, default=4096)
    ap.add_argument("--target-active", type=float, default=6.0e7)
    ap.add_argument("--tol", type=float, default=1e-6)
    ap.add_argument("--island-report", default="",
                    help="write one JSON line per island of the last timed solve (team, iterations, times)")
    ap.add_argument("--precision", choices=["bf16", "fp16", "fp32"], default="bf16")
    ap.add_argument("--cycle", choices=["v", "w"], default=None,
                    help="multigrid cycle of the batched solve: default W for the fracture workload (the "
                         "configuration asks for W), V otherwise")
    ap.add_argument("--amg", action="store_true",
                    help="tick_dbb workload: the aggregation correction at every PCG start (pfsf_set_amg)")
    ap.add_argument("--plain-sample", type=int, default=64)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    return ap.parse_args()


def dist_info():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def make_workload(args, rank):
    from pfsf_b200 import synth
    if args.workload == "single":
        isl = synth.noise_island(tuple(int(v) for v in args.dims.split(",")), seed=11 + rank)
        return [isl], {"grid_total": isl.n, "active_total": isl.n_active, "scale": 1.0}
    if args.scaling == "strong":
        # one workload, partitioned across the ranks by active voxels
        from pfsf_b200 import shard
        ws = int(os.environ.get("WORLD_SIZE", "1"))
        isls, meta = synth.batch(args.islands, seed=7, target_active=args.target_active,
                                 workers=min(32, os.cpu_count() or 1))
        mine = shard.plan_shards([i.n_active for i in isls], ws)[rank]
        isls = [isls[i] for i in mine]
        meta = dict(meta, grid_total=sum(i.n for i in isls), active_total=sum(i.n_active for i in isls))
        return isls, meta
    return synth.batch(args.islands, seed=7 + 1000 * rank, target_active=args.target_active,
                       workers=min(32, os.cpu_count() or 1))


def write_island_report(path, eng, ids, isls):
    from pfsf_b200.capi import IslandReport
    with open(path, "w") as f:
        for iid, isl in zip(ids, isls):
            rc, r = eng.island_report(int(iid))
            if rc != 0:
                raise RuntimeError(f"pfsf_island_solve_report({iid}) returned {rc}")
            f.write(json.dumps({"id": int(iid), "dims": [r.lx, r.ly, r.lz], "n": int(isl.n),
                                "active": int(isl.n_active), "levels": r.levels,
                                "team": IslandReport.TEAMS.get(r.team, str(r.team)), "team_ctas": r.team_ctas,
                                "inner": r.inner_iterations, "outer": r.outer_iterations,
                                "converged": r.converged, "rel_residual": r.rel_residual,
                                "solve_ms": r.solve_ms, "setup_ms": r.setup_ms,
                                "precond_ms": r.precond_ms, "start_ms": r.start_ms}) + "\n")


def stratified(isls, k):
    """k islands evenly spaced in size order (largest first)."""
    order = sorted(range(len(isls)), key=lambda i: -isls[i].n)
    if k >= len(order):
        return order
    step = len(order) / k
    return [order[int(j * step)] for j in range(k)]


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def _oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.lib()
    return O


def cpu_solve_islands(isls, idx, tol, threads):
    """Solves islands idx with the oracle's plain FP32 scheme (FP32 V-cycle
    PCG inside FP64 residual refinement, oracle/kappa_mg.c o_kappa_mgpcg32) on
    `threads` host threads: islands larger than half a thread's share of the
    set first, one at a time, each threaded across all host threads (OpenMP
    inside the solve); the rest one island per thread, largest first.
    Returns (wall s, [(island, seconds, threads used)], islands converged)."""
    import concurrent.futures as cf
    O = _oracle()
    order = sorted(idx, key=lambda i: -isls[i].n)
    share = sum(isls[i].n for i in order) / max(threads, 1)
    big = [i for i in order if threads > 1 and isls[i].n > share / 2]
    rest = [i for i in order if i not in set(big)]

    def run(i, nt):
        s = isls[i]
        t0 = time.perf_counter()
        _, _, rel, _ = O.kappa_mgpcg32(s.dims, s.kappa.astype(np.float64), s.vtype, s.source.astype(np.float64),
                                       tol=tol, maxit=100000, threads=nt)
        return i, time.perf_counter() - t0, nt, rel <= tol

    t0 = time.perf_counter()
    res = [run(i, threads) for i in big]
    with cf.ThreadPoolExecutor(max_workers=threads) as ex:
        res += list(ex.map(lambda i: run(i, 1), rest))
    wall = time.perf_counter() - t0
    return wall, [(r[0], r[1], r[2]) for r in res], sum(r[3] for r in res)


def cpu_baseline(isls, seconds, tol):
    """The plain FP32 scheme on the host cores (cpu_solve_islands), on an
    interleaved sample of the tick's islands (every m-th island in size order,
    so every size is represented), m chosen from a calibration solve so the
    sample takes about `seconds` on all threads.  The tick estimate scales the
    sample's wall time by grid voxels (the CPU passes sweep every cell of an
    island's box): all threads = wall x N_all / N_sample; one thread = the
    single-threaded per-island times of the sample, per grid voxel, x N_all."""
    threads = os.cpu_count() or 1
    order = sorted(range(len(isls)), key=lambda i: -isls[i].n)
    n_all = float(sum(i.n for i in isls))
    # calibration: the island at the 25th size percentile
    cal = order[len(order) // 4]
    _, tc, _ = cpu_solve_islands(isls, [cal], tol, 1)
    est_1t = tc[0][1] / isls[cal].n * n_all  # whole tick on one thread
    m = max(1, int(est_1t / threads / max(seconds, 1.0)))
    sample = order[m // 2::m] if (m > 1 and len(order) >= 2 * m) else order
    wall, recs, conv = cpu_solve_islands(isls, sample, tol, threads)
    n_s = float(sum(isls[i].n for i in sample))
    one = [(isls[i].n, t) for i, t, nt in recs if nt == 1]
    one_ms = (sum(t for _, t in one) / sum(n for n, _ in one) * n_all * 1000.0) if one else None
    return {"value": wall * 1000.0 * n_all / n_s, "unit": "ms/tick", "cores": threads, "kind": "port",
            "one_thread_ms": one_ms, "cpu": cpu_model(),
            "sample": (f"every {m}th island in size order: {len(sample)} of {len(isls)} islands, "
                       f"{n_s / n_all:.4f} of the grid voxels, {wall:.1f} s wall on {threads} threads, scaled by "
                       f"grid voxels; one-thread figure from the sample's single-threaded island times per grid "
                       f"voxel; converged {conv}/{len(sample)}"),
            "algorithm": (f"plain FP32 scheme on the host (oracle/kappa_mg.c): 8-colour RBGS V-cycle PCG in FP32 "
                          f"inside FP64 residual refinement, to {tol:g} FP64 relative residual; islands above half a "
                          f"thread's share threaded across all cores, the rest one per thread")}


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, gpu_index):
        self.rows = []
        self.p = None
        self.gpu = gpu_index

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.p = None
        return self

    def _read(self):
        for line in self.p.stdout:
            self.rows.append([v.strip() for v in line.split(",")])

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()

    def summary(self):
        mhz, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                mhz.append(float(r[1]))
                mx = float(r[2])
                for k, nm in enumerate(names):
                    if r[5 + k].lower().startswith("active"):
                        reasons.add(nm)
            except (ValueError, IndexError):
                pass
        return {"sm_mhz": float(np.median(mhz)) if mhz else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(mhz)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def traffic_model():
    """DRAM bytes per active voxel of the batched kernel from the committed ncu
    summary (profiles/batched_solve_traffic.json), or None."""
    try:
        with open(os.path.join(ROOT, "profiles", "batched_solve_traffic.json")) as f:
            return json.load(f)
    except (OSError, ValueError):
        return None


def run_reference(args):
    """The reference arm: the CPU scheme on the host cores for the same
    workload.  The K timed steps partition the tick's islands (step j takes
    every K-th island in size order from offset j), so together they solve
    every island of one tick once: value = the sum of the step times = one
    whole tick, measured; each step is a bounded, representative slice.
    Warm-up steps solve the 16 smallest islands."""
    ws, rank, _ = dist_info()
    if rank != 0:
        return
    isls, meta = make_workload(args, 0)
    threads = os.cpu_count() or 1
    order = sorted(range(len(isls)), key=lambda i: -isls[i].n)
    for _ in range(args.warmup):
        cpu_solve_islands(isls, order[-16:], args.tol, threads)
    k = max(args.steps, 1)
    times, conv, cpu_s = [], 0, 0.0
    for j in range(k):
        wall, recs, c = cpu_solve_islands(isls, order[j::k], args.tol, threads)
        times.append(wall * 1000.0)
        conv += c
        cpu_s += sum(t * nt for _, t, nt in recs)
    tick_ms = float(sum(times))
    cb = {"value": tick_ms, "unit": "ms/tick", "cores": threads, "kind": "port", "cpu": cpu_model(),
          "thread_seconds": cpu_s,
          "sample": (f"the whole tick: {len(isls)} islands split over {k} timed steps (every {k}th island in size "
                     f"order); islands above half a thread's share threaded across all cores, the rest one per "
                     f"thread, largest first; converged {conv}/{len(isls)}"),
          "algorithm": (f"plain FP32 scheme on the host (oracle/kappa_mg.c): 8-colour RBGS V-cycle PCG in FP32 "
                        f"inside FP64 residual refinement, to {args.tol:g} FP64 relative residual")}
    line = {"metric": METRIC, "value": tick_ms, "unit": "ms/tick", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": float(np.mean(times)), "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": {"workload": (f"{len(isls)} islands (log-uniform sides, scale {meta['scale']:.3f}), "
                                    f"{meta['grid_total']} grid / {meta['active_total']} active voxels, cold start, "
                                    f"tol {args.tol:g}"),
                       "islands": len(isls), "grid_voxels": meta["grid_total"],
                       "active_voxels": meta["active_total"],
                       "step": "1/K of the tick's islands; value = sum over the K steps = one tick"},
            "cpu_baseline": cb,
            "e2e": {"value": tick_ms, "unit": "ms/tick", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args):
    ws, rank, local = dist_info()
    isls, meta = make_workload(args, rank)  # CPU pool work happens before any CUDA use
    import torch
    from pfsf_b200 import capi

    torch.cuda.set_device(local)
    os.environ["PFSF_CUDA_DEVICE"] = str(local)
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device("cuda", local))
    cfg = capi.default_config(max_island_size=1 << 28, tick_budget_ms=1 << 30, vram=180 << 30)
    eng = capi.Engine(cfg)
    rc = eng.init()
    if rc != capi.PFSF_OK:
        raise RuntimeError(f"pfsf_init failed rc={rc}")
    host = []
    ids = []
    for k, isl in enumerate(isls):
        iid = k + 1
        assert eng.add_island(iid, isl.dims) == capi.PFSF_OK
        h = {"phi": np.zeros(isl.n, np.float32), "source": isl.source, "kappa": isl.kappa, "type": isl.vtype}
        assert eng.register_kappa(iid, h["phi"], h["source"], h["kappa"], h["type"]) == capi.PFSF_OK
        host.append(h)
        ids.append(iid)
    prec = {"bf16": capi.PREC_BF16, "fp16": capi.PREC_FP16, "fp32": capi.PREC_FP32}[args.precision]
    # the product path is the persistent launch in both workloads (a single
    # giant island takes its whole-GPU tier); the plain arm is per-island FP32
    mode = capi.SOLVE_BATCHED
    eng.set_solve_mode(mode)
    eng.set_precision(prec)
    eng.set_mg_cycle(capi.MG_W if args.cycle == "w" else capi.MG_V)
    rc, st0 = eng.solve(ids, tol=args.tol, flags=capi.SOLVE_COLD_START)  # builds and uploads the arena
    assert rc == capi.PFSF_OK
    resident = capi.SOLVE_NO_UPLOAD | capi.SOLVE_NO_READBACK | capi.SOLVE_COLD_START
    for _ in range(args.warmup):
        eng.solve(ids, tol=args.tol, flags=resident)
    stream = torch.cuda.ExternalStream(eng.stream())
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = eng.launches()
    stats = []
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            rc, st = eng.solve(ids, tol=args.tol, flags=resident)
            stats.append(st)
        ev1.record(stream)
        torch.cuda.synchronize()
    launches = eng.launches() - launches0
    ms = ev0.elapsed_time(ev1) / args.steps
    tuning = eng.tuning()[1].as_dict()  # launch shapes (tuning file / environment / defaults)
    if args.island_report and rank == 0:
        write_island_report(args.island_report, eng, ids, isls)
    if ws > 1:
        t = torch.tensor([ms], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
        torch.distributed.barrier()
    torch.cuda.synchronize()
    # e2e through the C ABI with host buffers (pinned by the engine at registration)
    h2d = sum(isl.n * (4 + 4 + 4 + 1) for isl in isls)
    d2h = sum(isl.n * 4 for isl in isls)
    e2e = []
    for _ in range(max(1, args.steps)):
        t0 = time.perf_counter()
        rc, st_e = eng.solve(ids, tol=args.tol, flags=capi.SOLVE_COLD_START)
        e2e.append((time.perf_counter() - t0) * 1000.0)
    e2e_ms = float(np.mean(e2e))
    if ws > 1:
        t = torch.tensor([e2e_ms], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_ms = float(t.item())
    kern_ms = float(np.mean([s.device_ms for s in stats]))
    conv = min(s.islands_converged for s in stats)
    maxrel = max(s.max_rel_residual for s in stats)
    alg_bytes = float(np.mean([s.algorithmic_bytes for s in stats]))
    peak, peak_kind = peaks()
    achieved = alg_bytes / (kern_ms * 1e-3) / 1e9
    tm = traffic_model()
    traffic = None
    # the committed capture is of k_batched; the whole-GPU tier (single workload)
    # has no capture at a size whose working set exceeds L2, so no traffic figure
    if tm and tm.get("dram_bytes_per_active_voxel") and mode == capi.SOLVE_BATCHED and args.workload == "batch":
        traffic = tm["dram_bytes_per_active_voxel"] * st0.active_voxels
    # FP64-oracle error (read the FP64 accumulator back): the oracle's FP64
    # multigrid CG (all host threads) solves the same island to 1e-11; for
    # the batch, 4 islands evenly spaced in size order (the largest included)
    oracle_err = None
    oracle_relres = None
    if rank == 0:
        O = _oracle()
        errs, rels = [], []
        for k in stratified(isls, 4):
            isl = isls[k]
            rc, x64 = eng.read_solution64(ids[k], isl.n)
            k64 = isl.kappa.astype(np.float64)
            s64 = isl.source.astype(np.float64)
            r = s64 - O.kappa_apply(isl.dims, k64, isl.vtype, x64)
            solid = isl.vtype == 1
            rels.append(float(np.linalg.norm(r[solid]) / np.linalg.norm(s64[solid])))
            xr, _, _ = O.kappa_mgpcg64(isl.dims, k64, isl.vtype, s64, tol=1e-11, maxit=5000,
                                       threads=os.cpu_count() or 1)
            errs.append(float(np.abs(x64 - xr).max() / max(np.abs(xr).max(), 1e-300)))
        oracle_relres = max(rels)
        oracle_err = max(errs)
    # the same persistent kernel with FP32 kappa / coarse storage: isolates
    # what the 16-bit storage contributes
    fp32_ms = None
    if args.precision != "fp32" and not args.no_plain and rank == 0:
        eng.set_solve_mode(capi.SOLVE_BATCHED)
        eng.set_precision(capi.PREC_FP32)
        eng.solve(ids, tol=args.tol, flags=capi.SOLVE_COLD_START)  # rebuilds the arena for FP32 storage
        ev2, ev3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        ev2.record(stream)
        nrep = max(1, min(args.steps, 5))
        for _ in range(nrep):
            rc, st32 = eng.solve(ids, tol=args.tol, flags=resident)
        ev3.record(stream)
        torch.cuda.synchronize()
        fp32_ms = ev2.elapsed_time(ev3) / nrep
        fp32_conv = st32.islands_converged
    # plain FP32 per-island kernels on a stratified sample
    plain_ms = None
    plain_note = None
    if not args.no_plain and rank == 0:
        sample = stratified(isls, args.plain_sample) if args.workload == "batch" else [0]
        sids = [ids[k] for k in sample]
        eng.set_solve_mode(capi.SOLVE_PER_ISLAND)
        eng.set_precision(capi.PREC_FP32)
        eng.solve(sids, tol=args.tol, flags=capi.SOLVE_COLD_START)
        rc, stp = eng.solve(sids, tol=args.tol, flags=resident)
        plain_ms = stp.device_ms * len(isls) / len(sample)
        plain_note = (f"{len(sample)} of {len(isls)} islands (size-stratified), {stp.device_ms:.1f} ms, "
                      f"converged {stp.islands_converged}/{len(sample)}, scaled by island count")
    # the CPU FP64 solve of the single 5 M-voxel island does not fit a bounded sample
    cb = (cpu_baseline(isls, args.cpu_seconds, args.tol)
          if (rank == 0 and ws == 1 and not args.no_cpu) else None)
    if rank == 0:
        line = {
            "metric": METRIC, "value": ms, "unit": "ms/tick", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": args.scaling,
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": ((f"{len(isls)} islands/GPU (log-uniform sides, scale {meta['scale']:.3f}), "
                                     if args.workload == "batch" else
                                     f"one {args.dims.replace(',', 'x')} noise island (60 % occupancy, anchored "
                                     "component), ")
                                    + f"{meta['grid_total']} grid / {meta['active_total']} active voxels, "
                                    f"cold start, tol {args.tol:g}"),
                       "islands": len(isls), "grid_voxels": meta["grid_total"], "active_voxels": meta["active_total"],
                       "mode": "batched persistent" if mode == capi.SOLVE_BATCHED else "per-island",
                       "precision": f"{args.precision} kappa/coarse, fp32 vectors, fp64 dots+outer residual",
                       "l2": "inputs and solve arena far larger than L2 (126 MB)"},
            "e2e": {"value": e2e_ms, "unit": "ms/tick", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "dram_gbs": (traffic / (kern_ms * 1e-3) / 1e9) if traffic else None,
                         "dram_frac": (traffic / (kern_ms * 1e-3) / 1e9 / peak) if traffic else None,
                         "note": ("achieved/frac: the engine's byte model (every array a pass touches counted "
                                  "once per pass) over the kernel time; dram_gbs/dram_frac: DRAM bytes from the "
                                  "committed ncu capture scaled to this workload over the same time -- islands "
                                  "stay L2-resident while their team solves them"),
                         "kernel": ("k_batched (persistent solve)" if args.workload == "batch"
                                    else "k_grid (whole-GPU persistent solve)"), "kernel_ms": kern_ms,
                         "algorithmic_bytes": alg_bytes},
            "cpu_baseline": cb,
            "clocks": clk.summary(),
            "gpu_launches": int(launches),
            "converged": f"{conv}/{len(isls)}", "max_rel_residual_fp64": maxrel,
            "fp64_oracle_error": oracle_err, "fp64_oracle_relres": oracle_relres,
            "plain_fp32_ms_per_tick": plain_ms, "plain_fp32_sample": plain_note,
            "speedup_vs_plain_fp32": (plain_ms / ms) if plain_ms else None,
            "batched_fp32_ms_per_tick": fp32_ms,
            "batched_fp32_converged": (f"{fp32_conv}/{len(isls)}" if fp32_ms else None),
            "speedup_vs_batched_fp32": (fp32_ms / ms) if fp32_ms else None,
            "inner_iterations_total": int(stats[-1].inner_iterations_total),
            "schedule": {"island_ms_sum": stats[-1].island_ms_sum, "island_ms_max": stats[-1].island_ms_max,
                         "span_ms": stats[-1].span_ms, "setup_ms_sum": stats[-1].setup_ms_sum,
                         "precond_ms_sum": stats[-1].precond_ms_sum,
                         "vcycle_ms_sum": {"fine": stats[-1].vcycle_fine_ms_sum,
                                           "coarse": stats[-1].vcycle_coarse_ms_sum,
                                           "tail": stats[-1].vcycle_tail_ms_sum},
                         "persistent_ctas": stats[-1].persistent_ctas,
                         "tuning": tuning,
                         "cycle": "W" if args.cycle == "w" else "V",
                         "smoother": os.environ.get("PFSF_SMOOTHER", "chebyshev(batched)")},
        }
        print(json.dumps(line), flush=True)
    eng.close()
    if ws > 1:
        torch.distributed.destroy_process_group()


def run_adjoint(args):
    """Calibration gradient over a trajectory: one 128x128x64 noise island,
    32 ticks with the load ramped linearly to 2x (checkpoint every 8 ticks),
    L = sum over ticks of [sum softplus(flux_in / rcomp - 1) + 1/2 ||phi_t -
    f_t phi_target||^2] + sum softplus(H / h_scale - 1) with H = max over
    ticks of psi_e (Amor split, the history update's formula) --
    pfsf_b200.adjoint.trajectory_loss; rcomp in Pa (flux in N over a 1 m^2
    face), phi_target = the solution for kappa perturbed by a seeded lognormal
    (sigma 0.2) factor, h_scale = half the largest psi_e of the last tick.
    Backward: every tick's device adjoint in reverse order, every tick but the
    last re-solved from its checkpoint first.  Reports ms per forward tick,
    the backward, the gradient's error against central differences
    (h = 2^-10 on kappa, --fd-voxels voxels, the whole trajectory re-evaluated
    per step) and, on a reduced 32x32x16 island over 8 ticks, against the
    oracle's FP64 trajectory gradient."""
    os.environ.setdefault("PFSF_GRID_MIN_VOXELS", str(1 << 18))  # a lone island takes the whole GPU
    from pfsf_b200 import adjoint as AD
    from pfsf_b200 import capi, synth
    import torch

    O = _oracle()
    eng = capi.Engine(capi.default_config(max_island_size=1 << 28, tick_budget_ms=1 << 30, vram=180 << 30))
    if eng.init() != capi.PFSF_OK:
        raise RuntimeError("pfsf_init failed")
    eng.set_solve_mode(capi.SOLVE_BATCHED)
    eng.set_precision({"bf16": capi.PREC_BF16, "fp16": capi.PREC_FP16, "fp32": capi.PREC_FP32}[args.precision])
    ticks = 32

    def setup(dims, seed, iid):
        isl = synth.noise_island(dims, seed=seed)
        rng = np.random.default_rng(seed)
        sess = AD.Session(eng, iid, isl.dims, isl.vtype, tol=1e-10, max_iter=4000)
        k_target = (isl.kappa * np.exp(0.2 * rng.standard_normal(isl.n))).astype(np.float32)
        phi_target = sess.solve(k_target, isl.source.astype(np.float32))
        rcomp = np.maximum(isl.rcomp.astype(np.float64), 1.0) * 1e6
        x2 = sess.solve(isl.kappa, (2.0 * isl.source).astype(np.float32))
        psi, _ = O.amor_psi64(isl.dims, isl.kappa.astype(np.float64), isl.vtype, x2)
        return isl, rng, sess, phi_target, rcomp, 0.5 * float(psi.max())

    isl, rng, sess, phi_target, rcomp, hs = setup((128, 128, 64), 41, 1)
    kt = torch.tensor(isl.kappa.astype(np.float64), requires_grad=True)
    st = torch.tensor(isl.source.astype(np.float64))
    for _ in range(max(args.warmup, 1)):
        sess.solve(isl.kappa, isl.source)
    sess.recomputes = 0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    L, phis, H = AD.trajectory_loss(sess, kt, st, rcomp, phi_target, ticks=ticks, ramp=2.0, checkpoint_every=8,
                                    h_scale=hs)
    torch.cuda.synchronize()
    t_fwd = (time.perf_counter() - t0) * 1000.0
    t0 = time.perf_counter()
    L.backward()
    torch.cuda.synchronize()
    t_bwd = (time.perf_counter() - t0) * 1000.0
    adj_stats = sess.last_stats
    g = kt.grad.detach().cpu().numpy()
    vox = rng.choice(np.where(isl.vtype != 0)[0], args.fd_voxels, replace=False)
    phis0 = [p.detach().numpy() for p in phis]
    t0 = time.perf_counter()
    fd, kink = AD.trajectory_finite_difference(sess, isl.kappa.astype(np.float32), isl.source, phis0, rcomp,
                                               phi_target, vox, ramp=2.0, h_scale=hs)
    t_fd = time.perf_counter() - t0
    ok = ~kink
    rel = np.abs(g[vox][ok] - fd[ok]) / np.maximum(np.abs(fd[ok]), 1e-300)
    # FP64 oracle gradient of the same trajectory loss on a reduced island
    risl, _, rsess, rpt, rrc, rhs_ = setup((32, 32, 16), 43, 2)
    rk = torch.tensor(risl.kappa.astype(np.float64), requires_grad=True)
    Lr, _, _ = AD.trajectory_loss(rsess, rk, torch.tensor(risl.source.astype(np.float64)), rrc, rpt, ticks=8,
                                  ramp=2.0, checkpoint_every=4, h_scale=rhs_)
    Lr.backward()
    Lo, gko, _, _ = O.trajectory_grad64(risl.dims, risl.kappa.astype(np.float64), risl.vtype,
                                        risl.source.astype(np.float64), rrc, rpt, 8, 2.0, rhs_,
                                        threads=os.cpu_count() or 1)
    oracle_err = float(np.abs(rk.grad.detach().cpu().numpy() - gko).max() / np.abs(gko).max())
    line = {
        "metric": "config-4 adjoint: max rel. error of dL/dkappa of the 32-tick trajectory loss vs central FD "
                  "(non-kink voxels)",
        "value": float(rel.max()) if rel.size else None, "unit": "relative", "higher_is_better": False,
        "n_gpus": 1, "data": "synthetic", "dtype": "f32",
        "config": {"workload": "one 128x128x64 noise island (60 % occupancy, anchored component), 32 ticks, "
                               "load ramped 1x->2x, checkpoint every 8 ticks, loss over every tick + history term",
                   "active_voxels": int(isl.n_active), "precision": args.precision, "tol": 1e-10},
        "median_rel_error": float(np.median(rel)) if rel.size else None,
        "fd_voxels": int(len(vox)), "kink_hits": int(kink.sum()), "fd_step": 2.0 ** -10,
        "forward_ms_per_tick": t_fwd / ticks, "backward_ms": t_bwd, "recomputes": sess.recomputes,
        "adjoint_device_ms_last": float(adj_stats.device_ms), "loss": float(L.detach()), "fd_seconds": t_fd,
        "fp64_oracle_gradient_error": oracle_err,
        "fp64_oracle_island": "32x32x16 noise island, 8 ticks, checkpoint every 4 (the same loss)",
    }
    print(json.dumps(line), flush=True)
    eng.close()


def run_fracture(args):
    """Fracture run: one noise island (default 512x512x256, 55 % occupancy),
    --ticks tolerance ticks (pfsf_tick_tolerance: solve to 1e-6, history
    H = max(H, psi_e), phase field, failure scan, failure compaction) with the
    load ramped linearly 1x -> 2x, face conductivity = the kappa link value.
    Runs the mixed-precision batched solve and then the plain FP32 per-island
    solve on fresh state and compares final damage and failure codes."""
    os.environ.setdefault("PFSF_GRID_MIN_VOXELS", str(1 << 21))
    from pfsf_b200 import capi, synth

    dims = tuple(int(v) for v in args.dims.split(","))
    t0 = time.perf_counter()
    isl = synth.noise_island(dims, seed=51, occupancy=0.55)
    sig = synth.face_sigma_from_kappa(isl.dims, isl.vtype, isl.kappa)
    t_gen = time.perf_counter() - t0
    eng = capi.Engine(capi.default_config(max_island_size=1 << 30, tick_budget_ms=1 << 30, vram=180 << 30))
    if eng.init() != capi.PFSF_OK:
        raise RuntimeError("pfsf_init failed")
    n = isl.n
    rcomp = isl.rcomp.astype(np.float32)
    rtens = isl.rtens.astype(np.float32)
    maxphi = np.full(n, 1e9, np.float32)
    cap = 1 << 20
    runs = {}
    scale = None
    for name, mode, prec in (("mixed", capi.SOLVE_BATCHED, {"bf16": capi.PREC_BF16, "fp16": capi.PREC_FP16,
                                                              "fp32": capi.PREC_FP32}[args.precision]),
                             ("plain_fp32", capi.SOLVE_PER_ISLAND, capi.PREC_FP32)):
        if name == "plain_fp32" and args.no_plain:
            continue
        iid = len(runs) + 1
        assert eng.add_island(iid, isl.dims) == capi.PFSF_OK
        phi = np.zeros(n, np.float32)
        phik = np.zeros(n, np.float32)
        src = isl.source.copy()
        assert eng.register_buffers(iid, phi, src, sig, isl.vtype, rcomp, rtens, maxphi) == capi.PFSF_OK
        assert eng.register_kappa(iid, phik, src, isl.kappa, isl.vtype) == capi.PFSF_OK
        eng.set_solve_mode(mode)
        eng.set_precision(prec)
        eng.set_mg_cycle(capi.MG_V if args.cycle == "v" else capi.MG_W)
        if scale is None:  # loads scaled so max phi = 20 at 1x: the phase field and the scan act
            rc, st = eng.solve([iid], tol=1e-6, flags=capi.SOLVE_COLD_START)
            scale = 20.0 / float(np.abs(phik).max())
            phik[:] = 0.0
        base = (isl.source * np.float32(scale)).astype(np.float32)
        fb = np.zeros(1 + 4 * cap, np.int32)
        wall, dev, fails, iters, rel = [], [], [], [], 0.0
        for t in range(args.ticks):
            src[:] = base * np.float32(1.0 + t / max(args.ticks - 1, 1))
            eng.L.pfsf_mark_full_rebuild(eng.h, iid)  # the Java runtime marks islands dirty every tick
            t1 = time.perf_counter()
            rc, st = eng.tick_tolerance([iid], fb, tol=args.tol)
            wall.append((time.perf_counter() - t1) * 1000.0)
            if rc != capi.PFSF_OK or st.islands_converged != 1:
                raise RuntimeError(f"tick {t}: rc={rc} relres={st.max_rel_residual}")
            dev.append(st.device_ms)
            fails.append(int(fb[0]))
            iters.append(int(st.inner_iterations_total))
            rel = max(rel, st.max_rel_residual)
        runs[name] = {"D": eng.debug_field(iid, 2), "fail": eng.debug_field(iid, 3), "wall": wall, "dev": dev,
                      "fails": fails, "iters": iters, "relres": rel}
        if mode == capi.SOLVE_BATCHED:
            # one fine-level pass of the whole-GPU tier alone, on this island
            # (a working set far larger than L2): GB/s of its algorithmic bytes
            peak, peak_kind = peaks()
            for pname, pid in (("chebyshev_step", 0), ("matvec", 1)):
                rc, pms, pbytes = eng.time_pass(iid, pid, 20)
                if rc == capi.PFSF_OK and pms > 0:
                    runs[name].setdefault("passes", {})[pname] = {
                        "ms": pms, "bytes": pbytes, "gbs": pbytes / (pms * 1e-3) / 1e9,
                        "frac_of_hbm": pbytes / (pms * 1e-3) / 1e9 / peak, "peak": peak, "peak_kind": peak_kind}
        eng.L.pfsf_remove_island(eng.h, iid)
    m = runs["mixed"]
    line = {
        "metric": "config-5 fracture: ms per tolerance tick (solve to 1e-6 + history + phase field + failure scan)",
        "value": float(np.mean(m["wall"])), "unit": "ms/tick", "higher_is_better": False, "n_gpus": 1,
        "data": "synthetic", "dtype": "f32",
        "config": {"workload": f"one {args.dims.replace(',', 'x')} noise island (55 % occupancy, anchored "
                               f"component), {args.ticks} ticks, load ramped 1x->2x, warm start",
                   "grid_voxels": n, "active_voxels": int(isl.n_active), "precision": args.precision,
                   "tol": args.tol, "generation_s": t_gen,
                   "cycle": ("V" if args.cycle == "v" else "W") + "-cycle preconditioner (batched solve; the plain "
                            "per-island solve runs V-cycles)"},
        "solve_device_ms_mean": float(np.mean(m["dev"])), "inner_iterations_mean": float(np.mean(m["iters"])),
        "max_rel_residual_fp64": m["relres"], "failures_last_tick": m["fails"][-1],
        "failures_first_tick": m["fails"][0], "damage_max": float(m["D"].max()),
        "fine_passes": m.get("passes"),
    }
    if "plain_fp32" in runs:
        p = runs["plain_fp32"]
        line["plain_fp32_ms_per_tick"] = float(np.mean(p["wall"]))
        line["plain_fp32_solve_device_ms_mean"] = float(np.mean(p["dev"]))
        line["speedup_vs_plain_fp32"] = line["plain_fp32_ms_per_tick"] / line["value"]
        line["failure_code_agreement"] = float(np.mean(m["fail"] == p["fail"]))
        line["failure_code_mismatches"] = int(np.sum(m["fail"] != p["fail"]))
        dd = np.abs(m["D"] - p["D"])
        line["damage_max_abs_diff"] = float(dd.max())
        # psi_e switches by 100x where flux_in crosses 3 flux_out (rbgs_smooth.comp.glsl:186):
        # voxels on that switch can differ between two solves that agree to 1e-6
        line["damage_voxels_differing_1e-3"] = int(np.sum(dd > 1e-3))
        line["damage_voxels"] = int(np.sum((m["D"] > 0) | (p["D"] > 0)))
    print(json.dumps(line), flush=True)
    eng.close()


def run_tick_dbb(args):
    """The drop-in reference tick (pfsf_tick_dbb: the fixed 16-step adaptive
    RBGS / PCG / V-cycle schedule, phase field, failure scan, failure
    compaction, stress readback) over the batch workload's islands, every
    island dirty every tick as the Java runtime marks them
    (NativePFSFRuntime.java:289), so every tick also uploads every island's
    arrays from the caller's pinned host buffers.  Face conductivity = the
    kappa link value; loads x 1e-4 so phi stays in the range the reference
    clamps to (phi <= 1e7).  value = device time of a tick (CUDA events on
    the engine stream, upload included); e2e = wall time of the call."""
    from pfsf_b200 import capi
    isls, meta = make_workload(args, 0)
    t0 = time.perf_counter()
    host = []
    for isl in isls:
        host.append({"phi": np.zeros(isl.n, np.float32), "source": (isl.source * np.float32(1e-4)).astype(np.float32),
                     "cond": synth_face_sigma(isl), "type": isl.vtype, "rcomp": isl.rcomp.astype(np.float32),
                     "rtens": isl.rtens.astype(np.float32), "max_phi": np.full(isl.n, 1e9, np.float32)})
    t_gen = time.perf_counter() - t0
    import torch
    eng = capi.Engine(capi.default_config(max_island_size=1 << 28, tick_budget_ms=1 << 30, vram=180 << 30))
    if eng.init() != capi.PFSF_OK:
        raise RuntimeError("pfsf_init failed")
    eng.set_amg(args.amg)
    ids = []
    for k, (isl, h) in enumerate(zip(isls, host)):
        iid = k + 1
        assert eng.add_island(iid, isl.dims, (0, 0, 128 * k)) == capi.PFSF_OK
        assert eng.register_buffers(iid, h["phi"], h["source"], h["cond"], h["type"], h["rcomp"], h["rtens"],
                                    h["max_phi"]) == capi.PFSF_OK
        assert eng.register_stress(iid, h["phi"]) == capi.PFSF_OK
        ids.append(iid)
    cap = 1024  # the Java runtime's failure buffer: 4 + 1024 x 16 bytes (NativePFSFRuntime.java:251-252)
    fb = np.zeros(1 + 4 * cap, np.int32)

    def tick():
        for iid in ids:
            eng.L.pfsf_mark_full_rebuild(eng.h, iid)
        rc = eng.tick_dbb(ids, fb)
        if rc != capi.PFSF_OK:
            raise RuntimeError(f"pfsf_tick_dbb rc={rc}")
        rc, rep = eng.tick_report()
        return rep

    for _ in range(max(args.warmup, 1)):
        tick()
    reps, walls = [], []
    with Clocks(0) as clk:
        for _ in range(args.steps):
            t1 = time.perf_counter()
            reps.append(tick())
            walls.append((time.perf_counter() - t1) * 1000.0)
    dev_ms = float(np.mean([r.device_ms for r in reps]))
    bytes_ = float(np.mean([r.algorithmic_bytes for r in reps]))
    peak, peak_kind = peaks()
    h2d = sum(isl.n * (4 + 4 + 24 + 1 + 4 + 4 + 4) for isl in isls)
    d2h = sum(isl.n * 4 for isl in isls) + 4 + 16 * int(fb[0])
    line = {
        "metric": "drop-in reference tick (pfsf_tick_dbb) ms/tick", "value": dev_ms, "unit": "ms/tick",
        "higher_is_better": False, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_ms,
        "data": "synthetic", "dtype": "f32",
        "config": {"workload": (f"{len(isls)} islands (log-uniform sides, scale {meta['scale']:.3f}), "
                                f"{meta['grid_total']} grid / {meta['active_total']} active voxels, all dirty every "
                                f"tick, 16-step reference schedule"
                                + (", aggregation correction at every PCG start" if args.amg else "")),
                   "islands": len(isls),
                   "grid_voxels": meta["grid_total"], "active_voxels": meta["active_total"],
                   "generation_s": t_gen},
        "e2e": {"value": float(np.mean(walls)), "unit": "ms/tick", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h)},
        "roofline": {"bound": "hbm", "achieved": bytes_ / (dev_ms * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": bytes_ / (dev_ms * 1e-3) / 1e9 / peak, "traffic": None, "peak_kind": peak_kind,
                     "algorithmic_bytes": bytes_, "kernel": "the tick's graph (dominant: kb_rbgs_color)",
                     "note": ("model bytes of every pass (pfsf_last_tick_report) over the tick's stream time, "
                              "which includes the zero-copy upload of every island's arrays over the host link")},
        "voxel_updates_per_s": 16.0 * meta["grid_total"] / (dev_ms * 1e-3),
        "gpu_launches": int(np.mean([r.kernel_launches for r in reps])),
        "groups": int(reps[-1].groups), "graph_replayed": int(reps[-1].graph_replayed),
        "host_ms_per_tick": float(np.mean([r.host_us for r in reps])) * 1e-3,
        "host_ms_by_graph_use": {k: (float(np.mean([r.host_us for r in reps if r.graph_replayed == v])) * 1e-3
                                     if any(r.graph_replayed == v for r in reps) else None)
                                 for k, v in (("replayed", 1), ("updated", 2), ("instantiated", 0))},
        "graph_use": {"replayed": sum(r.graph_replayed == 1 for r in reps),
                      "updated": sum(r.graph_replayed == 2 for r in reps),
                      "instantiated": sum(r.graph_replayed == 0 for r in reps)},
        "failures_last_tick": int(fb[0]), "clocks": clk.summary(),
        "macro_residual_max": float(max(eng.debug_field(i, 5)["last_macro"] for i in ids)),
    }
    print(json.dumps(line), flush=True)
    eng.close()


def synth_face_sigma(isl):
    from pfsf_b200 import synth
    return synth.face_sigma_from_kappa(isl.dims, isl.vtype, isl.kappa)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "adjoint":
        run_adjoint(args)
    elif args.workload == "fracture":
        run_fracture(args)
    elif args.workload == "tick_dbb":
        run_tick_dbb(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
