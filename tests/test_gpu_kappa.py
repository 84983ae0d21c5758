"""GPU tolerance solve of the symmetric harmonic-mean operator vs the FP64 oracle.

Bar: every island reports convergence, and the FP64 oracle evaluates the
relative residual ||s - A x||_2 / ||s||_2 of the returned FP64 accumulator at
<= 1e-6 (the target); the FP64 accumulator agrees with the oracle's own
solve (tol 1e-12) to <= 1e-4 relative (inf-norm), which is what a 1e-6
residual allows for condition numbers ~L^2.  The FP32 phi written back is
that accumulator rounded.
"""
import os

import numpy as np
import pytest

import oracle as O
from pfsf_b200 import capi, synth

pytestmark = pytest.mark.gpu

TOL = 1e-6


@pytest.fixture(scope="module")
def eng(lib_built):
    cfg = capi.default_config(max_island_size=1 << 26, tick_budget_ms=1 << 30)
    e = capi.Engine(cfg)
    assert e.init() == capi.PFSF_OK, "CUDA device required"
    yield e
    e.close()


_ids = [5000]


def _register(eng, isl):
    iid = _ids[0]
    _ids[0] += 1
    assert eng.add_island(iid, isl.dims) == capi.PFSF_OK
    host = {"phi": np.zeros(isl.n, np.float32), "source": isl.source.copy(), "kappa": isl.kappa.copy(),
            "type": isl.vtype.copy()}
    assert eng.register_kappa(iid, host["phi"], host["source"], host["kappa"], host["type"]) == capi.PFSF_OK
    return iid, host


def _check(eng, isl, iid, host):
    rc, x64 = eng.read_solution64(iid, isl.n)
    assert rc == capi.PFSF_OK and x64.size == isl.n
    k = isl.kappa.astype(np.float64)
    s = isl.source.astype(np.float64)
    y = O.kappa_apply(isl.dims, k, isl.vtype, x64)
    solid = isl.vtype == 1
    rel = np.linalg.norm((s - y)[solid]) / np.linalg.norm(s[solid])
    assert rel <= TOL, f"FP64-evaluated relres {rel:.3e}"
    xr, _, rr = O.kappa_solve64(isl.dims, k, isl.vtype, s, tol=1e-12)
    err = np.abs(x64 - xr).max() / np.abs(xr).max()
    assert err <= 1e-4, f"error vs FP64 oracle {err:.3e}"
    np.testing.assert_array_equal(host["phi"], x64.astype(np.float32))
    return rel, err


@pytest.mark.parametrize("mode,prec", [(capi.SOLVE_PER_ISLAND, capi.PREC_FP32), (capi.SOLVE_BATCHED, capi.PREC_FP32),
                                       (capi.SOLVE_BATCHED, capi.PREC_BF16), (capi.SOLVE_BATCHED, capi.PREC_FP16)])
def test_single_islands(eng, mode, prec):
    eng.set_solve_mode(mode)
    eng.set_precision(prec)
    for isl in (synth.solid_block((16, 16, 16), seed=2), synth.noise_island((24, 20, 16), seed=4)):
        iid, host = _register(eng, isl)
        rc, st = eng.solve([iid], tol=TOL)
        assert rc == capi.PFSF_OK
        assert st.islands_converged == 1, (st.max_rel_residual, st.max_iterations)
        _check(eng, isl, iid, host)


def test_batched_uneven_islands(eng):
    eng.set_solve_mode(capi.SOLVE_BATCHED)
    eng.set_precision(capi.PREC_BF16)
    dims = synth.batch_dims(24, seed=3, lo=3, hi=28)
    isls = [synth.noise_island(tuple(int(v) for v in d), seed=100 + k) for k, d in enumerate(dims)]
    isls = [i for i in isls if i.n_active > 0]
    reg = [_register(eng, isl) for isl in isls]
    rc, st = eng.solve([r[0] for r in reg], tol=TOL)
    assert rc == capi.PFSF_OK
    assert st.islands_converged == len(isls)
    assert st.max_rel_residual <= TOL
    inner = 0
    for isl, (iid, host) in zip(isls, reg):
        _check(eng, isl, iid, host)
        rc, r = eng.island_report(iid)
        assert rc == capi.PFSF_OK
        assert (r.lx, r.ly, r.lz) == isl.dims and r.converged == 1 and r.rel_residual <= TOL
        assert capi.IslandReport.TEAMS[r.team] in ("cta", "warp", "cluster") and r.solve_ms > 0
        assert r.setup_ms + r.precond_ms <= r.solve_ms
        inner += r.inner_iterations
    assert inner == st.inner_iterations_total
    rc, _ = eng.island_report(987654)
    assert rc == capi.PFSF_ERROR_INVALID_ARG


@pytest.mark.parametrize("cluster", ["8", "4", "1"])
def test_tile_shapes_and_teams(lib_built, cluster):
    """Every team that marches plane tiles (one CTA, 8- and 4-CTA clusters,
    the whole GPU) on islands whose sides need several tiles: x wider than
    one 126-column tile, y split into bands, odd depths and odd widths (an
    aggregate of the next level cut by the island edge)."""
    env = {"PFSF_CLUSTER_MIN_VOXELS": "20000", "PFSF_GRID_MIN_VOXELS": "60000", "PFSF_CLUSTER": cluster}
    old = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        e = capi.Engine(capi.default_config(max_island_size=1 << 26, tick_budget_ms=1 << 30))
        assert e.init() == capi.PFSF_OK
    finally:
        for k, v in old.items():
            if v is None:
                del os.environ[k]
            else:
                os.environ[k] = v
    try:
        e.set_solve_mode(capi.SOLVE_BATCHED)
        e.set_precision(capi.PREC_BF16)
        dims = [(131, 9, 5), (127, 40, 7), (7, 300, 6), (33, 31, 17), (141, 23, 21), (9, 11, 13), (250, 30, 9)]
        isls = [synth.noise_island(d, seed=40 + k) for k, d in enumerate(dims)]
        isls = [i for i in isls if i.n_active > 0]
        reg = [_register(e, isl) for isl in isls]
        rc, st = e.solve([r[0] for r in reg], tol=TOL)
        assert rc == capi.PFSF_OK
        assert st.islands_converged == len(isls), st.max_rel_residual
        teams = set()
        for isl, (iid, host) in zip(isls, reg):
            _check(e, isl, iid, host)
            rc, r = e.island_report(iid)
            teams.add(capi.IslandReport.TEAMS[r.team])
        assert "grid" in teams and "cta" in teams and ("cluster" in teams or cluster == "1")
    finally:
        e.close()


def test_warm_start_resolve_is_immediate(eng):
    eng.set_solve_mode(capi.SOLVE_BATCHED)
    eng.set_precision(capi.PREC_BF16)
    isl = synth.noise_island((20, 20, 12), seed=9)
    iid, host = _register(eng, isl)
    rc, st = eng.solve([iid], tol=1e-4)
    assert st.islands_converged == 1
    # solving again from the written-back phi reaches 1e-4 with no inner iteration
    rc, st2 = eng.solve([iid], tol=1e-4)
    assert st2.islands_converged == 1


def test_wcycle_converges_and_matches_oracle(lib_built):
    """The W-cycle preconditioner (levels below the first coarse level visited
    twice) solves to the tolerance, agrees with the FP64 oracle, and needs no
    more inner iterations than the V-cycle on the same island."""
    e = capi.Engine(capi.default_config(max_island_size=1 << 26, tick_budget_ms=1 << 30))
    assert e.init() == capi.PFSF_OK
    isl = synth.noise_island((64, 48, 32), seed=77)
    phi = np.zeros(isl.n, np.float32)
    assert e.add_island(1, isl.dims) == capi.PFSF_OK
    assert e.register_kappa(1, phi, isl.source, isl.kappa, isl.vtype) == capi.PFSF_OK
    e.set_solve_mode(capi.SOLVE_BATCHED)
    e.set_precision(capi.PREC_BF16)
    xr, _, _ = O.kappa_mgpcg64(isl.dims, isl.kappa.astype(np.float64), isl.vtype, isl.source.astype(np.float64),
                               tol=1e-12, threads=os.cpu_count() or 1)
    iters = {}
    for cyc in (capi.MG_V, capi.MG_W):
        e.set_mg_cycle(cyc)
        rc, st = e.solve([1], tol=1e-6, flags=capi.SOLVE_COLD_START)
        assert rc == capi.PFSF_OK and st.islands_converged == 1 and st.max_rel_residual <= 1e-6
        rc, x64 = e.read_solution64(1, isl.n)
        assert np.abs(x64 - xr).max() <= 1e-4 * np.abs(xr).max()
        iters[cyc] = st.inner_iterations_total
    assert iters[capi.MG_W] <= iters[capi.MG_V], iters
    e.close()


def test_tail_threshold_changes_no_result(lib_built):
    """The coarse-level size from which one warp runs the rest of the V-cycle
    (tail_cells, a tuned launch shape) moves work between the team and its
    leader warp without changing any arithmetic: every threshold gives the
    same iterations and the same solution, bit for bit, on islands solved by
    CTAs and by a cluster."""
    e = capi.Engine(capi.default_config(max_island_size=1 << 26, tick_budget_ms=1 << 30))
    assert e.init() == capi.PFSF_OK
    isls = [synth.noise_island((40, 36, 28), seed=81), synth.noise_island((72, 64, 40), seed=82),
            synth.solid_block((20, 18, 16), seed=83)]
    keep = []
    for k, isl in enumerate(isls):
        phi = np.zeros(isl.n, np.float32)
        keep.append(phi)
        assert e.add_island(k + 1, isl.dims) == capi.PFSF_OK
        assert e.register_kappa(k + 1, phi, isl.source, isl.kappa, isl.vtype) == capi.PFSF_OK
    ids = [1, 2, 3]
    e.set_solve_mode(capi.SOLVE_BATCHED)
    e.set_precision(capi.PREC_BF16)
    assert e.set_tuning(cluster=4, cluster_min_voxels=150000) == capi.PFSF_OK  # island 2 on a cluster
    ref = None
    for tail in (512, 0, 64, 4096):
        assert e.set_tuning(tail_cells=tail) == capi.PFSF_OK
        rc, st = e.solve(ids, tol=1e-6, flags=capi.SOLVE_COLD_START)
        assert rc == capi.PFSF_OK and st.islands_converged == 3
        xs = [e.read_solution64(i, isls[i - 1].n)[1].copy() for i in ids]
        got = (st.inner_iterations_total, xs)
        if ref is None:
            ref = got
            continue
        assert got[0] == ref[0], (tail, got[0], ref[0])
        for a, b in zip(got[1], ref[1]):
            assert np.array_equal(a.view(np.uint64), b.view(np.uint64)), tail
    e.close()


def test_mapped_and_copied_islands_in_one_solve(lib_built):
    """One batched solve over an island whose arrays the engine maps into the
    device address space (the teams read its inputs and write its phi inside
    the persistent launch) and one whose arrays were page-locked by another
    allocator (torch pinned memory: the engine cannot map them and copies
    them instead).  Both islands converge and each caller phi array holds
    the FP32 rounding of the island's FP64 solution, bit for bit."""
    torch = pytest.importorskip("torch")
    e = capi.Engine(capi.default_config(max_island_size=1 << 26, tick_budget_ms=1 << 30))
    assert e.init() == capi.PFSF_OK
    e.set_solve_mode(capi.SOLVE_BATCHED)
    e.set_precision(capi.PREC_BF16)
    isls = [synth.noise_island((40, 36, 28), seed=91), synth.noise_island((30, 28, 20), seed=92)]

    def pinned(a):
        t = torch.empty(a.size, dtype={np.float32: torch.float32, np.uint8: torch.uint8}[a.dtype.type],
                        pin_memory=True)
        v = t.numpy()
        v[:] = a.reshape(-1)
        return t, v

    keep, phis = [], []
    for k, isl in enumerate(isls):
        assert e.add_island(k + 1, isl.dims) == capi.PFSF_OK
        if k == 0:
            arrs = [np.zeros(isl.n, np.float32), isl.source.copy(), isl.kappa.copy(), isl.vtype.copy()]
        else:
            ts = [pinned(np.zeros(isl.n, np.float32)), pinned(isl.source), pinned(isl.kappa), pinned(isl.vtype)]
            keep.append(ts)
            arrs = [v for _, v in ts]
        keep.append(arrs)
        phis.append(arrs[0])
        assert e.register_kappa(k + 1, *arrs) == capi.PFSF_OK
    for rep in range(2):  # the second solve replays the captured launch
        for p in phis:
            p[:] = 0.0
        rc, st = e.solve([1, 2], tol=1e-6, flags=capi.SOLVE_COLD_START)
        assert rc == capi.PFSF_OK and st.islands_converged == 2 and st.max_rel_residual <= 1e-6
        for k, isl in enumerate(isls):
            rc, x64 = e.read_solution64(k + 1, isl.n)
            assert rc == capi.PFSF_OK
            assert np.array_equal(phis[k].view(np.uint32), x64.astype(np.float32).view(np.uint32)), (rep, k)
            assert np.abs(phis[k]).max() > 0.0
    e.close()
