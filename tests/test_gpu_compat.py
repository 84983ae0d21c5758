"""GPU parity of the reference-schedule tick (pfsf_tick_dbb) against the CPU oracle.

Every case drives libpfsf.so through its C ABI exactly as the Java bridge
does (pfsf_create -> pfsf_init -> pfsf_add_island ->
pfsf_register_island_buffers -> pfsf_register_stress_readback aliased to the
phi buffer -> pfsf_tick_dbb with a failure buffer) and compares with the
oracle island after every tick.

Tolerances (FP32 path): phi agrees within 1e-5 of max|phi| per tick; the
failure DBB (count and every {x,y,z,type} tuple) is bit-exact; H and the
damage field agree within 1e-5 relative to their maxima.
"""
import numpy as np
import pytest

import cases
import oracle as O
from pfsf_b200 import capi

pytestmark = pytest.mark.gpu

PHI_TOL = 1e-5


@pytest.fixture(scope="module")
def eng(lib_built):
    cfg = capi.default_config(max_island_size=1 << 26, tick_budget_ms=1 << 30)
    e = capi.Engine(cfg)
    assert e.init() == capi.PFSF_OK, "CUDA device required"
    yield e
    e.close()


_next_id = [100]


def _setup(eng, case, origin=(3, -2, 7)):
    iid = _next_id[0]
    _next_id[0] += 1
    assert eng.add_island(iid, case["dims"], origin) == capi.PFSF_OK
    host = {k: np.ascontiguousarray(case[k]).copy() for k in
            ("phi", "source", "conductivity", "type", "rcomp", "rtens", "max_phi")}
    assert eng.register_buffers(iid, host["phi"], host["source"], host["conductivity"], host["type"],
                                host["rcomp"], host["rtens"], host["max_phi"]) == capi.PFSF_OK
    assert eng.register_stress(iid, host["phi"]) == capi.PFSF_OK  # warm start, as the Java runtime does
    ref = O.Island(*case["dims"])
    ref.load(phi=case["phi"], source=case["source"], conductivity=case["conductivity"], type=case["type"],
             rcomp=case["rcomp"], rtens=case["rtens"], max_phi=case["max_phi"], hydration=case["hydration"])
    return iid, host, ref


def _tick_both(eng, iid, host, ref, origin, cap=4096):
    fb = np.zeros(1 + 4 * cap, np.int32)
    fb[0] = 77  # pre-zeroed by pfsf_tick_dbb
    assert eng.tick_dbb([iid], fb) == capi.PFSF_OK
    ref.tick()
    want = ref.failures(origin, capacity=cap)
    return fb, want


def _assert_tick_parity(eng, iid, host, ref, fb, want, t):
    assert fb[0] == want[0], f"tick {t}: failure count {fb[0]} vs {want[0]}"
    assert np.array_equal(fb[: 1 + 4 * fb[0]], want[: 1 + 4 * want[0]]), f"tick {t}: failure tuples"
    _assert_island_state(eng, iid, host, ref, t)


def _assert_island_state(eng, iid, host, ref, t):
    phi_ref = ref.view("phi")
    scale = max(float(np.abs(phi_ref).max()), 1e-30)
    err = float(np.abs(host["phi"].astype(np.float64) - phi_ref).max()) / scale
    assert err <= PHI_TOL, f"tick {t}: phi rel err {err:.3e}"
    assert np.array_equal(eng.debug_field(iid, 3), ref.view("fail").astype(np.uint8)), f"tick {t}: fail flags"
    # the island's phi maximum, reduced in the failure pass
    rc, pm = eng.phi_max(iid)
    assert rc == capi.PFSF_OK and pm == float(eng.debug_field(iid, 0).max()), f"tick {t}: phi max"
    for field, name in ((1, "H"), (2, "D")):
        g = eng.debug_field(iid, field)
        r = ref.view(name)
        sc = max(float(np.abs(r).max()), 1e-30)
        assert float(np.abs(g - r).max()) / sc <= PHI_TOL, f"tick {t}: {name}"
    st = eng.debug_field(iid, 5)
    rs = ref.state()
    assert st["chebyshev_iter"] == rs["chebyshev_iter"]
    assert st["pcg_allocated"] == rs["pcg_allocated"]
    assert st["mg_allocated"] == rs["mg_allocated"]


@pytest.mark.parametrize("name,ticks", [("block8", 4), ("noise20", 4), ("slab", 3), ("rod", 3), ("tiny", 3)])
def test_tick_parity(eng, name, ticks):
    case = cases.compat_case(name)
    origin = (3, -2, 7)
    iid, host, ref = _setup(eng, case, origin)
    for t in range(ticks):
        eng.L.pfsf_mark_full_rebuild(eng.h, iid)
        fb, want = _tick_both(eng, iid, host, ref, origin)
        _assert_tick_parity(eng, iid, host, ref, fb, want, t)


def test_pcg_tail_engages_and_matches(eng):
    """Run until the stall ratio switches the schedule to RBGS(2) + PCG(14)
    (dispatcher.cpp:123-167) and keep comparing."""
    case = cases.compat_case("block16")
    origin = (0, 0, 0)
    iid, host, ref = _setup(eng, case, origin)
    saw_pcg = False
    for t in range(8):
        eng.L.pfsf_mark_full_rebuild(eng.h, iid)
        fb, want = _tick_both(eng, iid, host, ref, origin)
        _assert_tick_parity(eng, iid, host, ref, fb, want, t)
        saw_pcg |= ref.state()["pcg_allocated"] == 1
    assert saw_pcg


def test_isolated_voxel_no_support_gpu(eng):
    case, centre = cases.isolated_voxel_case()
    iid, host, ref = _setup(eng, case, (0, 0, 0))
    fb, want = _tick_both(eng, iid, host, ref, (0, 0, 0))
    assert host["phi"][centre] == 0.0
    assert fb[0] == 1 and fb[4] == 3


def test_source_free_gpu(eng):
    case = cases.compat_case("noise20")
    case["source"][:] = 0.0
    iid, host, ref = _setup(eng, case)
    for _ in range(2):
        eng.L.pfsf_mark_full_rebuild(eng.h, iid)
        eng.tick_dbb([iid])
    assert np.all(host["phi"] == 0.0)


def test_failure_buffer_saturation(eng):
    """More failures than tuples: count saturates at capacity, tuples in voxel order."""
    case = cases.compat_case("noise20")
    case["rcomp"][:] = 1e-9
    case["rtens"][:] = 1e-9
    origin = (1, 2, 3)
    iid, host, ref = _setup(eng, case, origin)
    fb, want = _tick_both(eng, iid, host, ref, origin, cap=5)
    assert fb[0] == 5
    assert np.array_equal(fb, want)


def test_multi_island_tick_order(eng):
    """Two dirty islands in one tick: failures appended island by island."""
    c1 = cases.compat_case("block8")
    c2 = cases.compat_case("tiny")
    c1["rcomp"][:] = 1e-9
    c2["rcomp"][:] = 1e-9
    o1, o2 = (0, 0, 0), (100, 0, 0)
    i1, h1, r1 = _setup(eng, c1, o1)
    i2, h2, r2 = _setup(eng, c2, o2)
    cap = 4096
    fb = np.zeros(1 + 4 * cap, np.int32)
    assert eng.tick_dbb([i1, i2], fb) == capi.PFSF_OK
    r1.tick()
    r2.tick()
    want = np.zeros(1 + 4 * cap, np.int32)
    r1.failures(o1, capacity=cap, dbb=want)
    r2.failures(o2, capacity=cap, dbb=want)
    assert fb[0] == want[0] and fb[0] > 0
    assert np.array_equal(fb[: 1 + 4 * fb[0]], want[: 1 + 4 * want[0]])


def test_batched_tick_many_islands(eng):
    """Two dozen islands of different shapes and schedules (plain RBGS, PCG
    after a stall, V-cycles every 4 / 2 / 1 steps, none) in one
    pfsf_tick_dbb call per tick: every island matches its own oracle island
    each tick, the failure buffer holds the islands' tuples in call order,
    and the kernel launches of a tick do not grow with the island count (one
    launch per schedule step and island group, replayed from a CUDA graph)."""
    names = ["block8", "noise20", "slab", "rod", "tiny", "block16"]
    isl = []
    for k in range(24):
        c = cases.compat_case(names[k % len(names)])
        if k % 4 == 1:
            c["rcomp"][::5] = 1e-9
        origin = (40 * k, -3 * k, k)
        iid, host, ref = _setup(eng, c, origin)
        isl.append((iid, host, ref, origin))
    ids = [x[0] for x in isl]
    cap = 1 << 15
    per_tick = []
    for t in range(5):
        for iid in ids:
            eng.L.pfsf_mark_full_rebuild(eng.h, iid)
        fb = np.zeros(1 + 4 * cap, np.int32)
        l0 = eng.launches()
        assert eng.tick_dbb(ids, fb) == capi.PFSF_OK
        rc, rep = eng.tick_report()
        assert rc == capi.PFSF_OK and rep.islands == len(ids) and rep.kernel_launches == eng.launches() - l0
        per_tick.append((rep.groups, rep.kernel_launches, rep.graph_replayed))
        want = np.zeros(1 + 4 * cap, np.int32)
        for iid, host, ref, origin in isl:
            ref.tick()
            ref.failures(origin, capacity=cap, dbb=want)
        assert fb[0] == want[0] and fb[0] > 0, (t, fb[0], want[0])
        assert np.array_equal(fb[: 1 + 4 * fb[0]], want[: 1 + 4 * want[0]]), f"tick {t}: failure tuples"
        for iid, host, ref, origin in isl:
            _assert_island_state(eng, iid, host, ref, t)
    # one launch per schedule step and GROUP: at most one group per distinct
    # (shape, schedule) here, and a schedule is at most ~700 launches (the
    # aspect-8 rod: a V-cycle every step, twice); one island at a time the
    # 24 islands would take at least 24 x 16 x 8 RBGS colour launches
    for groups, launches, _ in per_tick:
        assert groups <= 12 and launches <= 700 * groups and launches < 24 * 16 * 8, per_tick
    # the structure repeats between some consecutive ticks: replayed graph
    assert any(r for _, _, r in per_tick[1:]), per_tick


def test_reference_fixtures_parity(eng):
    """The reference's own fixture shapes (inputs only), one tick each."""
    import glob
    import os
    fx = os.path.join(os.path.dirname(__file__), "golden", "fixtures_compat.npz")
    data = np.load(fx, allow_pickle=False)
    names = sorted({k.split("__")[0] for k in data.files})
    assert len(names) >= 10
    for nm in names:
        case = {k.split("__")[1]: data[k] for k in data.files if k.startswith(nm + "__")}
        case["dims"] = tuple(int(v) for v in case["dims"])
        iid, host, ref = _setup(eng, case, (0, 0, 0))
        for t in range(2):
            eng.L.pfsf_mark_full_rebuild(eng.h, iid)
            fb, want = _tick_both(eng, iid, host, ref, (0, 0, 0))
            _assert_tick_parity(eng, iid, host, ref, fb, want, t)


def test_not_dirty_island_is_skipped(eng):
    case = cases.compat_case("block8")
    iid, host, ref = _setup(eng, case)
    assert eng.tick_dbb([iid]) == capi.PFSF_OK  # first tick (dirty after registration)
    before = host["phi"].copy()
    fb = np.zeros(1 + 4 * 16, np.int32)
    fb[0] = 9
    assert eng.tick_dbb([iid], fb) == capi.PFSF_OK  # clean: nothing dispatched
    assert fb[0] == 0
    assert np.array_equal(before, host["phi"])


def test_sparse_scatter_updates_device_arrays(eng):
    """48-byte records (SH/sparse_scatter.comp.glsl:47-66: flat index, source,
    type, maxPhi, rcomp, rtens, six face conductivities in SoA order) land in
    the device arrays; out-of-island indices are skipped; the island is marked
    dirty and the next tick -- which, as in the reference, re-uploads the
    caller's arrays, kept in step with the edits -- matches the oracle run on
    the edited inputs."""
    import ctypes as C
    case = cases.compat_case("noise20")
    origin = (3, -2, 7)
    iid, host, ref = _setup(eng, case, origin)
    fb, want = _tick_both(eng, iid, host, ref, origin)
    _assert_tick_parity(eng, iid, host, ref, fb, want, 0)
    n = int(np.prod(case["dims"]))
    addr = C.c_void_p()
    nbytes = C.c_int64()
    assert eng.L.pfsf_get_sparse_upload_buffer(eng.h, iid, C.byref(addr), C.byref(nbytes)) == capi.PFSF_OK
    assert nbytes.value == 512 * 48
    rec = np.frombuffer((C.c_byte * nbytes.value).from_address(addr.value), dtype=np.uint32).reshape(512, 12)
    rng = np.random.default_rng(21)
    idx = rng.choice(n, 40, replace=False)
    src = rng.uniform(0.0, 3.0, idx.size).astype(np.float32)
    vt = rng.integers(0, 3, idx.size).astype(np.uint32)
    mphi = rng.uniform(5.0, 50.0, idx.size).astype(np.float32)
    rc_ = rng.uniform(0.5, 40.0, idx.size).astype(np.float32)
    rt_ = rng.uniform(0.1, 5.0, idx.size).astype(np.float32)
    cond = rng.uniform(0.0, 1.0, (idx.size, 6)).astype(np.float32)
    cond[vt == 0] = 0.0
    rec[:] = 0
    rec[: idx.size, 0] = idx
    rec[: idx.size, 1] = src.view(np.uint32)
    rec[: idx.size, 2] = vt
    rec[: idx.size, 3] = mphi.view(np.uint32)
    rec[: idx.size, 4] = rc_.view(np.uint32)
    rec[: idx.size, 5] = rt_.view(np.uint32)
    rec[: idx.size, 6:] = cond.view(np.uint32)
    # two records outside the island: skipped
    rec[idx.size: idx.size + 2, 0] = [n, n + 1000]
    rec[idx.size: idx.size + 2, 1:] = np.float32(123.0).view(np.uint32)
    # the Java side keeps its zero-copy arrays in step with the edits it scatters
    host["source"][idx] = src
    host["type"][idx] = vt.astype(np.uint8)
    host["max_phi"][idx] = mphi
    host["rcomp"][idx] = rc_
    host["rtens"][idx] = rt_
    cv = host["conductivity"].reshape(-1)
    for d in range(6):
        cv[d * n + idx] = cond[:, d]
    assert eng.L.pfsf_notify_sparse_updates(eng.h, iid, idx.size + 2) == capi.PFSF_OK
    assert eng.L.pfsf_notify_sparse_updates(eng.h, iid, 0) == capi.PFSF_OK
    for field, name, dt in ((6, "source", np.float32), (7, "conductivity", np.float32), (8, "type", np.uint8),
                            (9, "max_phi", np.float32), (10, "rcomp", np.float32), (11, "rtens", np.float32)):
        dev = eng.debug_field(iid, field)
        want_arr = np.ascontiguousarray(host[name]).reshape(-1).astype(dt)
        assert np.array_equal(dev.view(np.uint8), want_arr.view(np.uint8)), f"device {name} after scatter"
    # the edit marked the island dirty: the next tick runs on the edited inputs
    ref.load(source=host["source"], conductivity=host["conductivity"], type=host["type"], rcomp=host["rcomp"],
             rtens=host["rtens"], max_phi=host["max_phi"])
    for t in range(1, 3):
        fb, want = _tick_both(eng, iid, host, ref, origin)
        _assert_tick_parity(eng, iid, host, ref, fb, want, t)
        eng.L.pfsf_mark_full_rebuild(eng.h, iid)


def test_amg_correction_matches_oracle(eng):
    """pfsf_set_amg: every PCG start applies the aggregation correction
    (NP/src/solver/dispatcher_amg.cpp:83-161 with the aggregates of
    amg_builder.cpp:9-63).  Two islands ticked together in one batched tick
    until PCG engages; after every tick the state agrees with oracle islands
    that run the same correction, and the device-built aggregates, weights
    and coarse diagonal equal the oracle builder's bit for bit (the oracle
    builder is itself bit-exact against the reference's, test_amg_oracle.py)."""
    eng.set_amg(True)
    try:
        origins = [(0, 0, 0), (40, 1, -3)]
        setups = []
        for name, origin in zip(("block16", "noise20"), origins):
            case = cases.compat_case(name)
            iid, host, _ = _setup(eng, case, origin)
            ref = O.Island(*case["dims"], amg=True)
            ref.load(phi=case["phi"], source=case["source"], conductivity=case["conductivity"], type=case["type"],
                     rcomp=case["rcomp"], rtens=case["rtens"], max_phi=case["max_phi"],
                     hydration=case["hydration"])
            setups.append((iid, host, ref, case))
        built = False
        for t in range(8):
            for iid, _, _, _ in setups:
                eng.L.pfsf_mark_full_rebuild(eng.h, iid)
            fb = np.zeros(1 + 4 * 8192, np.int32)
            assert eng.tick_dbb([s[0] for s in setups], fb) == capi.PFSF_OK
            want_count = 0
            for (iid, host, ref, case), origin in zip(setups, origins):
                ref.tick()
                want_count += int(ref.failures(origin, capacity=8192)[0])
                _assert_island_state(eng, iid, host, ref, t)
                if ref.state()["pcg_allocated"] == 1:
                    agg, w, dc = O.amg_build(case["dims"], case["conductivity"], case["type"])
                    g_agg = eng.debug_field(iid, 12)
                    if g_agg.size:
                        built = True
                        assert np.array_equal(g_agg, agg), f"tick {t}: aggregates"
                        assert np.array_equal(eng.debug_field(iid, 13).view(np.uint32), w.view(np.uint32))
                        assert np.array_equal(eng.debug_field(iid, 14).view(np.uint32), dc.view(np.uint32))
            assert fb[0] == want_count, f"tick {t}: failure count"
        assert built, "PCG (and with it the correction) never engaged"
    finally:
        eng.set_amg(False)
