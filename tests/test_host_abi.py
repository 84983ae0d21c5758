"""Host-side frozen ABI: exports, known answers, and bit-exact A/B.

CPU only.  Three layers:
  * the library loads without a GPU and exports every function that
    include/pfsf/*.h declares;
  * known answers restated from the reference's Java/native golden-parity
    suite (Block Reality/api/src/test/java/com/blockreality/api/physics/pfsf/
    GoldenParityTest.java, line numbers per test);
  * bit-exact A/B against the reference's own CPU primitives compiled from
    their sources (oracle/ref.mk -> oracle/_ref/libpfsf_ref.so) on seeded
    random inputs; skipped when that library has not been built.
"""
import glob
import os
import re
import struct

import numpy as np
import pytest

from pfsf_b200 import capi
from pfsf_b200 import host as H

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libpfsf_ref.so")

# PFSFConstants.java:63, :142, :331
DIVERGENCE_RATIO, DAMPING_SETTLE, LOD_DORMANT = 1.5, 0.01, 3

# pfsf_v1.abi.json feature_flags_required_true
REQUIRED_FEATURES = ["compute.v1", "compute.v2", "compute.v3", "compute.v4", "compute.v5", "compute.v6",
                     "compute.v7", "compute.v8", "diagnostics.v1", "extension.v1", "plan.v1", "plan.v1.1",
                     "plan_buffer", "trace.ring", "abi.v1", "crash.handler.test"]


@pytest.fixture(scope="module")
def lib(lib_built):
    return H.Host()


@pytest.fixture(scope="module")
def ref():
    if not os.path.exists(REF_LIB):
        pytest.skip("reference CPU primitives not built (make -C oracle -f ref.mk)")
    return H.Host(REF_LIB)


def bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint32 if a.dtype.itemsize == 4 else np.uint8)


def same(a, b):
    np.testing.assert_array_equal(bits(a), bits(b))


# ---------------------------------------------------------------- exports


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "pfsf", "*.h")):
        names |= set(re.findall(r"PFSF_API[^;(]*?\b(pfsf_\w+)\s*\(", open(h).read()))
    return sorted(names)


def test_library_exports_every_declared_function(lib):
    names = declared_functions()
    assert len(names) >= 87
    missing = [n for n in names if not hasattr(lib.L, n)]
    assert not missing, missing


def test_version_and_features(lib):
    assert lib.L.pfsf_abi_contract_version() == b"1.5.0"
    assert lib.L.pfsf_abi_version() == 0x000A00
    for f in REQUIRED_FEATURES:
        assert lib.L.pfsf_has_feature(f.encode()), f
    assert lib.L.pfsf_has_feature(b"solve.tolerance")
    assert not lib.L.pfsf_has_feature(b"compute.v99")
    assert not lib.L.pfsf_has_feature(None)


# ---------------------------------------------------------- known answers


def test_wind_pressure_and_timoshenko_edges(lib):  # GoldenParityTest.java:257-260, 285-286, 212-213
    L = lib.L
    assert L.pfsf_wind_pressure_source(0.0, 2400.0, True) == 0.0
    assert L.pfsf_wind_pressure_source(-5.0, 2400.0, True) == 0.0
    assert L.pfsf_wind_pressure_source(10.0, 2400.0, False) == 0.0
    assert L.pfsf_wind_pressure_source(10.0, 0.0, True) == 0.0
    assert L.pfsf_timoshenko_moment_factor(0.3, 0.5, 0, 30.0, 0.2) == 1.0
    assert L.pfsf_timoshenko_moment_factor(0.3, 0.0, 5, 30.0, 0.2) == 1.0
    rng = np.random.default_rng(7)
    for _ in range(200):
        f = L.pfsf_timoshenko_moment_factor(rng.uniform(0.1, 3), rng.uniform(0.1, 3), int(rng.integers(1, 40)),
                                            rng.uniform(1, 210), rng.uniform(0, 0.5))
        assert 1.0 <= f <= 11.0


def test_downsample_anchor_tie_break(lib):  # GoldenParityTest.java:573-589
    c, ct = lib.downsample(np.arange(1, 9, dtype=np.float32), np.array([2, 2, 2, 2, 0, 0, 0, 0], np.uint8), (2, 2, 2))
    assert c[0] == np.float32(36.0 / 8.0) and ct[0] == 2


def test_tiled_layout(lib):  # GoldenParityTest.java:593-637, 640-656
    dims = (10, 8, 9)
    rng = np.random.default_rng(0xDEADF00D)
    lin = (rng.random(int(np.prod(dims))) * 100).astype(np.float32)
    out = lib.tiled(lin, dims)
    lx, ly, lz = dims
    want = np.zeros(2 * 1 * 2 * 512, np.float32)
    for z in range(lz):
        for y in range(ly):
            for x in range(lx):
                t = ((z // 8) * 1 + y // 8) * 2 + x // 8
                want[t * 512 + ((z % 8) * 8 + y % 8) * 8 + x % 8] = lin[x + lx * (y + ly * z)]
    same(out[: want.size], want)
    lin4 = np.arange(1, 65, dtype=np.float32)
    out4 = np.zeros(64, np.float32)
    lib.L.pfsf_tiled_layout_build(H._f32(lin4), 4, 4, 4, 4, H._f32(out4))
    assert np.all(out4 == 0)


def test_normalize_noop_below_one(lib):  # GoldenParityTest.java:660-686
    n = 64
    src, rc, rt = np.ones(n, np.float32), np.full(n, 2, np.float32), np.full(n, 3, np.float32)
    cond = np.full(6 * n, 0.5, np.float32)
    assert lib.normalize_soa6(src, rc, rt, cond) == 1.0
    assert np.all(src == 1) and np.all(rc == 2) and np.all(rt == 3) and np.all(cond == 0.5)


def _div_state(prev, prev2, osc, damping, cheby, prev_macro):
    s = np.zeros(7, np.int32)
    s[0] = 28
    s[1], s[2] = np.array([prev, prev2], np.float32).view(np.int32)
    s[3], s[4], s[5] = osc, int(damping), cheby
    s[6] = np.array([prev_macro], np.float32).view(np.int32)[0]
    return s


def _f(s, k):
    return float(s[k : k + 1].view(np.float32)[0])


def test_divergence_known_answers(lib):  # GoldenParityTest.java:816-857
    s = _div_state(5.0, 4.0, 0, False, 50, 1e-5)
    assert lib.check_divergence(s, float("nan"), None, DIVERGENCE_RATIO, DAMPING_SETTLE) == H.DIV_NAN_INF
    assert s[4] == 1 and s[5] == 0 and _f(s, 1) == -1.0
    s = _div_state(1.0, 0.9, 0, False, 20, 0.0)
    assert lib.check_divergence(s, 3.0, None, DIVERGENCE_RATIO, DAMPING_SETTLE) == H.DIV_RAPID_GROWTH
    assert s[5] == 0 and _f(s, 1) == 3.0 and _f(s, 2) == 1.0
    s = _div_state(2.0, 2.0, 0, True, 10, 0.0)
    assert lib.check_divergence(s, 2.005, None, DIVERGENCE_RATIO, DAMPING_SETTLE) == H.DIV_NONE
    assert s[4] == 0 and _f(s, 1) == np.float32(2.005) and _f(s, 2) == 2.0


def test_island_features_known_answers(lib):  # GoldenParityTest.java:862-905
    rng = np.random.default_rng(0x5EED5EED)
    res = (rng.random(32) * 5e-4).astype(np.float32)
    f = lib.features(16, 24, 8, 37, 0.93, 1.2e-4, 2, 1, 17, 1, LOD_DORMANT, 1, res)
    r64 = res.astype(np.float64)
    mean = r64.mean()
    cv = np.sqrt(max((r64 * r64).mean() - mean * mean, 0)) / mean
    want = [np.log2(16 * 24 * 8), 3.0, 37 / 64, 0.93, np.log10(np.float32(1.2e-4)), res.max() / np.float32(1.2e-4),
            0.2, 1.0, 0.17, cv, 1 / LOD_DORMANT, 1.0]
    np.testing.assert_allclose(f, np.array(want, np.float32), rtol=0, atol=1e-5)


def test_arm_and_arch_known_answers(lib):  # GoldenParityTest.java:341-424
    dims = (6, 4, 3)
    n = 72
    mem = np.ones(n, np.uint8)
    anc = np.zeros(n, np.uint8)
    for z in range(3):
        anc[0 + 6 * (0 + 4 * z)] = 1
    rc, arm = lib.arm_map(mem, anc, dims)
    assert rc == 0 and arm[0] == 0 and arm[1 * 6 + 0] == 0
    assert arm[5] == 5  # (5,0,0): five horizontal steps from the anchor row
    dims = (7, 3, 2)
    mem = np.ones(42, np.uint8)
    anc = np.zeros(42, np.uint8)
    for z in range(2):
        for x in (0, 6):
            anc[x + 7 * (0 + 3 * z)] = 1
    rc, arch = lib.arch_factor(mem, anc, dims)
    assert rc == 0 and np.all((arch >= 0) & (arch <= 1))
    assert arch[3] == 1.0  # mid-span voxel equidistant from both pillars
    dims = (4, 2, 2)
    mem = np.ones(16, np.uint8)
    anc = np.zeros(16, np.uint8)
    anc[:4] = 1
    rc, arch = lib.arch_factor(mem, anc, dims)
    assert rc == 0 and np.all(arch == 0)


def test_morton_known_answers(lib):  # GoldenParityTest.java:470-503
    L = lib.L
    assert L.pfsf_morton_encode(0, 0, 0) == 0
    assert L.pfsf_morton_encode(1023, 1023, 1023) == (1 << 30) - 1
    assert L.pfsf_morton_encode(1, 0, 0) == 1 and L.pfsf_morton_encode(0, 1, 0) == 2
    assert L.pfsf_morton_encode(0, 0, 1) == 4
    rng = np.random.default_rng(3)
    for x, y, z in rng.integers(0, 1024, size=(300, 3)):
        assert lib.morton_decode(L.pfsf_morton_encode(int(x), int(y), int(z))) == (x, y, z)


def test_plan_conductivity_known_answers(lib):  # GoldenParityTest.java:1455-1500
    dims = (3, 3, 3)
    n = 27
    vt = np.ones(n, np.uint8)
    rc, rt = np.full(n, 20, np.float32), np.full(n, 5, np.float32)
    cond = np.zeros(6 * n, np.float32)
    p = H.Plan(7003).op(H.OP_COMPUTE_CONDUCTIVITY, struct.pack("<qqqqiiiiffff", H.addr(cond), H.addr(rc), H.addr(rt),
                                                                H.addr(vt), 3, 3, 3, 0, 0, 0, 0, 0))
    code, r = lib.plan_execute(p.bytes())
    assert code == 0 and r.executed_count == 1
    i = 13
    assert cond[2 * n + i] == 20 and cond[3 * n + i] == 20
    for d in (0, 1, 4, 5):
        assert cond[d * n + i] == 5.0
    assert cond[0] == 0 and cond[2 * n] == 0 and cond[4 * n] == 0


def test_augmentation_registry(lib):  # GoldenParityTest.java:946-1020, 1311-1330
    L = lib.L
    isl = 424242
    L.pfsf_aug_clear_island(isl)
    buf = np.zeros(256, np.float32)
    assert lib.aug_register(isl, H.AUG_THERMAL_FIELD, buf, 4, 7) == 0
    assert L.pfsf_aug_island_count(isl) == 1
    found, s = lib.aug_query(isl, H.AUG_THERMAL_FIELD)
    assert found == 1 and s.stride_bytes == 4 and s.version == 7 and s.dbb_bytes == 1024
    assert s.struct_bytes == 32
    assert lib.aug_query(isl, H.AUG_FLUID_PRESSURE)[0] == 0
    L.pfsf_aug_clear(isl, H.AUG_THERMAL_FIELD)
    assert L.pfsf_aug_island_count(isl) == 0
    for k, v in ((H.AUG_THERMAL_FIELD, 1), (H.AUG_FLUID_PRESSURE, 2), (H.AUG_CURING_FIELD, 3)):
        assert lib.aug_register(isl + 1, k, buf, 4, v) == 0
    assert lib.aug_register(isl + 1, H.AUG_FLUID_PRESSURE, buf, 4, 42) == 0
    assert L.pfsf_aug_island_count(isl + 1) == 3 and lib.aug_query(isl + 1, H.AUG_FLUID_PRESSURE)[1].version == 42
    L.pfsf_aug_clear_island(isl + 1)
    assert L.pfsf_aug_island_count(isl + 1) == 0
    # malformed slots
    assert lib.aug_register(isl, 0, buf, 4, 1) == capi.PFSF_ERROR_INVALID_ARG
    assert lib.aug_register(isl, 10, buf, 4, 1) == capi.PFSF_ERROR_INVALID_ARG
    assert lib.aug_register(isl, H.AUG_EM_FIELD, buf, 4, 1, struct_bytes=16) == capi.PFSF_ERROR_INVALID_ARG
    assert L.pfsf_aug_register(isl, None) == capi.PFSF_ERROR_INVALID_ARG


def test_plan_counter_hooks_and_errors(lib):  # GoldenParityTest.java:1024-1200
    L = lib.L
    L.pfsf_plan_test_counter_read_reset()
    i32 = lambda v: struct.pack("<i", v)  # noqa: E731
    p = H.Plan(0x1001).op(H.OP_NO_OP).op(H.OP_INCR_COUNTER, i32(3)).op(H.OP_INCR_COUNTER, i32(5)).op(H.OP_NO_OP)
    p.op(H.OP_INCR_COUNTER, i32(-1))
    code, r = lib.plan_execute(p.bytes())
    assert (code, r.executed_count, r.failed_index, r.error_code, r.hook_fire_count) == (0, 5, -1, 0, 0)
    assert r.struct_bytes == 20
    assert L.pfsf_plan_test_counter_read_reset() == 7
    # hooks
    isl, pt = 0x1003, H.HOOK_POST_SOURCE
    L.pfsf_hook_clear_island(isl)
    L.pfsf_plan_test_hook_install(isl, pt)
    p = H.Plan(isl)
    for e in (1, 2, 3):
        p.op(H.OP_FIRE_HOOK, struct.pack("<iq", pt, e))
    code, r = lib.plan_execute(p.bytes())
    assert code == 0 and r.executed_count == 3 and r.hook_fire_count == 3
    assert L.pfsf_plan_test_hook_count_read_reset(isl, pt) == 3
    code, r = lib.plan_execute(H.Plan(isl).op(H.OP_FIRE_HOOK, struct.pack("<iq", H.HOOK_PRE_SCAN, 99)).bytes())
    assert r.hook_fire_count == 0
    L.pfsf_hook_clear_island(isl)
    # bad magic, truncated body
    code, r = lib.plan_execute(struct.pack("<IHHii", 0xDEADBEEF, 1, 0, 0, 0))
    assert code == capi.PFSF_ERROR_INVALID_ARG and r.executed_count == 0
    code, r = lib.plan_execute(struct.pack("<IHHiiH", H.PLAN_MAGIC, 1, 0, 9001, 3, 0))
    assert code == capi.PFSF_ERROR_INVALID_ARG and r.executed_count == 0 and r.failed_index == 0
    # unknown opcode stops the plan where it stands
    L.pfsf_plan_test_counter_read_reset()
    p = H.Plan(0xBEEF).op(H.OP_NO_OP).op(H.OP_INCR_COUNTER, i32(4)).op(0xFFFF).op(H.OP_INCR_COUNTER, i32(100))
    code, r = lib.plan_execute(p.bytes())
    assert code == capi.PFSF_ERROR_INVALID_ARG and r.executed_count == 2 and r.failed_index == 2
    assert L.pfsf_plan_test_counter_read_reset() == 4
    # 100 ops
    p = H.Plan(0x1004)
    for _ in range(100):
        p.op(H.OP_INCR_COUNTER, i32(1))
    code, r = lib.plan_execute(p.bytes())
    assert code == 0 and r.executed_count == 100 and L.pfsf_plan_test_counter_read_reset() == 100
    # short argument block
    code, r = lib.plan_execute(H.Plan(1).op(H.OP_TIMOSHENKO, b"\0" * 27).bytes())
    assert code == capi.PFSF_ERROR_INVALID_ARG and r.failed_index == 0


def test_plan_augmentation_opcodes(lib):
    L = lib.L
    isl, n = 31337, 50
    L.pfsf_aug_clear_island(isl)
    rng = np.random.default_rng(11)
    slot = rng.uniform(-2, 3, n).astype(np.float32)
    assert lib.aug_register(isl, H.AUG_THERMAL_FIELD, slot, 4, 1) == 0
    src = rng.random(n).astype(np.float32)
    want = src + np.clip(slot, -1, 1)
    payload = struct.pack("<qiqiff", isl, H.AUG_THERMAL_FIELD, H.addr(src), n, -1.0, 1.0)
    L.pfsf_trace_clear()
    L.pfsf_set_trace_level_global(H.TRACE_VERBOSE)
    code, r = lib.plan_execute(H.Plan(isl).op(H.OP_AUG_SOURCE_ADD, payload).bytes())
    assert code == 0 and r.executed_count == 1
    same(src, want.astype(np.float32))
    ev = lib.drain(8)
    assert len(ev) == 1 and ev[0].msg == b"plan: aug clamp" and ev[0].voxel_index == int(np.sum(np.abs(slot) > 1))
    # unpublished kind: silent no-op
    before = src.copy()
    payload = struct.pack("<qiqiff", isl, H.AUG_EM_FIELD, H.addr(src), n, -1.0, 1.0)
    assert lib.plan_execute(H.Plan(isl).op(H.OP_AUG_SOURCE_ADD, payload).bytes())[0] == 0
    same(src, before)
    # stride mismatch for the 3-D wind form: skipped with a warning
    cond = np.ones(6 * n, np.float32)
    payload = struct.pack("<qiqifff", isl, H.AUG_THERMAL_FIELD, H.addr(cond), n, 0.5, 0.0, 2.0)
    assert lib.plan_execute(H.Plan(isl).op(H.OP_AUG_WIND_3D_BIAS, payload).bytes())[0] == 0
    assert np.all(cond == 1) and lib.drain(8)[0].msg == b"plan: aug stride mismatch"
    L.pfsf_aug_clear_island(isl)
    L.pfsf_set_trace_level_global(H.TRACE_INFO)


def test_trace_ring(lib, tmp_path):  # GoldenParityTest.java:1208-1305
    L = lib.L
    L.pfsf_trace_clear()
    L.pfsf_set_trace_level_global(H.TRACE_VERBOSE)
    L.pfsf_trace_emit(H.TRACE_ERROR, 42, 2, 777, 88, -4, b"hello trace")
    L.pfsf_trace_emit(H.TRACE_WARN, 43, 3, 777, -1, 0, b"second event")
    assert L.pfsf_trace_size() == 2
    ev = lib.drain(16)
    assert [(e.epoch, e.stage, e.island_id, e.voxel_index, e.errno_val, e.level, e.msg) for e in ev] == [
        (42, 2, 777, 88, -4, H.TRACE_ERROR, b"hello trace"), (43, 3, 777, -1, 0, H.TRACE_WARN, b"second event")]
    assert L.pfsf_trace_size() == 0
    L.pfsf_set_trace_level_global(H.TRACE_WARN)
    for lv, m in ((1, b"error"), (2, b"warn"), (3, b"info"), (4, b"verbose")):
        L.pfsf_trace_emit(lv, lv, 0, 1, -1, 0, m)
    assert L.pfsf_trace_size() == 2
    L.pfsf_set_trace_level_global(H.TRACE_OFF)
    L.pfsf_trace_emit(H.TRACE_ERROR, 5, 0, 1, -1, 0, b"even error")
    assert L.pfsf_trace_size() == 2
    L.pfsf_trace_clear()
    L.pfsf_set_trace_level_global(H.TRACE_ERROR)
    code, _ = lib.plan_execute(struct.pack("<IHHii", 0xDEADBEEF, 1, 0, 123, 0))
    e = lib.drain(4)[0]
    assert code == capi.PFSF_ERROR_INVALID_ARG and e.island_id == 123 and e.errno_val == -4 and b"plan" in e.msg
    L.pfsf_set_trace_level_global(H.TRACE_VERBOSE)
    for i in range(4100):
        L.pfsf_trace_emit(H.TRACE_INFO, i, 0, 0, -1, 0, b"e%d" % i)
    assert L.pfsf_trace_size() == 4096 and lib.drain(1)[0].epoch == 4
    # a long message is truncated to 35 bytes + NUL
    L.pfsf_trace_clear()
    L.pfsf_trace_emit(H.TRACE_INFO, 0, 0, 0, 0, 0, b"x" * 80)
    assert lib.drain(1)[0].msg == b"x" * 35
    # crash dump written synchronously (no signal is raised)
    L.pfsf_trace_emit(H.TRACE_WARN, 9, 1, 2, 3, 4, b"before crash")
    path = str(tmp_path / "dump.trace")
    assert L.pfsf_dump_now_for_test(path.encode(), 11, 0xDEADBEEF) == 1
    raw = open(path, "rb").read()
    head, body = raw.split(b"\n", 1)
    assert head == b"PFSF-CRASH signo=11 pid=%d addr=0xdeadbeef events=1" % os.getpid()
    assert len(body) == 64 and body[28:40] == b"before crash"
    assert L.pfsf_dump_now_for_test(None, 11, 0) == capi.PFSF_ERROR_INVALID_ARG
    # install / uninstall are idempotent and leave the previous handlers in place
    import signal
    prev = signal.getsignal(signal.SIGSEGV)
    assert L.pfsf_install_crash_handler() == 0 and L.pfsf_install_crash_handler() == 0
    L.pfsf_uninstall_crash_handler()
    L.pfsf_uninstall_crash_handler()
    assert signal.getsignal(signal.SIGSEGV) == prev
    L.pfsf_trace_clear()
    L.pfsf_set_trace_level_global(H.TRACE_INFO)


# ------------------------------------------------- A/B vs the reference build


def _island(rng, dims, fill=0.7):
    n = int(np.prod(dims))
    vt = (rng.random(n) < fill).astype(np.uint8)
    vt[(rng.random(n) < 0.1) & (vt == 1)] = 2
    rc = rng.uniform(0.1, 40, n).astype(np.float32)
    rt = rng.uniform(0.1, 40, n).astype(np.float32)
    rc[rng.random(n) < 0.02] = 0.0
    return vt, rc, rt


DIMS = [(1, 1, 1), (2, 3, 1), (5, 5, 5), (7, 4, 9), (16, 3, 11), (13, 17, 6)]


@pytest.mark.parametrize("dims", DIMS)
def test_ab_conductivity_normalize_phantom(lib, ref, dims):
    rng = np.random.default_rng(sum(dims))
    vt, rc, rt = _island(rng, dims)
    for wind, up in (((0, 0, 0), 0.0), ((1.5, 0, -2.0), 0.3), ((-1, 7, 0.5), 1.2)):
        a = lib.conductivity(rc, rt, vt, dims, wind, up)
        b = ref.conductivity(rc, rt, vt, dims, wind, up)
        same(a, b)
    n = vt.size
    s1 = rng.random(n).astype(np.float32) * 50
    s2 = s1.copy()
    r1, r2, t1, t2 = rc.copy(), rc.copy(), rt.copy(), rt.copy()
    c1, c2 = (a * 3).astype(np.float32), (a * 3).astype(np.float32)
    assert lib.normalize_soa6(s1, r1, t1, c1) == ref.normalize_soa6(s2, r2, t2, c2)
    for x, y in ((s1, s2), (r1, r2), (t1, t2), (c1, c2)):
        same(x, y)
    mem = (vt > 0).astype(np.uint8)
    c1, c2 = a.copy(), a.copy()
    assert lib.phantom_edges(mem, c1, rc, dims, 0.35, 0.15) == ref.phantom_edges(mem, c2, rc, dims, 0.35, 0.15)
    same(c1, c2)


@pytest.mark.parametrize("dims", DIMS + [(32, 8, 32), (9, 1, 40)])
def test_ab_topology_maps(lib, ref, dims):
    rng = np.random.default_rng(100 + sum(dims))
    n = int(np.prod(dims))
    for fill, afrac in ((0.9, 0.05), (0.6, 0.2), (1.0, 0.01)):
        mem = (rng.random(n) < fill).astype(np.uint8)
        anc = (rng.random(n) < afrac).astype(np.uint8)
        ra, a1 = lib.arm_map(mem, anc, dims)
        rb, a2 = ref.arm_map(mem, anc, dims)
        assert ra == rb == 0
        same(a1, a2)
        ra, f1 = lib.arch_factor(mem, anc, dims)
        rb, f2 = ref.arch_factor(mem, anc, dims)
        assert ra == rb == 0
        same(f1, f2)
    assert lib.arm_map(mem, anc, (0, 1, 1))[0] == capi.PFSF_ERROR_INVALID_ARG


@pytest.mark.parametrize("dims", DIMS + [(8, 8, 8), (17, 9, 3)])
def test_ab_downsample_tiled(lib, ref, dims):
    rng = np.random.default_rng(200 + sum(dims))
    n = int(np.prod(dims))
    fine = rng.normal(size=n).astype(np.float32)
    ft = rng.integers(0, 3, n).astype(np.uint8)
    for a, b in zip(lib.downsample(fine, ft, dims), ref.downsample(fine, ft, dims)):
        same(a, b)
    same(lib.tiled(fine, dims), ref.tiled(fine, dims))


def test_ab_scalars(lib, ref):
    rng = np.random.default_rng(5)
    A, B = lib.L, ref.L
    for _ in range(2000):
        b, h, E, nu = (float(v) for v in rng.uniform([-1, -1, 0.5, -0.2], [4, 4, 250, 0.8]))
        arm = int(rng.integers(-2, 60))
        assert bits(np.float32(A.pfsf_timoshenko_moment_factor(b, h, arm, E, nu))) == bits(
            np.float32(B.pfsf_timoshenko_moment_factor(b, h, arm, E, nu)))
        v, d = float(rng.uniform(-5, 60)), float(rng.uniform(-100, 8000))
        assert A.pfsf_wind_pressure_source(v, d, True) == B.pfsf_wind_pressure_source(v, d, True)
        x, y, z = (int(t) for t in rng.integers(0, 1 << 12, 3))
        assert A.pfsf_morton_encode(x, y, z) == B.pfsf_morton_encode(x, y, z)
        code = int(rng.integers(0, 1 << 32))
        assert lib.morton_decode(code) == ref.morton_decode(code)
    for rho in list(rng.uniform(0, 1.2, 60)) + [0.0, 0.9245, 0.999, 1.0, float("nan")]:
        for it in range(0, 90, 7):
            a, b = A.pfsf_chebyshev_omega(it, rho), B.pfsf_chebyshev_omega(it, rho)
            assert bits(np.float32(a)) == bits(np.float32(b))
        for cap in (1, 2, 64, 100):
            (ra, ta), (rb, tb) = lib.omega_table(rho, cap), ref.omega_table(rho, cap)
            assert ra == rb
            same(ta, tb)
    assert lib.omega_table(0.9, 0)[0] == capi.PFSF_ERROR_INVALID_ARG
    for lmax in (-3, 0, 1, 2, 7, 64, 513):
        for m in (0.95, 1.0, 0.5):
            assert A.pfsf_estimate_spectral_radius(lmax, m) == B.pfsf_estimate_spectral_radius(lmax, m)
    for args in rng.integers(-3, 140, size=(500, 7)):
        a = [int(v) for v in args]
        a[2], a[3] = a[2] % 2, a[3] % 2
        assert A.pfsf_recommend_steps(*a) == B.pfsf_recommend_steps(*a)
    res = rng.uniform(0, 3e-4, 300).astype(np.float32)
    was = rng.integers(0, 2, 300).astype(np.uint8)
    for r, w in zip(res, was):
        assert A.pfsf_macro_block_active(float(r), int(w)) == B.pfsf_macro_block_active(float(r), int(w))
    assert lib.macro_active_ratio(res, was) == ref.macro_active_ratio(res, was)
    assert lib.macro_active_ratio(res) == ref.macro_active_ratio(res)


def test_ab_divergence_and_features(lib, ref):
    rng = np.random.default_rng(9)
    s1 = _div_state(0, 0, 0, False, 0, 0)
    s2 = s1.copy()
    phi = 1.0
    for t in range(3000):
        r = rng.random()
        if r < 0.01:
            phi = float("nan")
        elif r < 0.02:
            phi = float("inf")
        else:
            phi = abs(phi if np.isfinite(phi) else 1.0) * float(rng.choice([0.5, 0.9, 0.99, 1.0, 1.01, 1.2, 1.6, 3]))
        macro = None if rng.random() < 0.3 else (rng.random(int(rng.integers(1, 20))) * 1e-3).astype(np.float32)
        ka = lib.check_divergence(s1, phi, macro, DIVERGENCE_RATIO, DAMPING_SETTLE)
        kb = ref.check_divergence(s2, phi, macro, DIVERGENCE_RATIO, DAMPING_SETTLE)
        assert ka == kb, t
        same(s1, s2)
    for _ in range(300):
        lx, ly, lz = (int(v) for v in rng.integers(-1, 70, 3))
        m = None if rng.random() < 0.2 else rng.random(int(rng.integers(0, 40))).astype(np.float32) * 1e-3
        args = (lx, ly, lz, int(rng.integers(0, 80)), float(rng.random()), float(rng.choice([0, 1e-30, 2e-4])),
                int(rng.integers(-2, 15)), int(rng.integers(0, 2)), int(rng.integers(-5, 150)),
                int(rng.integers(0, 4)), int(rng.integers(-1, 4)), int(rng.integers(0, 2)), m)
        same(lib.features(*args), ref.features(*args))


def _full_plan(isl, bufs):
    """One plan exercising every compute opcode over the arrays in bufs."""
    b = bufs
    dims = b["dims"]
    n = int(np.prod(dims))
    p = H.Plan(isl)
    p.op(H.OP_COMPUTE_CONDUCTIVITY, struct.pack("<qqqqiiiiffff", H.addr(b["cond"]), H.addr(b["rc"]), H.addr(b["rt"]),
                                                H.addr(b["vt"]), *dims, 0, 1.0, 0.0, -0.5, 0.25))
    p.op(H.OP_PHANTOM_EDGES, struct.pack("<qqqqiiiiff", H.addr(b["mem"]), H.addr(b["cond"]), H.addr(b["rc"]),
                                         H.addr(b["inj"]), *dims, 0, 0.3, 0.1))
    p.op(H.OP_NORMALIZE_SOA6, struct.pack("<qqqqqqii", H.addr(b["src"]), H.addr(b["rc"]), H.addr(b["rt"]),
                                          H.addr(b["cond"]), 0, H.addr(b["sig"]), n, 0))
    p.op(H.OP_APPLY_WIND_BIAS, struct.pack("<qiiffff", H.addr(b["cond"]), n, 0, 1.0, 0.0, 0.0, 0.5))
    p.op(H.OP_ARM_MAP, struct.pack("<qqqiiii", H.addr(b["mem"]), H.addr(b["anc"]), H.addr(b["arm"]), *dims, 0))
    p.op(H.OP_ARCH_FACTOR, struct.pack("<qqqiiii", H.addr(b["mem"]), H.addr(b["anc"]), H.addr(b["arch"]), *dims, 0))
    p.op(H.OP_DOWNSAMPLE_2TO1, struct.pack("<qqqqiiii", H.addr(b["src"]), H.addr(b["vt"]), H.addr(b["crs"]),
                                           H.addr(b["ctyp"]), *dims, 0))
    p.op(H.OP_TILED_LAYOUT, struct.pack("<qqiiii", H.addr(b["src"]), H.addr(b["tiled"]), *dims, 8))
    p.op(H.OP_CHEBYSHEV, struct.pack("<qiif", H.addr(b["scal"][0:]), 17, 0, 0.97))
    p.op(H.OP_CHECK_DIVERGENCE, struct.pack("<qqqfiff", H.addr(b["div"]), H.addr(b["macro"]), H.addr(b["kind"]),
                                            2.5, b["macro"].size, 1.5, 0.01))
    p.op(H.OP_EXTRACT_FEATURES, struct.pack("<qq" + "i" * 12 + "ff", H.addr(b["macro"]), H.addr(b["feat"]), *dims,
                                            12, 3, 1, 40, 1, 3, 1, b["macro"].size, 0, 0.91, 2e-4))
    p.op(H.OP_WIND_PRESSURE, struct.pack("<qffii", H.addr(b["scal"][1:]), 23.0, 2400.0, 1, 0))
    p.op(H.OP_TIMOSHENKO, struct.pack("<qffiff", H.addr(b["scal"][2:]), 0.5, 1.5, 6, 30.0, 0.2))
    return p


def _plan_buffers(seed):
    rng = np.random.default_rng(seed)
    dims = (11, 6, 9)
    n = int(np.prod(dims))
    vt, rc, rt = _island(rng, dims, 0.8)
    nc = 6 * 3 * 5
    return {"dims": dims, "vt": vt, "rc": rc, "rt": rt, "mem": (vt > 0).astype(np.uint8),
            "anc": ((rng.random(n) < 0.1) & (vt > 0)).astype(np.uint8), "cond": np.zeros(6 * n, np.float32),
            "inj": np.zeros(1, np.int32), "src": (rng.random(n) * 30).astype(np.float32), "sig": np.zeros(1, np.float32),
            "arm": np.zeros(n, np.int32), "arch": np.zeros(n, np.float32), "crs": np.zeros(nc, np.float32),
            "ctyp": np.zeros(nc, np.uint8), "tiled": np.zeros(2 * 1 * 2 * 512, np.float32),
            "scal": np.zeros(3, np.float32), "div": _div_state(2.0, 1.9, 1, True, 5, 1e-4),
            "macro": (rng.random(12) * 5e-4).astype(np.float32), "kind": np.zeros(1, np.int32),
            "feat": np.zeros(12, np.float32)}


def test_ab_full_plan(lib, ref):
    b1, b2 = _plan_buffers(77), _plan_buffers(77)
    c1, r1 = lib.plan_execute(_full_plan(5, b1).bytes())
    c2, r2 = ref.plan_execute(_full_plan(5, b2).bytes())
    assert c1 == c2 == 0
    assert (r1.executed_count, r1.failed_index) == (r2.executed_count, r2.failed_index) == (13, -1)
    for k in b1:
        if k != "dims":
            same(b1[k], b2[k])
    assert b1["inj"][0] > 0 and b1["sig"][0] > 1


@pytest.mark.parametrize("cut", [0, 1, 15, 16, 17, 19, 20, 40, 75])
def test_ab_plan_truncation_and_bad_args(lib, ref, cut):
    b1, b2 = _plan_buffers(3), _plan_buffers(3)
    p1, p2 = _full_plan(5, b1).bytes(), _full_plan(5, b2).bytes()
    c1, r1 = lib.plan_execute(p1, cut)
    c2, r2 = ref.plan_execute(p2, cut)
    assert (c1, r1.executed_count, r1.failed_index, r1.error_code) == (c2, r2.executed_count, r2.failed_index,
                                                                       r2.error_code)
    # a zero pointer or an oversize box is rejected at the record
    for op, payload in ((H.OP_TILED_LAYOUT, struct.pack("<qqiiii", 0, H.addr(b1["tiled"]), 4, 4, 4, 8)),
                        (H.OP_ARM_MAP, struct.pack("<qqqiiii", H.addr(b1["mem"]), H.addr(b1["anc"]), H.addr(b1["arm"]),
                                                   513, 1, 1, 0)),
                        (H.OP_NORMALIZE_SOA6, struct.pack("<qqqqqqii", *([H.addr(b1["src"])] * 6), 1000001, 0)),
                        (H.OP_AUG_COND_MUL, struct.pack("<qiqiff", 1, 1, H.addr(b1["cond"]), 4, 2.0, 1.0))):
        pl = H.Plan(1).op(H.OP_NO_OP).op(op, payload).bytes()
        ra, rb = lib.plan_execute(pl), ref.plan_execute(pl)
        assert ra[0] == rb[0] == capi.PFSF_ERROR_INVALID_ARG
        assert ra[1].failed_index == rb[1].failed_index == 1


def test_ab_augmentation_kernels(lib, ref):
    rng = np.random.default_rng(21)
    n = 257
    for L in (lib, ref):
        L.L.pfsf_aug_clear_island(900)
        L.L.pfsf_set_trace_level_global(H.TRACE_VERBOSE)
        L.L.pfsf_trace_clear()
    s1 = rng.normal(size=n).astype(np.float32) * 2
    s1[::17] = np.nan
    w3 = rng.normal(size=3 * n).astype(np.float32)
    outs = []
    for L in (lib, ref):
        L.aug_register(900, H.AUG_FLUID_PRESSURE, s1, 4, 1)
        L.aug_register(900, H.AUG_WIND_FIELD_3D, w3, 12, 1)
        src = np.linspace(0, 1, n, dtype=np.float32)
        rc = np.linspace(1, 2, n, dtype=np.float32)
        cond = np.linspace(0.5, 3, 6 * n, dtype=np.float32)
        p = H.Plan(900)
        p.op(H.OP_AUG_SOURCE_ADD, struct.pack("<qiqiff", 900, H.AUG_FLUID_PRESSURE, H.addr(src), n, -1.0, 1.5))
        p.op(H.OP_AUG_RCOMP_MUL, struct.pack("<qiqiff", 900, H.AUG_FLUID_PRESSURE, H.addr(rc), n, 0.2, 1.0))
        p.op(H.OP_AUG_COND_MUL, struct.pack("<qiqiff", 900, H.AUG_FLUID_PRESSURE, H.addr(cond), n, 0.0, 2.0))
        p.op(H.OP_AUG_WIND_3D_BIAS, struct.pack("<qiqifff", 900, H.AUG_WIND_FIELD_3D, H.addr(cond), n, 0.7, 0.5,
                                                1.4))
        p.op(H.OP_AUG_SOURCE_ADD, struct.pack("<qiqiff", 900, H.AUG_FLUID_PRESSURE, H.addr(src), n + 1, -1.0, 1.5))
        code, r = L.plan_execute(p.bytes())
        ev = [(e.level, e.island_id, e.voxel_index, e.errno_val, e.msg) for e in L.drain(64)]
        outs.append((code, r.executed_count, src, rc, cond, ev))
        L.L.pfsf_aug_clear_island(900)
        L.L.pfsf_set_trace_level_global(H.TRACE_INFO)
    a, b = outs
    assert a[:2] == b[:2] == (0, 5)
    for x, y in zip(a[2:5], b[2:5]):
        same(x, y)
    assert a[5] == b[5] and len(a[5]) == 5


def test_ab_trace_and_dump_bytes(lib, ref, tmp_path):
    files = []
    for k, L in enumerate((lib, ref)):
        L.L.pfsf_trace_clear()
        L.L.pfsf_set_trace_level_global(H.TRACE_VERBOSE)
        for i in range(130):
            L.L.pfsf_trace_emit(1 + i % 4, i * 1000, i % 6, 7, i, -i, b"event %d with a long tail text" % i)
        L.L.pfsf_trace_emit(2, -5, -1, -1, -1, 0, None)
        path = str(tmp_path / ("d%d" % k))
        assert L.L.pfsf_dump_now_for_test(path.encode(), 6, 0x7F00ABC) == 100
        files.append(open(path, "rb").read())
        raw = (H.TraceEvent * 200)()
        assert L.L.pfsf_drain_trace_dbb(raw, 64 * 10 + 5, 200) == 10
        files.append(bytes(raw)[:640])
        assert L.L.pfsf_drain_trace_dbb(None, 0, 50) == capi.PFSF_ERROR_INVALID_ARG
        assert L.L.pfsf_drain_trace_dbb(None, 0, 0) == 0
        assert L.L.pfsf_trace_size() == 121
        assert L.L.pfsf_drain_trace_dbb(None, 0, -1) == capi.PFSF_ERROR_INVALID_ARG
        L.L.pfsf_trace_clear()
        L.L.pfsf_set_trace_level_global(H.TRACE_INFO)
    assert files[0] == files[2] and files[1] == files[3]
