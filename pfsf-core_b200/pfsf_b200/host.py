"""ctypes binding of the host-side primitives of the frozen ABI.

pfsf_compute.h, pfsf_diagnostics.h, pfsf_extension.h, pfsf_plan.h,
pfsf_trace.h and pfsf_version.h: the CPU functions the Java bridge reaches
through NativePFSFBridge.native* (reference:
Block Reality/api/src/main/java/com/blockreality/api/physics/pfsf/NativePFSFBridge.java).
They run on the caller's thread and need no GPU.

``Host(path)`` binds any library exporting these symbols, so the same
wrappers drive libpfsf.so and, in tests, a reference-built library.
Arrays are numpy arrays modified in place where the C function writes.
"""
from __future__ import annotations

import ctypes as C
import struct

import numpy as np

from . import capi

f32p = C.POINTER(C.c_float)
i32p = C.POINTER(C.c_int32)
u8p = C.POINTER(C.c_uint8)
u32p = C.POINTER(C.c_uint32)

# pfsf_trace.h
TRACE_OFF, TRACE_ERROR, TRACE_WARN, TRACE_INFO, TRACE_VERBOSE = range(5)
TRACE_RING_CAPACITY = 4096
CRASH_MAX_EVENTS = 100
# pfsf_extension.h
AUG_THERMAL_FIELD, AUG_TENSION_OVERRIDE, AUG_FLUID_PRESSURE, AUG_EM_FIELD, AUG_FUSION_MASK = 1, 2, 3, 4, 5
AUG_WIND_FIELD_3D, AUG_MATERIAL_OVR, AUG_CURING_FIELD, AUG_LOADPATH_HINT = 6, 7, 8, 9
HOOK_PRE_SOURCE, HOOK_POST_SOURCE, HOOK_PRE_SOLVE, HOOK_POST_SOLVE, HOOK_PRE_SCAN, HOOK_POST_SCAN = range(6)
# pfsf_diagnostics.h
DIV_NONE, DIV_NAN_INF, DIV_RAPID_GROWTH, DIV_OSCILLATION, DIV_PERSISTENT_OSC, DIV_MACRO_REGION = range(6)
# pfsf_plan.h
PLAN_MAGIC = 0x46534650
PLAN_VERSION = 1
(OP_NO_OP, OP_INCR_COUNTER, OP_CLEAR_AUG, OP_CLEAR_AUG_ISLAND, OP_FIRE_HOOK, OP_NORMALIZE_SOA6, OP_APPLY_WIND_BIAS,
 OP_COMPUTE_CONDUCTIVITY, OP_ARM_MAP, OP_ARCH_FACTOR, OP_PHANTOM_EDGES, OP_DOWNSAMPLE_2TO1, OP_TILED_LAYOUT,
 OP_CHEBYSHEV, OP_CHECK_DIVERGENCE, OP_EXTRACT_FEATURES, OP_WIND_PRESSURE, OP_TIMOSHENKO, OP_AUG_SOURCE_ADD,
 OP_AUG_COND_MUL, OP_AUG_RCOMP_MUL, OP_AUG_WIND_3D_BIAS) = range(22)


class TraceEvent(C.Structure):
    _fields_ = [("epoch", C.c_int64), ("stage", C.c_int32), ("island_id", C.c_int32), ("voxel_index", C.c_int32),
                ("errno_val", C.c_int32), ("level", C.c_int16), ("_pad", C.c_int16), ("msg", C.c_char * 36)]


class AugSlot(C.Structure):
    _fields_ = [("struct_bytes", C.c_int32), ("kind", C.c_int32), ("dbb_addr", C.c_void_p),
                ("dbb_bytes", C.c_int64), ("stride_bytes", C.c_int32), ("version", C.c_int32)]


class PlanResult(C.Structure):
    _fields_ = [("struct_bytes", C.c_int32), ("executed_count", C.c_int32), ("failed_index", C.c_int32),
                ("error_code", C.c_int32), ("hook_fire_count", C.c_int32)]


HOOK_FN = C.CFUNCTYPE(None, C.c_int32, C.c_int64, C.c_void_p)

assert C.sizeof(TraceEvent) == 64

_SIGS = {
    "pfsf_normalize_soa6": (None, [f32p, f32p, f32p, f32p, f32p, C.c_int32, f32p]),
    "pfsf_apply_wind_bias": (None, [f32p, C.c_int32, capi.Vec3, C.c_float]),
    "pfsf_timoshenko_moment_factor": (C.c_float, [C.c_float, C.c_float, C.c_int32, C.c_float, C.c_float]),
    "pfsf_wind_pressure_source": (C.c_float, [C.c_float, C.c_float, C.c_bool]),
    "pfsf_compute_arm_map": (C.c_int32, [u8p, u8p, C.c_int32, C.c_int32, C.c_int32, i32p]),
    "pfsf_compute_arch_factor_map": (C.c_int32, [u8p, u8p, C.c_int32, C.c_int32, C.c_int32, f32p]),
    "pfsf_inject_phantom_edges": (C.c_int32, [u8p, f32p, f32p, C.c_int32, C.c_int32, C.c_int32, C.c_float,
                                              C.c_float]),
    "pfsf_compute_conductivity": (None, [f32p, f32p, f32p, u8p, C.c_int32, C.c_int32, C.c_int32, capi.Vec3,
                                         C.c_float]),
    "pfsf_downsample_2to1": (None, [f32p, u8p, C.c_int32, C.c_int32, C.c_int32, f32p, u8p]),
    "pfsf_morton_encode": (C.c_uint32, [C.c_uint32, C.c_uint32, C.c_uint32]),
    "pfsf_morton_decode": (None, [C.c_uint32, u32p, u32p, u32p]),
    "pfsf_tiled_layout_build": (None, [f32p, C.c_int32, C.c_int32, C.c_int32, C.c_int32, f32p]),
    "pfsf_chebyshev_omega": (C.c_float, [C.c_int32, C.c_float]),
    "pfsf_precompute_omega_table": (C.c_int32, [C.c_float, f32p, C.c_int32]),
    "pfsf_estimate_spectral_radius": (C.c_float, [C.c_int32, C.c_float]),
    "pfsf_check_divergence": (C.c_int32, [C.c_void_p, C.c_float, f32p, C.c_int32, C.c_float, C.c_float]),
    "pfsf_recommend_steps": (C.c_int32, [C.c_int32] * 7),
    "pfsf_macro_block_active": (C.c_int32, [C.c_float, C.c_int32]),
    "pfsf_macro_active_ratio": (C.c_float, [f32p, C.c_int32, u8p]),
    "pfsf_extract_island_features": (None, [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_float, C.c_float,
                                            C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                            f32p, C.c_int32, f32p]),
    "pfsf_abi_version": (C.c_uint32, []),
    "pfsf_has_feature": (C.c_bool, [C.c_char_p]),
    "pfsf_build_info": (C.c_char_p, []),
    "pfsf_abi_contract_version": (C.c_char_p, []),
    "pfsf_aug_register": (C.c_int32, [C.c_int32, C.POINTER(AugSlot)]),
    "pfsf_aug_clear": (None, [C.c_int32, C.c_int32]),
    "pfsf_aug_clear_island": (None, [C.c_int32]),
    "pfsf_aug_query": (C.c_int32, [C.c_int32, C.c_int32, C.POINTER(AugSlot)]),
    "pfsf_aug_island_count": (C.c_int32, [C.c_int32]),
    "pfsf_hook_set": (None, [C.c_int32, C.c_int32, HOOK_FN, C.c_void_p]),
    "pfsf_hook_fire": (C.c_int32, [C.c_int32, C.c_int32, C.c_int64]),
    "pfsf_hook_clear": (None, [C.c_int32, C.c_int32]),
    "pfsf_hook_clear_island": (None, [C.c_int32]),
    "pfsf_plan_execute": (C.c_int32, [C.c_void_p, C.c_int64, C.POINTER(PlanResult)]),
    "pfsf_plan_test_counter_read_reset": (C.c_int64, []),
    "pfsf_plan_test_hook_install": (None, [C.c_int32, C.c_int32]),
    "pfsf_plan_test_hook_count_read_reset": (C.c_int64, [C.c_int32, C.c_int32]),
    "pfsf_trace_emit": (None, [C.c_int16, C.c_int64, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_char_p]),
    "pfsf_drain_trace_dbb": (C.c_int32, [C.c_void_p, C.c_int64, C.c_int32]),
    "pfsf_set_trace_level_global": (None, [C.c_int32]),
    "pfsf_get_trace_level_global": (C.c_int32, []),
    "pfsf_trace_size": (C.c_int32, []),
    "pfsf_trace_clear": (None, []),
    "pfsf_install_crash_handler": (C.c_int32, []),
    "pfsf_uninstall_crash_handler": (None, []),
    "pfsf_dump_now_for_test": (C.c_int32, [C.c_char_p, C.c_int32, C.c_size_t]),
}


def _p(a, t):
    return None if a is None else a.ctypes.data_as(t)


def _f32(a):
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(f32p)


class Host:
    """Host primitives of one loaded library (libpfsf.so by default)."""

    def __init__(self, path: str | None = None):
        self.L = C.CDLL(path or capi.LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(self.L, name)
            fn.restype = res
            fn.argtypes = args
        self._hooks = []  # keep ctypes callbacks alive

    # ---- compute.v1..v3
    def normalize_soa6(self, source, rcomp, rtens, cond, hydration=None):
        out = C.c_float()
        self.L.pfsf_normalize_soa6(_f32(source), _f32(rcomp), _f32(rtens), _f32(cond), _p(hydration, f32p),
                                   source.size, C.byref(out))
        return out.value

    def conductivity(self, rcomp, rtens, vtype, dims, wind=(0.0, 0.0, 0.0), upwind=0.0):
        n = int(np.prod(dims))
        out = np.full(6 * n, np.nan, np.float32)
        self.L.pfsf_compute_conductivity(_f32(out), _f32(rcomp), _f32(rtens), _p(vtype, u8p), *dims,
                                         capi.Vec3(*wind), upwind)
        return out

    def arm_map(self, members, anchors, dims):
        out = np.full(int(np.prod(dims)), -7, np.int32)
        rc = self.L.pfsf_compute_arm_map(_p(members, u8p), _p(anchors, u8p), *dims, _p(out, i32p))
        return rc, out

    def arch_factor(self, members, anchors, dims):
        out = np.full(int(np.prod(dims)), np.nan, np.float32)
        rc = self.L.pfsf_compute_arch_factor_map(_p(members, u8p), _p(anchors, u8p), *dims, _f32(out))
        return rc, out

    def phantom_edges(self, members, cond, rcomp, dims, edge, corner):
        return self.L.pfsf_inject_phantom_edges(_p(members, u8p), _f32(cond), _f32(rcomp), *dims, edge, corner)

    def downsample(self, fine, ftype, dims):
        nc = int(np.prod([(d + 1) // 2 for d in dims]))
        c = np.full(nc, np.nan, np.float32)
        ct = np.full(nc, 77, np.uint8)
        self.L.pfsf_downsample_2to1(_f32(fine), _p(ftype, u8p), *dims, _f32(c), _p(ct, u8p))
        return c, ct

    def tiled(self, linear, dims, tile=8):
        nt = int(np.prod([(d + 7) // 8 for d in dims])) * 512
        out = np.full(max(nt, linear.size), np.nan, np.float32)
        self.L.pfsf_tiled_layout_build(_f32(linear), *dims, tile, _f32(out))
        return out

    def morton_decode(self, code):
        x, y, z = C.c_uint32(), C.c_uint32(), C.c_uint32()
        self.L.pfsf_morton_decode(code, C.byref(x), C.byref(y), C.byref(z))
        return x.value, y.value, z.value

    # ---- compute.v4
    def omega_table(self, rho, cap=64):
        out = np.zeros(max(cap, 1), np.float32)
        rc = self.L.pfsf_precompute_omega_table(rho, _f32(out), cap)
        return rc, out

    def check_divergence(self, state, now, macro=None, ratio=2.0, settle=0.01):
        """state: int32[7] (Java's view: struct_bytes, floats as raw bits)."""
        assert state.dtype == np.int32 and state.size == 7
        m = None if macro is None else np.ascontiguousarray(macro, np.float32)
        return self.L.pfsf_check_divergence(state.ctypes.data, now, _p(m, f32p), 0 if m is None else m.size,
                                            ratio, settle)

    def features(self, lx, ly, lz, cheby, rho, prev, osc, damping, stable, lod, dormant, pcg, macro):
        out = np.full(12, np.nan, np.float32)
        m = None if macro is None else np.ascontiguousarray(macro, np.float32)
        self.L.pfsf_extract_island_features(lx, ly, lz, cheby, rho, prev, osc, damping, stable, lod, dormant, pcg,
                                            _p(m, f32p), 0 if m is None else m.size, _f32(out))
        return out

    def macro_active_ratio(self, residuals, was_active=None):
        r = np.ascontiguousarray(residuals, np.float32)
        return self.L.pfsf_macro_active_ratio(_f32(r), r.size, _p(was_active, u8p))

    # ---- compute.v5
    def aug_register(self, island, kind, buf, stride, version, nbytes=None, struct_bytes=None):
        s = AugSlot(C.sizeof(AugSlot) if struct_bytes is None else struct_bytes, kind,
                    None if buf is None else buf.ctypes.data, buf.nbytes if nbytes is None else nbytes, stride,
                    version)
        return self.L.pfsf_aug_register(island, C.byref(s))

    def aug_query(self, island, kind):
        s = AugSlot()
        s.struct_bytes = C.sizeof(AugSlot)
        found = self.L.pfsf_aug_query(island, kind, C.byref(s))
        return found, s

    def hook_set(self, island, point, fn, user_data=None):
        cb = HOOK_FN(fn)
        self._hooks.append(cb)
        self.L.pfsf_hook_set(island, point, cb, user_data)

    # ---- compute.v6
    def plan_execute(self, plan: bytes, nbytes: int | None = None):
        buf = C.create_string_buffer(plan, len(plan))
        r = PlanResult()
        rc = self.L.pfsf_plan_execute(buf, len(plan) if nbytes is None else nbytes, C.byref(r))
        return rc, r

    # ---- compute.v7
    def drain(self, capacity):
        arr = (TraceEvent * max(capacity, 1))()
        n = self.L.pfsf_drain_trace_dbb(arr, C.sizeof(arr), capacity)
        return [arr[i] for i in range(max(n, 0))] if n >= 0 else n


class Plan:
    """Little-endian tick-plan assembler (the Java PFSFTickPlanner's format)."""

    def __init__(self, island: int):
        self.island = island
        self.ops: list[bytes] = []

    def op(self, opcode: int, payload: bytes = b"") -> "Plan":
        self.ops.append(struct.pack("<HH", opcode, len(payload)) + payload)
        return self

    def bytes(self) -> bytes:
        return struct.pack("<IHHii", PLAN_MAGIC, PLAN_VERSION, 0, self.island, len(self.ops)) + b"".join(self.ops)


def addr(a) -> int:
    """Raw address of a numpy array (the int64 a plan record carries)."""
    return 0 if a is None else int(a.ctypes.data)
