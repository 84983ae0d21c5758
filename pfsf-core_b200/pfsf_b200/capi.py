"""ctypes binding of libpfsf.so (the C ABI in include/pfsf/*.h).

This is the binding a Python caller -- or a test -- uses; the Java caller
binds the same symbols through a JNI shim.  Loading fails
loudly when the library has not been built: there is no fallback path.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libpfsf.so")

# ---- pfsf_types.h
PFSF_OK, PFSF_ERROR_VULKAN, PFSF_ERROR_NO_DEVICE, PFSF_ERROR_OUT_OF_VRAM = 0, -1, -2, -3
PFSF_ERROR_INVALID_ARG, PFSF_ERROR_NOT_INIT, PFSF_ERROR_ISLAND_FULL = -4, -5, -6
PREC_FP32, PREC_BF16, PREC_FP16 = 0, 1, 2
SOLVE_PER_ISLAND, SOLVE_BATCHED = 0, 1
SOLVE_NO_UPLOAD, SOLVE_NO_READBACK, SOLVE_COLD_START = 0x1, 0x2, 0x4


class Pos(C.Structure):
    _fields_ = [("x", C.c_int32), ("y", C.c_int32), ("z", C.c_int32)]


class Vec3(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("z", C.c_float)]


class IslandDesc(C.Structure):
    _fields_ = [("island_id", C.c_int32), ("origin", Pos), ("lx", C.c_int32), ("ly", C.c_int32),
                ("lz", C.c_int32)]


class Config(C.Structure):
    _fields_ = [("max_island_size", C.c_int32), ("tick_budget_ms", C.c_int32),
                ("vram_budget_bytes", C.c_int64), ("enable_phase_field", C.c_bool),
                ("enable_multigrid", C.c_bool)]


class Stats(C.Structure):
    _fields_ = [("island_count", C.c_int32), ("total_voxels", C.c_int64), ("vram_used_bytes", C.c_int64),
                ("vram_budget_bytes", C.c_int64), ("last_tick_ms", C.c_float)]


class FailureEvent(C.Structure):
    _fields_ = [("pos", Pos), ("type", C.c_int32)]


class TickResult(C.Structure):
    _fields_ = [("events", C.POINTER(FailureEvent)), ("capacity", C.c_int32), ("count", C.c_int32)]


class VoxelUpdate(C.Structure):
    _fields_ = [("flat_index", C.c_int32), ("source", C.c_float), ("type", C.c_int32), ("max_phi", C.c_float),
                ("rcomp", C.c_float), ("cond", C.c_float * 6)]


class IslandBuffers(C.Structure):
    _fields_ = [(n, t) for pair in [("phi", None), ("source", None), ("conductivity", None), ("voxel_type", None),
                                    ("rcomp", None), ("rtens", None), ("max_phi", None)]
                for n, t in ((pair[0] + "_addr", C.c_void_p), (pair[0] + "_bytes", C.c_int64))]


class IslandLookups(C.Structure):
    _fields_ = [(n, t) for pair in ["material_id", "anchor_bitmap", "fluid_pressure", "curing"]
                for n, t in ((pair + "_addr", C.c_void_p), (pair + "_bytes", C.c_int64))]


class KappaBuffers(C.Structure):
    _fields_ = [(n, t) for pair in ["phi", "source", "kappa", "voxel_type"]
                for n, t in ((pair + "_addr", C.c_void_p), (pair + "_bytes", C.c_int64))]


class AdjointBuffers(C.Structure):
    _fields_ = [(n, t) for pair in ["grad_phi", "grad_source", "grad_kappa"]
                for n, t in ((pair + "_addr", C.c_void_p), (pair + "_bytes", C.c_int64))]


class SolveStats(C.Structure):
    _fields_ = [("struct_bytes", C.c_int32), ("islands_solved", C.c_int32), ("islands_converged", C.c_int32),
                ("max_iterations", C.c_int32), ("max_rel_residual", C.c_double), ("device_ms", C.c_float),
                ("upload_ms", C.c_float), ("readback_ms", C.c_float), ("kernel_launches", C.c_int32),
                ("inner_iterations_total", C.c_int64), ("algorithmic_bytes", C.c_double),
                ("active_voxels", C.c_int64), ("island_ms_sum", C.c_double), ("island_ms_max", C.c_double),
                ("span_ms", C.c_double), ("setup_ms_sum", C.c_double), ("precond_ms_sum", C.c_double),
                ("vcycle_fine_ms_sum", C.c_double), ("vcycle_coarse_ms_sum", C.c_double),
                ("vcycle_tail_ms_sum", C.c_double), ("persistent_ctas", C.c_int32), ("reserved", C.c_int32)]


class IslandReport(C.Structure):
    TEAMS = {0: "plain", 1: "grid", 2: "cluster", 3: "cta", 4: "warp"}
    _fields_ = [("struct_bytes", C.c_int32), ("lx", C.c_int32), ("ly", C.c_int32), ("lz", C.c_int32),
                ("levels", C.c_int32), ("inner_iterations", C.c_int32), ("outer_iterations", C.c_int32),
                ("converged", C.c_int32), ("team", C.c_int32), ("team_ctas", C.c_int32),
                ("rel_residual", C.c_double), ("solve_ms", C.c_double), ("setup_ms", C.c_double),
                ("precond_ms", C.c_double), ("start_ms", C.c_double)]


class TickReport(C.Structure):
    _fields_ = [("struct_bytes", C.c_int32), ("islands", C.c_int32), ("groups", C.c_int32),
                ("graph_replayed", C.c_int32), ("kernel_launches", C.c_int64), ("algorithmic_bytes", C.c_double),
                ("grid_voxels", C.c_double), ("device_ms", C.c_float), ("host_us", C.c_int32)]


MG_V, MG_W = 0, 1


class Tuning(C.Structure):
    SOURCES = {0: "default", 1: "file", 2: "env", 3: "caller"}
    _fields_ = [("struct_bytes", C.c_int32), ("cluster", C.c_int32), ("cluster_min_voxels", C.c_int64),
                ("grid_min_voxels", C.c_int64), ("warp_max_voxels", C.c_int64), ("cheb_k", C.c_int32),
                ("source", C.c_int32), ("cheb_lower", C.c_float), ("coarse_weight", C.c_float),
                ("tail_cells", C.c_int32), ("coarse_sweeps", C.c_int32), ("inner_eta", C.c_float),
                ("reserved", C.c_int32)]

    def as_dict(self):
        return {"cluster": self.cluster, "cluster_min_voxels": self.cluster_min_voxels,
                "grid_min_voxels": self.grid_min_voxels, "warp_max_voxels": self.warp_max_voxels,
                "cheb_k": self.cheb_k, "cheb_lower": round(float(self.cheb_lower), 6),
                "coarse_weight": round(float(self.coarse_weight), 6),
                "tail_cells": self.tail_cells,
                "coarse_sweeps": self.coarse_sweeps, "inner_eta": round(float(self.inner_eta), 8),
                "source": self.SOURCES.get(self.source, str(self.source))}


_lib = None


def load():
    """Load libpfsf.so; raises if it is missing (build it with pfsf-core_b200/build.py)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"libpfsf.so not built at {LIB_PATH}; run pfsf-core_b200/build.py")
    L = C.CDLL(LIB_PATH)
    E = C.c_void_p
    sig = {
        "pfsf_create": ([C.POINTER(Config)], E),
        "pfsf_create_with_vulkan": ([C.POINTER(Config), C.c_void_p], E),
        "pfsf_init": ([E], C.c_int),
        "pfsf_shutdown": ([E], None),
        "pfsf_destroy": ([E], None),
        "pfsf_is_available": ([E], C.c_bool),
        "pfsf_get_stats": ([E, C.POINTER(Stats)], C.c_int),
        "pfsf_set_pcg_enabled": ([E, C.c_int], None),
        "pfsf_set_wind": ([E, C.POINTER(Vec3)], None),
        "pfsf_add_island": ([E, C.POINTER(IslandDesc)], C.c_int),
        "pfsf_remove_island": ([E, C.c_int32], None),
        "pfsf_notify_block_change": ([E, C.c_int32, C.POINTER(VoxelUpdate)], C.c_int),
        "pfsf_mark_full_rebuild": ([E, C.c_int32], None),
        "pfsf_tick": ([E, C.POINTER(C.c_int32), C.c_int32, C.c_int64, C.POINTER(TickResult)], C.c_int),
        "pfsf_read_stress": ([E, C.c_int32, C.c_void_p, C.c_int32, C.POINTER(C.c_int32)], C.c_int),
        "pfsf_register_island_buffers": ([E, C.c_int32, C.POINTER(IslandBuffers)], C.c_int),
        "pfsf_register_island_lookups": ([E, C.c_int32, C.POINTER(IslandLookups)], C.c_int),
        "pfsf_register_stress_readback": ([E, C.c_int32, C.c_void_p, C.c_int64], C.c_int),
        "pfsf_tick_dbb": ([E, C.POINTER(C.c_int32), C.c_int32, C.c_int64, C.c_void_p, C.c_int64], C.c_int),
        "pfsf_drain_callbacks": ([E, C.c_void_p, C.c_int32], C.c_int32),
        "pfsf_get_sparse_upload_buffer": ([E, C.c_int32, C.POINTER(C.c_void_p), C.POINTER(C.c_int64)], C.c_int),
        "pfsf_notify_sparse_updates": ([E, C.c_int32, C.c_int32], C.c_int),
        "pfsf_version": ([], C.c_char_p),
        "pfsf_register_island_kappa": ([E, C.c_int32, C.POINTER(KappaBuffers)], C.c_int),
        "pfsf_set_precision_mode": ([E, C.c_int], None),
        "pfsf_set_solve_mode": ([E, C.c_int], None),
        "pfsf_solve_to_tolerance": ([E, C.POINTER(C.c_int32), C.c_int32, C.c_double, C.c_int32, C.c_uint32,
                                     C.POINTER(SolveStats)], C.c_int),
        "pfsf_read_solution64": ([E, C.c_int32, C.c_void_p, C.c_int64, C.POINTER(C.c_int64)], C.c_int),
        "pfsf_island_solve_report": ([E, C.c_int32, C.c_void_p], C.c_int),
        "pfsf_tick_tolerance": ([E, C.POINTER(C.c_int32), C.c_int32, C.c_int64, C.c_void_p, C.c_int64, C.c_double,
                                 C.c_int32, C.POINTER(SolveStats)], C.c_int),
        "pfsf_label_components": ([E, C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_int32,
                                   C.POINTER(C.c_int32), C.POINTER(C.c_int32)], C.c_int),
        "pfsf_register_island_adjoint": ([E, C.c_int32, C.POINTER(AdjointBuffers)], C.c_int),
        "pfsf_adjoint_to_tolerance": ([E, C.POINTER(C.c_int32), C.c_int32, C.c_double, C.c_int32, C.c_uint32,
                                       C.POINTER(SolveStats)], C.c_int),
        "pfsf_debug_read_field": ([E, C.c_int32, C.c_int32, C.c_void_p, C.c_int64, C.POINTER(C.c_int64)], C.c_int),
        "pfsf_compact_failures_noalloc": ([C.c_void_p, C.c_int32, C.c_int32, C.c_int32, Pos, C.c_void_p, C.c_int32,
                                           C.c_void_p, C.c_void_p], C.c_int),
        "pfsf_debug_rcp64": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64], C.c_int),
        "pfsf_last_tick_report": ([E, C.POINTER(TickReport)], C.c_int),
        "pfsf_island_phi_max": ([E, C.c_int32, C.POINTER(C.c_float)], C.c_int),
        "pfsf_get_tuning": ([E, C.POINTER(Tuning)], C.c_int),
        "pfsf_set_mg_cycle": ([E, C.c_int], None),
        "pfsf_set_amg": ([E, C.c_int32], None),
        "pfsf_debug_time_pass": ([E, C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_float), C.POINTER(C.c_double)],
                                 C.c_int),
        "pfsf_set_tuning": ([E, C.POINTER(Tuning)], C.c_int),
        "pfsf_get_stream": ([E], C.c_void_p),
        "pfsf_kernel_launch_count": ([E], C.c_int64),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _lib = L
    return L


def default_config(max_island_size=50000, tick_budget_ms=8, vram=512 << 20, phase_field=True, multigrid=True):
    return Config(max_island_size, tick_budget_ms, vram, phase_field, multigrid)


def _ptr(a):
    return C.c_void_p(a.ctypes.data)


class Engine:
    """Thin owner of a pfsf_engine handle (mirrors NativePFSFBridge's calls)."""

    def __init__(self, config: Config | None = None):
        self.L = load()
        self.h = self.L.pfsf_create(C.byref(config) if config is not None else None)
        if not self.h:
            raise RuntimeError("pfsf_create failed")
        self._keep = {}

    def init(self):
        return self.L.pfsf_init(self.h)

    def close(self):
        if self.h:
            self.L.pfsf_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_island(self, iid, dims, origin=(0, 0, 0)):
        d = IslandDesc(iid, Pos(*origin), *dims)
        return self.L.pfsf_add_island(self.h, C.byref(d))

    def register_buffers(self, iid, phi, source, cond, vtype, rcomp, rtens, max_phi):
        arrs = [phi, source, cond, vtype, rcomp, rtens, max_phi]
        b = IslandBuffers(*[v for a in arrs for v in (_ptr(a), a.nbytes)])
        self._keep[("buf", iid)] = arrs
        return self.L.pfsf_register_island_buffers(self.h, iid, C.byref(b))

    def register_lookups(self, iid, material, anchor_bitmap, fluid, curing):
        arrs = [material, anchor_bitmap, fluid, curing]
        b = IslandLookups(*[v for a in arrs for v in (_ptr(a), a.nbytes)])
        self._keep[("lk", iid)] = arrs
        return self.L.pfsf_register_island_lookups(self.h, iid, C.byref(b))

    def register_stress(self, iid, out):
        self._keep[("st", iid)] = out
        return self.L.pfsf_register_stress_readback(self.h, iid, _ptr(out), out.nbytes)

    def tick_dbb(self, ids, failure_buf=None, epoch=0):
        ids = np.ascontiguousarray(ids, np.int32)
        if failure_buf is None:
            return self.L.pfsf_tick_dbb(self.h, ids.ctypes.data_as(C.POINTER(C.c_int32)), ids.size, epoch, None, 0)
        return self.L.pfsf_tick_dbb(self.h, ids.ctypes.data_as(C.POINTER(C.c_int32)), ids.size, epoch,
                                    _ptr(failure_buf), failure_buf.nbytes)

    def register_kappa(self, iid, phi, source, kappa, vtype):
        arrs = [phi, source, kappa, vtype]
        b = KappaBuffers(*[v for a in arrs for v in (_ptr(a), a.nbytes)])
        self._keep[("k", iid)] = arrs
        return self.L.pfsf_register_island_kappa(self.h, iid, C.byref(b))

    def solve(self, ids, tol=1e-6, max_iter=500, flags=0):
        ids = np.ascontiguousarray(ids, np.int32)
        st = SolveStats()
        rc = self.L.pfsf_solve_to_tolerance(self.h, ids.ctypes.data_as(C.POINTER(C.c_int32)), ids.size, tol,
                                            max_iter, flags, C.byref(st))
        return rc, st

    def tick_tolerance(self, ids, failure_buf=None, tol=1e-6, max_iter=500, epoch=0):
        """pfsf_tick_tolerance: tolerance solve + the reference tick's tail."""
        ids = np.ascontiguousarray(ids, np.int32)
        st = SolveStats()
        rc = self.L.pfsf_tick_tolerance(self.h, ids.ctypes.data_as(C.POINTER(C.c_int32)), ids.size, epoch,
                                        None if failure_buf is None else _ptr(failure_buf),
                                        0 if failure_buf is None else failure_buf.nbytes, tol, max_iter,
                                        C.byref(st))
        return rc, st

    def label_components(self, vtype, dims, capacity=64, labels=True):
        """26-connected components of the non-air voxels on the GPU:
        (rc, labels uint32 [N] or None, components uint32 [count, 12], count, overflow)."""
        vt = np.ascontiguousarray(vtype, np.uint8)
        lab = np.zeros(int(np.prod(dims)), np.uint32) if labels else None
        comps = np.zeros((max(capacity, 1), 12), np.uint32)
        cnt, ovf = C.c_int32(0), C.c_int32(0)
        rc = self.L.pfsf_label_components(self.h, _ptr(vt), *dims, None if lab is None else _ptr(lab), _ptr(comps),
                                          capacity, C.byref(cnt), C.byref(ovf))
        return rc, lab, comps[: cnt.value], cnt.value, ovf.value

    def register_adjoint(self, iid, grad_phi, grad_source, grad_kappa):
        arrs = [grad_phi, grad_source, grad_kappa]
        for a in arrs:
            assert a.dtype == np.float32 and a.flags.c_contiguous
        b = AdjointBuffers(*[v for a in arrs for v in (_ptr(a), a.nbytes)])
        self._keep[("a", iid)] = arrs
        return self.L.pfsf_register_island_adjoint(self.h, iid, C.byref(b))

    def adjoint(self, ids, tol=1e-6, max_iter=500, flags=0):
        """dL/ds and dL/dkappa into the registered adjoint arrays, from the
        registered dL/dphi, through the last solve of the same island set."""
        ids = np.ascontiguousarray(ids, np.int32)
        st = SolveStats()
        rc = self.L.pfsf_adjoint_to_tolerance(self.h, ids.ctypes.data_as(C.POINTER(C.c_int32)), ids.size, tol,
                                              max_iter, flags, C.byref(st))
        return rc, st

    def island_report(self, iid):
        r = IslandReport()
        rc = self.L.pfsf_island_solve_report(self.h, iid, C.byref(r))
        return rc, r

    def tick_report(self):
        """pfsf_last_tick_report: (rc, TickReport) of the last reference tick or tolerance-tick tail."""
        r = TickReport()
        rc = self.L.pfsf_last_tick_report(self.h, C.byref(r))
        return rc, r

    def tuning(self):
        t = Tuning()
        t.struct_bytes = C.sizeof(Tuning)
        rc = self.L.pfsf_get_tuning(self.h, C.byref(t))
        return rc, t

    def set_tuning(self, **kw):
        """pfsf_set_tuning with the current values updated by kw."""
        rc, t = self.tuning()
        for k, v in kw.items():
            setattr(t, k, float(v) if k in ("cheb_lower", "coarse_weight", "inner_eta") else int(v))
        t.struct_bytes = C.sizeof(Tuning)
        return self.L.pfsf_set_tuning(self.h, C.byref(t))

    def phi_max(self, iid):
        """pfsf_island_phi_max: (rc, max phi of the island's last tick)."""
        v = C.c_float(0.0)
        rc = self.L.pfsf_island_phi_max(self.h, iid, C.byref(v))
        return rc, v.value

    def read_solution64(self, iid, n):
        out = np.zeros(n, np.float64)
        cnt = C.c_int64(0)
        rc = self.L.pfsf_read_solution64(self.h, iid, _ptr(out), n, C.byref(cnt))
        return rc, out[:cnt.value]

    def read_stress(self, iid, n):
        out = np.zeros(n, np.float32)
        cnt = C.c_int32(0)
        rc = self.L.pfsf_read_stress(self.h, iid, _ptr(out), n, C.byref(cnt))
        return rc, out[:cnt.value]

    FIELD_DTYPES = {0: np.float32, 1: np.float32, 2: np.float32, 3: np.uint8, 4: np.uint32, 6: np.float32,
                    7: np.float32, 8: np.uint8, 9: np.float32, 10: np.float32, 11: np.float32, 12: np.int32,
                    13: np.float32, 14: np.float32}

    def debug_field(self, iid, field):
        """Tick-state array of an island (0 phi, 1 H, 2 d, 3 fail, 4 macro bits,
        6 source, 7 face conductivity SoA-6, 8 type, 9 max_phi, 10 rcomp,
        11 rtens, 12 aggregates, 13 aggregation weights, 14 coarse diagonal)
        or the schedule state dict (field 5)."""
        size = C.c_int64(0)
        tmp = np.zeros(32, np.uint8)
        rc = self.L.pfsf_debug_read_field(self.h, iid, field, _ptr(tmp), 0, C.byref(size))
        if rc != PFSF_OK:
            raise RuntimeError(f"pfsf_debug_read_field rc={rc}")
        if field == 5:
            rc = self.L.pfsf_debug_read_field(self.h, iid, field, _ptr(tmp), 20, C.byref(size))
            iv = tmp[:12].view(np.int32)
            fv = tmp[12:20].view(np.float32)
            return {"chebyshev_iter": int(iv[0]), "pcg_allocated": int(iv[1]), "mg_allocated": int(iv[2]),
                    "prev_macro": float(fv[0]), "last_macro": float(fv[1])}
        dt = self.FIELD_DTYPES[field]
        out = np.zeros(size.value // np.dtype(dt).itemsize, dt)
        rc = self.L.pfsf_debug_read_field(self.h, iid, field, _ptr(out), out.nbytes, C.byref(size))
        if rc != PFSF_OK:
            raise RuntimeError(f"pfsf_debug_read_field rc={rc}")
        return out

    def stats(self):
        s = Stats()
        rc = self.L.pfsf_get_stats(self.h, C.byref(s))
        return rc, s

    def set_precision(self, p):
        self.L.pfsf_set_precision_mode(self.h, p)

    def set_solve_mode(self, m):
        self.L.pfsf_set_solve_mode(self.h, m)

    def time_pass(self, iid, pass_, reps=10):
        """pfsf_debug_time_pass: (rc, ms per pass, algorithmic bytes per pass)."""
        ms, b = C.c_float(0.0), C.c_double(0.0)
        rc = self.L.pfsf_debug_time_pass(self.h, iid, pass_, reps, C.byref(ms), C.byref(b))
        return rc, ms.value, b.value

    def set_mg_cycle(self, cycle):
        """MG_V (0) or MG_W (1) for the batched tolerance solve's preconditioner."""
        self.L.pfsf_set_mg_cycle(self.h, int(cycle))

    def set_amg(self, on):
        """Aggregation correction at every PCG start of the reference tick."""
        self.L.pfsf_set_amg(self.h, int(bool(on)))

    def set_pcg_enabled(self, on):
        self.L.pfsf_set_pcg_enabled(self.h, int(bool(on)))

    def stream(self):
        return self.L.pfsf_get_stream(self.h)

    def launches(self):
        return self.L.pfsf_kernel_launch_count(self.h)
