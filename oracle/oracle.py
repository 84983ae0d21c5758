"""ctypes front-end of the CPU oracle (``liboracle.so`` built from pfsf_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py``.  The product library never imports it.

Each wrapper names the reference shader or host routine it restates (paths
relative to the PFSF-CORE checkout, SH = .../shaders/compute/pfsf).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

F32P = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
F64P = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
U8P = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
U32P = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
I32P = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def build() -> str:
    """Compile liboracle.so with the committed Makefile (gcc, FP contraction off)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        srcs = [os.path.join(_HERE, f) for f in ("pfsf_oracle.c", "kappa_mg.c", "kappa_mg_impl.h", "Makefile")]
        if not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < max(os.path.getmtime(f) for f in srcs):
            build()
        L = C.CDLL(_LIB_PATH)
        i = C.c_int
        L.o_rbgs_color.argtypes = [i, i, i, F32P, F32P, F32P, U8P, F32P, U32P, i, C.c_float]
        L.o_rbgs_step.argtypes = [i, i, i, F32P, F32P, F32P, U8P, F32P, U32P, C.c_float]
        L.o_jacobi_coarse.argtypes = [i, i, i, F32P, F32P, F32P, F32P, U8P, F32P, C.c_float]
        L.o_restrict.argtypes = [i, i, i, F32P, F32P, F32P, U8P, i, i, i, F32P, F32P]
        L.o_prolong.argtypes = [i, i, i, F32P, i, i, i, F32P]
        L.o_downsample.argtypes = [i, i, i, F32P, U8P, i, i, i, F32P, U8P]
        L.o_pcg_precompute.argtypes = [i, i, i, F32P, F32P]
        L.o_pcg_matvec.argtypes = [i, i, i, F32P, F32P, F32P, U8P]
        L.o_pcg_update.argtypes = [i, i, i, F32P, F32P, F32P, F32P, F32P, F32P, U8P, F32P, F32P, F32P, i]
        L.o_pcg_update.restype = C.c_double
        L.o_pcg_direction.argtypes = [i, i, i, F32P, F32P, U8P, F32P, F32P]
        L.o_rtz_limit.argtypes = [C.c_int64]
        L.o_rtz_limit.restype = C.c_int64
        L.o_phase_field.argtypes = [i, i, i, F32P, F32P, F32P, F32P, U8P, U32P, F32P, C.c_float, C.c_float,
                                    C.c_float, i]
        L.o_failure_scan.argtypes = [i, i, i, F32P, F32P, F32P, F32P, U8P, U32P, F32P, U32P, F32P, C.c_float]
        L.pfo_create.argtypes = [i, i, i]
        L.pfo_create.restype = C.c_void_p
        L.pfo_destroy.argtypes = [C.c_void_p]
        L.pfo_ptr.argtypes = [C.c_void_p, i]
        L.pfo_ptr.restype = C.c_void_p
        L.pfo_get_state.argtypes = [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_float)]
        L.pfo_set_flags.argtypes = [C.c_void_p, i, i]
        L.pfo_set_amg.argtypes = [C.c_void_p, i]
        L.o_amg_build.argtypes = [i, i, i, F32P, U8P, I32P, F32P, F32P]
        L.o_amg_build.restype = C.c_int64
        L.o_amg_correct.argtypes = [i, i, i, I32P, F32P, F32P, F32P, F32P, F32P]
        L.o_tick.argtypes = [C.c_void_p]
        L.o_solve_steps.argtypes = [C.c_void_p, i]
        L.o_solve_steps.restype = i
        L.o_readback_failures.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_int64]
        L.o_readback_failures.restype = C.c_int32
        L.o_kappa_apply.argtypes = [i, i, i, F64P, U8P, F64P, F64P]
        L.o_kappa_pcg64.argtypes = [i, i, i, F64P, U8P, F64P, F64P, C.c_double, i, C.POINTER(C.c_double)]
        L.o_kappa_pcg64.restype = i
        L.o_kappa_mgpcg64.argtypes = [i, i, i, F64P, U8P, F64P, F64P, C.c_double, i, i, C.POINTER(C.c_double)]
        L.o_kappa_mgpcg64.restype = i
        L.o_kappa_mgpcg32.argtypes = [i, i, i, F64P, U8P, F64P, F64P, C.c_double, i, i, C.POINTER(C.c_double),
                                      C.POINTER(C.c_int)]
        L.o_kappa_mgpcg32.restype = i
        L.o_kappa_relres.argtypes = [i, i, i, F64P, U8P, F64P, F32P]
        L.o_kappa_relres.restype = C.c_double
        L.o_history.argtypes = [i, i, i, F32P, F32P, U8P, F32P]
        L.o_label_components.argtypes = [i, i, i, U8P, U32P, U32P, i]
        L.o_label_components.restype = C.c_int64
        _lib = L
    return _lib


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


# ---------------------------------------------------------------- kernels
def rbgs_color(dims, phi, rho, sigma, vtype, H, macro, color, damping):
    """SH/rbgs_smooth.comp.glsl:73-211 (one colour pass, in place on phi/H)."""
    lx, ly, lz = dims
    lib().o_rbgs_color(lx, ly, lz, phi, _c(rho, np.float32), _c(sigma, np.float32), _c(vtype, np.uint8), H,
                       _c(macro, np.uint32), int(color), float(damping))


def rbgs_step(dims, phi, rho, sigma, vtype, H, macro, damping):
    lx, ly, lz = dims
    lib().o_rbgs_step(lx, ly, lz, phi, _c(rho, np.float32), _c(sigma, np.float32), _c(vtype, np.uint8), H,
                      _c(macro, np.uint32), float(damping))


def jacobi_coarse(dims, phi, phi_prev, rho, sigma, vtype, Hfine, damping):
    """SH/jacobi_smooth.comp.glsl:60-227 with omega=1, reading a pre-pass snapshot."""
    lx, ly, lz = dims
    lib().o_jacobi_coarse(lx, ly, lz, phi, _c(phi_prev, np.float32), _c(rho, np.float32),
                          _c(sigma, np.float32), _c(vtype, np.uint8), Hfine, float(damping))


def restrict(fdims, phi_f, rho_f, sig_f, type_f, cdims, phi_c, rho_c):
    """SH/mg_restrict.comp.glsl:118-195."""
    lib().o_restrict(*fdims, _c(phi_f, np.float32), _c(rho_f, np.float32), _c(sig_f, np.float32),
                     _c(type_f, np.uint8), *cdims, phi_c, rho_c)


def prolong(fdims, phi_f, cdims, phi_c):
    """SH/mg_prolong.comp.glsl:233-275 (adds into phi_f)."""
    lib().o_prolong(*fdims, phi_f, *cdims, _c(phi_c, np.float32))


def downsample(sdims, cond, vtype, ddims):
    """L1-native/libpfsf/src/core/island_buffer.cpp:600-700 (downsampleLevel)."""
    dn = int(np.prod(ddims))
    oc = np.zeros(6 * dn, np.float32)
    ot = np.zeros(dn, np.uint8)
    lib().o_downsample(*sdims, _c(cond, np.float32), _c(vtype, np.uint8), *ddims, oc, ot)
    return oc, ot


def pcg_precompute(dims, sigma):
    n = int(np.prod(dims))
    out = np.zeros(n, np.float32)
    lib().o_pcg_precompute(*dims, _c(sigma, np.float32), out)
    return out


def pcg_matvec(dims, x, sigma, vtype):
    n = int(np.prod(dims))
    out = np.zeros(n, np.float32)
    lib().o_pcg_matvec(*dims, _c(x, np.float32), out, _c(sigma, np.float32), _c(vtype, np.uint8))
    return out


def pcg_update(dims, phi, r, r_prev, p, ap, src, vtype, sigma, invdiag, red, is_init):
    return lib().o_pcg_update(*dims, phi, r, _c(r_prev, np.float32), p, _c(ap, np.float32), _c(src, np.float32),
                              _c(vtype, np.uint8), _c(sigma, np.float32), _c(invdiag, np.float32),
                              _c(red, np.float32), int(is_init))


def pcg_direction(dims, r, p, vtype, red, sigma):
    lib().o_pcg_direction(*dims, _c(r, np.float32), p, _c(vtype, np.uint8), _c(red, np.float32),
                          _c(sigma, np.float32))


def rtz_limit(n):
    return int(lib().o_rtz_limit(int(n)))


def phase_field(dims, phi, H, D, sigma, vtype, fail, hyd, l0=2.0, gc=100.0, relax=0.3, split=1):
    lib().o_phase_field(*dims, _c(phi, np.float32), _c(H, np.float32), D, _c(sigma, np.float32),
                        _c(vtype, np.uint8), fail, _c(hyd, np.float32), l0, gc, relax, split)


def failure_scan(dims, phi, sigma, maxphi, rcomp, vtype, fail, rtens, macro, rho, phi_orphan=1e6):
    lib().o_failure_scan(*dims, _c(phi, np.float32), _c(sigma, np.float32), _c(maxphi, np.float32),
                         _c(rcomp, np.float32), _c(vtype, np.uint8), fail, _c(rtens, np.float32), macro,
                         _c(rho, np.float32), phi_orphan)


def history(dims, phi, sigma, vtype, H):
    lib().o_history(*dims, _c(phi, np.float32), _c(sigma, np.float32), _c(vtype, np.uint8), H)


def tolerance_tick_tail(dims, phi32, case, H, D, fail):
    """The tail of the tolerance tick on a given FP32 phi: history update,
    phase field (D snapshot), failure scan -- in place on H, D, fail.
    `case` holds the reference-layout inputs (conductivity, type, rcomp,
    rtens, max_phi, hydration, source).  Returns the macro residual array."""
    n = int(np.prod(dims))
    history(dims, phi32, case["conductivity"], case["type"], H)
    phase_field(dims, phi32, H, D, case["conductivity"], case["type"], fail, case["hydration"])
    mb = [(v + 7) // 8 for v in dims]
    macro = np.full(mb[0] * mb[1] * mb[2], 0x38D1B717, np.uint32)
    failure_scan(dims, phi32, case["conductivity"], case["max_phi"], case["rcomp"], case["type"], fail,
                 case["rtens"], macro, case["source"])
    assert fail.size == n
    return macro


def amg_build(dims, sigma, vtype):
    """NP/src/solver/amg_builder.cpp:9-63 -> (aggregation int32[n],
    weights float32[n], coarse diagonal float32[nc])."""
    lx, ly, lz = dims
    n = lx * ly * lz
    nc = ((lx + 1) // 2) * ((ly + 1) // 2) * ((lz + 1) // 2)
    agg = np.zeros(n, np.int32)
    w = np.zeros(n, np.float32)
    dc = np.zeros(max(nc, 1), np.float32)
    lib().o_amg_build(lx, ly, lz, _c(sigma, np.float32), _c(vtype, np.uint8), agg, w, dc)
    return agg, w, dc[:nc]


def amg_correct(dims, agg, w, dc, r, phi):
    """NP/src/solver/dispatcher_amg.cpp:83-161: phi += P D_c^-1 P^T r (in place on phi)."""
    lx, ly, lz = dims
    nc = ((lx + 1) // 2) * ((ly + 1) // 2) * ((lz + 1) // 2)
    ec = np.zeros(max(nc, 1), np.float32)
    lib().o_amg_correct(lx, ly, lz, _c(agg, np.int32), _c(w, np.float32), _c(np.resize(dc, max(nc, 1)), np.float32),
                        _c(r, np.float32), phi, ec)


# ---------------------------------------------------------------- island state
class Island:
    """One island with the native engine's per-island device state
    (L1-native/libpfsf/src/core/island_buffer.h), held on the host."""

    FIELDS = {"phi": (0, np.float32, 1), "source": (1, np.float32, 1), "conductivity": (2, np.float32, 6),
              "type": (3, np.uint8, 1), "rcomp": (4, np.float32, 1), "rtens": (5, np.float32, 1),
              "max_phi": (6, np.float32, 1), "hydration": (7, np.float32, 1), "H": (8, np.float32, 1),
              "D": (9, np.float32, 1), "fail": (10, np.uint32, 1)}

    def __init__(self, lx, ly, lz, pcg_enabled=True, phase_field=True, amg=False):
        self.dims = (int(lx), int(ly), int(lz))
        self.n = lx * ly * lz
        self._h = lib().pfo_create(lx, ly, lz)
        lib().pfo_set_flags(self._h, int(pcg_enabled), int(phase_field))
        lib().pfo_set_amg(self._h, int(amg))
        self.nmb = ((lx + 7) // 8) * ((ly + 7) // 8) * ((lz + 7) // 8)

    def __del__(self):
        if getattr(self, "_h", None):
            lib().pfo_destroy(self._h)
            self._h = None

    def view(self, name):
        idx, dt, mult = self.FIELDS[name]
        ptr = lib().pfo_ptr(self._h, idx)
        n = self.n * mult
        buf = (C.c_byte * (n * np.dtype(dt).itemsize)).from_address(ptr)
        return np.frombuffer(buf, dtype=dt, count=n)

    def macro(self):
        ptr = lib().pfo_ptr(self._h, 11)
        buf = (C.c_byte * (self.nmb * 4)).from_address(ptr)
        return np.frombuffer(buf, dtype=np.uint32, count=self.nmb)

    def load(self, **arrays):
        for k, v in arrays.items():
            self.view(k)[:] = np.asarray(v).reshape(-1)

    def state(self):
        iv = (C.c_int32 * 3)()
        fv = (C.c_float * 2)()
        lib().pfo_get_state(self._h, iv, fv)
        return {"chebyshev_iter": iv[0], "pcg_allocated": iv[1], "mg_allocated": iv[2],
                "prev_macro": fv[0], "last_macro": fv[1]}

    def tick(self):
        """One dirty-island tick (L1-native/libpfsf/src/pfsf_engine.cpp:470-513)."""
        lib().o_tick(self._h)

    def failures(self, origin, capacity=1024, dbb=None):
        """Failure DBB {count}{x,y,z,type}*k (island_buffer.cpp:864-966)."""
        if dbb is None:
            dbb = np.zeros(1 + 4 * capacity, np.int32)
        lib().o_readback_failures(self._h, int(origin[0]), int(origin[1]), int(origin[2]),
                                  dbb.ctypes.data, dbb.nbytes)
        return dbb


# ---------------------------------------------------------------- kappa operator
def kappa_apply(dims, kappa, vtype, x):
    n = int(np.prod(dims))
    y = np.zeros(n, np.float64)
    lib().o_kappa_apply(*dims, _c(kappa, np.float64), _c(vtype, np.uint8), _c(x, np.float64), y)
    return y


def kappa_solve64(dims, kappa, vtype, source, tol=1e-12, maxit=20000, x0=None):
    """FP64 Jacobi-PCG on the symmetric harmonic-mean 26-point operator."""
    n = int(np.prod(dims))
    x = np.zeros(n, np.float64) if x0 is None else np.array(x0, np.float64)
    rr = C.c_double(0.0)
    it = lib().o_kappa_pcg64(*dims, _c(kappa, np.float64), _c(vtype, np.uint8), _c(source, np.float64), x,
                             float(tol), int(maxit), C.byref(rr))
    return x, it, rr.value


def kappa_mgpcg64(dims, kappa, vtype, source, tol=1e-12, maxit=2000, threads=1, x0=None):
    """FP64 multigrid-preconditioned CG (oracle/kappa_mg.c) on the same
    operator: the FP64 reference solution of large islands in seconds to
    minutes on the host's threads.  Returns (x, iterations, relres)."""
    n = int(np.prod(dims))
    x = np.zeros(n, np.float64) if x0 is None else np.array(x0, np.float64)
    rr = C.c_double(0.0)
    it = lib().o_kappa_mgpcg64(*dims, _c(kappa, np.float64), _c(vtype, np.uint8), _c(source, np.float64), x,
                               float(tol), int(maxit), int(threads), C.byref(rr))
    return x, it, rr.value


def kappa_mgpcg32(dims, kappa, vtype, source, tol=1e-6, maxit=2000, threads=1, x0=None):
    """The plain FP32 scheme on the CPU (oracle/kappa_mg.c): FP32 V-cycle PCG
    inside FP64 residual refinement.  Returns (x, inner iterations, relres,
    outer refinements)."""
    n = int(np.prod(dims))
    x = np.zeros(n, np.float64) if x0 is None else np.array(x0, np.float64)
    rr = C.c_double(0.0)
    outer = C.c_int(0)
    it = lib().o_kappa_mgpcg32(*dims, _c(kappa, np.float64), _c(vtype, np.uint8), _c(source, np.float64), x,
                               float(tol), int(maxit), int(threads), C.byref(rr), C.byref(outer))
    return x, it, rr.value, outer.value


def kappa_relres(dims, kappa, vtype, source, phi32):
    return lib().o_kappa_relres(*dims, _c(kappa, np.float64), _c(vtype, np.uint8), _c(source, np.float64),
                                _c(phi32, np.float32))


# ------------------------------------------------------- adjoint (FP64, numpy)
# The reference has no gradient code; these restate the calculus of the
# kappa operator above in FP64 so the device adjoint and the torch tooling
# can be checked against it (and it against finite differences).

def _dirs13():
    """The 13 link directions counted once: offsets (dx, dy, dz) after the
    centre in z-major order, with the operator's group scale c."""
    out = []
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                if (dz, dy, dx) > (0, 0, 0):
                    m = abs(dx) + abs(dy) + abs(dz)
                    out.append((dx, dy, dz, {1: 1.0, 2: 0.5, 3: 1.0 / 6.0}[m]))
    return out


def _pair_slices(d, n):
    if d == 0:
        return slice(0, n), slice(0, n)
    if d == 1:
        return slice(0, n - 1), slice(1, n)
    return slice(1, n), slice(0, n - 1)


def _links(dims):
    """(si, sj, c) per direction: 3-D slices of the voxels i and their
    neighbours j = i + offset, arrays shaped (lz, ly, lx)."""
    lx, ly, lz = dims
    for dx, dy, dz, c in _dirs13():
        zi, zj = _pair_slices(dz, lz)
        yi, yj = _pair_slices(dy, ly)
        xi, xj = _pair_slices(dx, lx)
        yield (zi, yi, xi), (zj, yj, xj), c


def _grid(a, dims):
    lx, ly, lz = dims
    return np.asarray(a, np.float64).reshape(lz, ly, lx)


def kappa_edge_product(dims, kappa, vtype, phi, lam):
    """-sum_j dw_ij/dk_i (lam_i - lam_j)(phi_i - phi_j) per voxel (FP64);
    lam = phi = 0 off the solid voxels; 0 on air."""
    k = _grid(kappa, dims)
    t = np.asarray(vtype).reshape(k.shape)
    solid = t == 1
    P = np.where(solid, _grid(phi, dims), 0.0)
    Lm = np.where(solid, _grid(lam, dims), 0.0)
    g = np.zeros_like(k)
    for si, sj, c in _links(dims):
        ki, kj = k[si], k[sj]
        both = (t[si] != 0) & (t[sj] != 0) & ((ki + kj) > 0)
        s = np.where(both, ki + kj, 1.0)
        prod = (Lm[si] - Lm[sj]) * (P[si] - P[sj])
        g[si] -= np.where(both, 2.0 * c * kj * kj / (s * s) * prod, 0.0)
        g[sj] -= np.where(both, 2.0 * c * ki * ki / (s * s) * prod, 0.0)
    g[t == 0] = 0.0
    return g.reshape(-1)


def kappa_adjoint64(dims, kappa, vtype, phi, grad_phi, tol=1e-13):
    """dL/ds, dL/dkappa for dL/dphi = grad_phi through A(kappa) phi = s:
    lambda = A^-1 grad_phi (A symmetric), dL/ds = lambda on solid voxels,
    dL/dkappa = the edge product."""
    g = np.where(np.asarray(vtype) == 1, np.asarray(grad_phi, np.float64), 0.0)
    lam, _, rr = kappa_solve64(dims, np.asarray(kappa, np.float64), vtype, g, tol=tol, maxit=400000)
    gs = np.where(np.asarray(vtype) == 1, lam, 0.0)
    return gs, kappa_edge_product(dims, kappa, vtype, phi, lam), rr


def flux_loss64(dims, kappa, vtype, phi, rcomp, phi_target):
    """L = sum_solid softplus(flux_in_i / rcomp_i - 1) + 1/2 sum_solid (phi_i - phi_target_i)^2
    with flux_in_i = sum_j w_ij max(phi_j - phi_i, 0) over the operator's links
    (the failure scan's compressive inflow, SH/failure_scan.comp.glsl:89-158,
    on the kappa link weights).  Returns (L, dL/dphi, direct dL/dkappa)."""
    k = _grid(kappa, dims)
    t = np.asarray(vtype).reshape(k.shape)
    solid = t == 1
    P = np.where(solid, _grid(phi, dims), 0.0)
    rc = _grid(rcomp, dims)
    links = []
    flux = np.zeros_like(k)
    for si, sj, c in _links(dims):
        ki, kj = k[si], k[sj]
        both = (t[si] != 0) & (t[sj] != 0) & ((ki + kj) > 0)
        s = np.where(both, ki + kj, 1.0)
        w = np.where(both, 2.0 * c * ki * kj / s, 0.0)
        u = P[sj] - P[si]
        flux[si] += w * np.maximum(u, 0.0)
        flux[sj] += w * np.maximum(-u, 0.0)
        links.append((si, sj, c, w, u, s, both))
    z = np.where(solid, flux / np.where(solid, rc, 1.0) - 1.0, 0.0)
    sp = np.logaddexp(0.0, z)
    d = np.where(solid, P - _grid(phi_target, dims), 0.0)
    L = float(np.sum(np.where(solid, sp, 0.0)) + 0.5 * np.sum(d * d))
    a = np.where(solid, 1.0 / (1.0 + np.exp(-z)) / np.where(solid, rc, 1.0), 0.0)  # dL/dflux
    gphi = d.copy()
    gk = np.zeros_like(k)
    for si, sj, c, w, u, s, both in links:
        pos, neg = u > 0, u < 0
        ai, aj = a[si], a[sj]
        gphi[sj] += np.where(pos, ai * w, 0.0) - np.where(neg, aj * w, 0.0)
        gphi[si] += np.where(neg, aj * w, 0.0) - np.where(pos, ai * w, 0.0)
        dLdw = ai * np.maximum(u, 0.0) + aj * np.maximum(-u, 0.0)
        ki, kj = k[si], k[sj]
        gk[si] += np.where(both, 2.0 * c * kj * kj / (s * s) * dLdw, 0.0)
        gk[sj] += np.where(both, 2.0 * c * ki * ki / (s * s) * dLdw, 0.0)
    gphi[~solid] = 0.0
    gk[t == 0] = 0.0
    return L, gphi.reshape(-1), gk.reshape(-1)


def amor_psi64(dims, kappa, vtype, phi):
    """psi_e of the history update (SH/rbgs_smooth.comp.glsl:177-191) in FP64:
    phi^2 / 2, times 0.01 where the face inflow exceeds three times the face
    outflow (face conductivity = the harmonic-mean kappa link value); solid
    voxels with phi > 0 only.  Returns (psi, factor)."""
    k = _grid(kappa, dims)
    t = np.asarray(vtype).reshape(k.shape)
    P = np.where(t == 1, _grid(phi, dims), 0.0)
    fin = np.zeros_like(P)
    fout = np.zeros_like(P)
    lz, ly, lx = k.shape
    for dx, dy, dz in ((-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1)):
        kj = np.zeros_like(k)
        tj = np.zeros_like(t)
        pj = np.zeros_like(P)
        src, dst = [slice(None)] * 3, [slice(None)] * 3
        for ax, o in zip((2, 1, 0), (dx, dy, dz)):
            if o == 1:
                dst[ax], src[ax] = slice(0, -1), slice(1, None)
            elif o == -1:
                dst[ax], src[ax] = slice(1, None), slice(0, -1)
        kj[tuple(dst)] = k[tuple(src)]
        tj[tuple(dst)] = t[tuple(src)]
        pj[tuple(dst)] = P[tuple(src)]
        ok = (t != 0) & (tj != 0) & ((k + kj) > 0)
        sig = np.where(ok, 2.0 * k * kj / np.where(ok, k + kj, 1.0), 0.0)
        flow = sig * (pj - P)
        fin += np.maximum(flow, 0.0)
        fout += np.maximum(-flow, 0.0)
    factor = np.where(fin > 3.0 * fout, 0.01, 1.0)
    live = (t == 1) & (P > 0)
    return np.where(live, 0.5 * P * P * factor, 0.0).reshape(-1), np.where(live, factor, 0.0).reshape(-1)


def trajectory_grad64(dims, kappa, vtype, source, rcomp, phi_target, ticks, ramp, h_scale, threads=1):
    """FP64 restatement of the config-4 trajectory loss and its gradient
    dL/dkappa (the torch tooling's trajectory_loss): per tick t the FP64
    solution of A(kappa) phi_t = f_t s, the flux / target terms of
    flux_loss64 with target f_t phi_target, the history H = max_t psi_e(phi_t)
    with the softplus(H / h_scale - 1) term (its gradient reaching the tick
    that attains the max), and one FP64 adjoint solve per tick.
    Returns (L, dL/dkappa, phis, argmax tick per voxel)."""
    k = np.asarray(kappa, np.float64)
    s = np.asarray(source, np.float64)
    solid = np.asarray(vtype) == 1
    phis, L = [], 0.0
    gk = np.zeros_like(k)
    gphis = []
    H = np.zeros_like(k)
    arg = np.full(k.size, -1)
    fac = []
    for t in range(ticks):
        f = 1.0 + (ramp - 1.0) * t / max(ticks - 1, 1)
        x, _, rel = kappa_mgpcg64(dims, k, vtype, f * s, tol=1e-13, threads=threads)
        phis.append(x)
        Lt, gphi, gkd = flux_loss64(dims, k, vtype, x, rcomp, f * np.asarray(phi_target, np.float64))
        L += Lt
        gk += gkd
        gphis.append(gphi)
        psi, fa = amor_psi64(dims, k, vtype, x)
        fac.append(fa)
        upd = psi > H
        arg[upd] = t
        H = np.maximum(H, psi)
    z = H / h_scale - 1.0
    L += float(np.sum(np.where(solid, np.logaddexp(0.0, z), 0.0)))
    dH = np.where(solid, 1.0 / (1.0 + np.exp(-z)) / h_scale, 0.0)
    for t in range(ticks):
        sel = arg == t
        gphi = gphis[t] + np.where(sel, dH * phis[t] * fac[t], 0.0)
        _, gke, _ = kappa_adjoint64(dims, k, vtype, phis[t], gphi)
        gk += gke
    return L, gk, phis, arg


# ------------------------------------------------------------- island labels
NO_ISLAND = 0xFFFFFFFF


def label_components(dims, vtype, cap=64):
    """(labels uint32 [N], components uint32 [min(count, cap), 12], count):
    breadth-first 26-connected components (oracle/pfsf_oracle.c
    o_label_components)."""
    n = int(np.prod(dims))
    labels = np.zeros(n, np.uint32)
    comps = np.zeros(max(cap, 1) * 12, np.uint32)
    cnt = lib().o_label_components(*dims, _c(vtype, np.uint8), labels, comps, int(cap))
    return labels, comps.reshape(-1, 12)[: min(cnt, cap)], int(cnt)


def label_propagation(dims, vtype, max_iters=100000):
    """The reference's label propagation restated in numpy and run to its
    fixed point: init label i + 1 on solid/anchor voxels
    (SH/label_prop_init.comp.glsl:33-50), then alternate a hook pass (each
    voxel takes the smallest label among itself and its in-box 26 neighbours,
    label_prop_iterate.comp.glsl:70-93) and a jump pass (label <- label of
    voxel label - 1 when smaller, :94-104) -- synchronous, as in
    PFSFLabelPropCpuSimulator.java:115-160 -- until nothing changes.
    Returns (labels, passes)."""
    lx, ly, lz = dims
    t = np.asarray(vtype).reshape(lz, ly, lx)
    big = np.uint64(1 << 40)
    lab = np.where(t != 0, np.arange(1, lx * ly * lz + 1, dtype=np.uint64).reshape(lz, ly, lx), big)
    for it in range(max_iters):
        pad = np.pad(lab, 1, constant_values=big)
        m = lab.copy()
        for dz in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dx in (-1, 0, 1):
                    m = np.minimum(m, pad[1 + dz:1 + dz + lz, 1 + dy:1 + dy + ly, 1 + dx:1 + dx + lx])
        m = np.where(t != 0, m, big)
        flat = m.reshape(-1)
        live = flat != big
        parent = np.where(live, flat[np.where(live, flat - 1, 0).astype(np.int64)], big)
        jumped = np.where(live & (parent < flat), parent, flat).reshape(lz, ly, lx)
        if np.array_equal(jumped, lab):
            break
        lab = jumped
    out = lab.reshape(-1)
    return np.where(out == big, NO_ISLAND, out).astype(np.uint32), it + 1
