"""Seeded synthetic islands for the structural solve (numpy / scipy.ndimage).

The reference measures on no public dataset; its configurations are described
by shape, occupancy and material mix only.  These generators produce inputs
with those shapes, sizes and value distributions:

* three materials drawn uniformly per voxel:
  concrete {E 30 GPa, rho 2400, rcomp 30, rtens 3}, steel {200, 7850, 250, 250},
  timber {11, 600, 40, 80};
* kappa proportional to E, normalised to mean 1 over non-air voxels;
* source s = rho * 9.81 * 1 m^3 (N);
* the z = 0 layer is anchored (phi = 0), out-of-box links are dropped;
* occupancy from seeded 3-D value noise (4 octaves, lattice 16) thresholded
  at a target fraction and kept to the 26-connected component that touches
  the anchor layer;
* point loads of 1e4..1e6 N (log-uniform) on 0.1 % of the top-surface voxels.

Flat index is x + Lx*(y + Ly*z) (L1-native/libpfsf/include/pfsf/pfsf_types.h
layout), arrays are returned flat in that order.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

AIR, SOLID, ANCHOR = 0, 1, 2

# (E GPa, density kg/m^3, rcomp MPa, rtens MPa)
MATERIALS = np.array([[30.0, 2400.0, 30.0, 3.0],
                      [200.0, 7850.0, 250.0, 250.0],
                      [11.0, 600.0, 40.0, 80.0]], dtype=np.float64)
GRAVITY = 9.81


@dataclass
class IslandInputs:
    dims: tuple
    vtype: np.ndarray          # uint8 [N]
    kappa: np.ndarray          # float32 [N], 0 on air
    source: np.ndarray         # float32 [N] (N units), 0 on air/anchor
    rcomp: np.ndarray          # float32 [N] (MPa)
    rtens: np.ndarray          # float32 [N] (MPa)
    material: np.ndarray       # int32 [N], -1 on air
    seed: int = 0
    meta: dict = field(default_factory=dict)

    @property
    def n(self):
        return int(np.prod(self.dims))

    @property
    def n_active(self):
        return int(np.count_nonzero(self.vtype == SOLID))


def _value_noise(dims, rng, octaves=4, lattice=16):
    """Sum of trilinearly interpolated random lattices; octave k has spacing
    lattice/2^k and amplitude 2^-k."""
    lx, ly, lz = dims
    total = np.zeros((lz, ly, lx), np.float64)
    amp = 1.0
    for k in range(octaves):
        sp = max(lattice / (2 ** k), 1.0)
        gx, gy, gz = int(math.ceil(lx / sp)) + 2, int(math.ceil(ly / sp)) + 2, int(math.ceil(lz / sp)) + 2
        lat = rng.random((gz, gy, gx))
        cx = np.arange(lx) / sp
        cy = np.arange(ly) / sp
        cz = np.arange(lz) / sp
        # separable linear interpolation along x, then y, then z
        ix = np.floor(cx).astype(np.int64); fx = cx - ix
        iy = np.floor(cy).astype(np.int64); fy = cy - iy
        iz = np.floor(cz).astype(np.int64); fz = cz - iz
        fx = fx * fx * (3 - 2 * fx); fy = fy * fy * (3 - 2 * fy); fz = fz * fz * (3 - 2 * fz)
        a = lat[:, :, ix] * (1 - fx) + lat[:, :, ix + 1] * fx
        a = a[:, iy, :] * (1 - fy)[None, :, None] + a[:, iy + 1, :] * fy[None, :, None]
        a = a[iz, :, :] * (1 - fz)[:, None, None] + a[iz + 1, :, :] * fz[:, None, None]
        total += amp * a
        amp *= 0.5
    return total


def _anchor_component(solid_zyx):
    """Keep voxels 26-connected to the solid part of the z = 0 layer."""
    from scipy import ndimage
    lab, _ = ndimage.label(solid_zyx, structure=np.ones((3, 3, 3), dtype=bool))
    keep_labels = np.unique(lab[0][lab[0] > 0])
    if keep_labels.size == 0:
        return np.zeros_like(solid_zyx)
    return np.isin(lab, keep_labels)


def _assign(dims, occ_zyx, rng, point_loads=True, load_frac=1e-3):
    lx, ly, lz = dims
    n = lx * ly * lz
    vtype = np.zeros((lz, ly, lx), np.uint8)
    vtype[occ_zyx] = SOLID
    vtype[0][occ_zyx[0]] = ANCHOR
    vtype = vtype.reshape(-1)
    mat = rng.integers(0, 3, size=n).astype(np.int32)
    mat[vtype == AIR] = -1
    solid_or_anchor = vtype != AIR
    E = np.where(solid_or_anchor, MATERIALS[np.maximum(mat, 0), 0], 0.0)
    mean_e = E[solid_or_anchor].mean() if solid_or_anchor.any() else 1.0
    kappa = (E / mean_e).astype(np.float32)
    rho = np.where(solid_or_anchor, MATERIALS[np.maximum(mat, 0), 1], 0.0)
    source = rho * GRAVITY * 1.0
    if point_loads:
        occ = occ_zyx
        above = np.zeros_like(occ)
        above[:-1] = occ[1:]
        top = (occ & ~above).reshape(-1) & (vtype == SOLID)
        idx = np.flatnonzero(top)
        k = max(1, int(round(load_frac * idx.size))) if idx.size else 0
        if k:
            pick = rng.choice(idx, size=k, replace=False)
            source[pick] += np.exp(rng.uniform(math.log(1e4), math.log(1e6), size=k))
    source[vtype != SOLID] = 0.0
    rcomp = np.where(solid_or_anchor, MATERIALS[np.maximum(mat, 0), 2], 0.0).astype(np.float32)
    rtens = np.where(solid_or_anchor, MATERIALS[np.maximum(mat, 0), 3], 0.0).astype(np.float32)
    return vtype, kappa, source.astype(np.float32), rcomp, rtens, mat


def solid_block(dims=(32, 32, 32), seed=1):
    """Fully occupied box, z = 0 anchored, no point loads (32^3 CPU-runnable case)."""
    rng = np.random.default_rng(seed)
    lx, ly, lz = dims
    occ = np.ones((lz, ly, lx), bool)
    vt, kap, src, rc, rt, mat = _assign(dims, occ, rng, point_loads=False)
    return IslandInputs(tuple(dims), vt, kap, src, rc, rt, mat, seed)


def noise_island(dims, seed, occupancy=0.6, octaves=4, lattice=16, point_loads=True):
    """Value-noise island kept to its anchored 26-connected component."""
    rng = np.random.default_rng(seed)
    noise = _value_noise(dims, rng, octaves, lattice)
    thr = np.quantile(noise, 1.0 - occupancy)
    occ = noise >= thr
    occ = _anchor_component(occ)
    vt, kap, src, rc, rt, mat = _assign(dims, occ, rng, point_loads=point_loads)
    return IslandInputs(tuple(dims), vt, kap, src, rc, rt, mat, seed, {"occupancy": occupancy})


def batch_dims(n_islands, seed, lo=8, hi=96, scale=1.0):
    """Per-axis side lengths log-uniform in [lo, hi], times a global scale
    factor (clamped to >= 2)."""
    rng = np.random.default_rng(seed)
    sides = np.exp(rng.uniform(math.log(lo), math.log(hi), size=(n_islands, 3))) * scale
    return np.maximum(np.rint(sides), 2).astype(np.int64)


def _batch_member(args):
    d, s, occupancy = args
    return noise_island(d, s, occupancy=occupancy, lattice=16, point_loads=True)


def batch(n_islands=4096, seed=7, target_active=6.0e7, occupancy=0.6, lo=8, hi=96, scale=None, workers=0):
    """Batch of islands with per-axis log-uniform side lengths in [lo, hi].
    Unscaled, that law gives ~1.8e8 grid voxels (~1e8 active) for 4096
    islands, above the stated ~60 M total, so one global side scale is
    applied (solved from the realised grid volume) to bring the ACTIVE
    total near ``target_active``.  The realised totals and the scale are
    recorded in the returned metadata.  workers > 1 generates islands in a
    spawn-started process pool (start it before any CUDA use)."""
    if scale is None:
        d0 = batch_dims(n_islands, seed, lo, hi, 1.0).astype(np.float64)
        grid = float(np.prod(d0, axis=1).sum())
        # active ~= occupancy * grid (anchored component keeps most of it)
        scale = (target_active / (occupancy * 0.93 * grid)) ** (1.0 / 3.0)
    dims = batch_dims(n_islands, seed, lo, hi, scale)
    jobs = [(tuple(int(v) for v in dims[k]), seed * 100003 + k, occupancy) for k in range(n_islands)]
    if workers and workers > 1:
        import concurrent.futures as cf
        import multiprocessing as mp
        with cf.ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
            out = list(ex.map(_batch_member, jobs, chunksize=16))
    else:
        out = [_batch_member(j) for j in jobs]
    meta = {"scale": scale, "grid_total": int(sum(i.n for i in out)),
            "active_total": int(sum(i.n_active for i in out))}
    return out, meta


# ------------------------------------------------------------------ compat inputs
def face_sigma_from_kappa(dims, vtype, kappa):
    """SoA-6 face conductivity sigma[d*N + i] = harmonic mean(kappa_i, kappa_j)
    for non-air i and face neighbour j, 0 otherwise (direction order
    -X,+X,-Y,+Y,-Z,+Z, pfsf_types.h pfsf_direction)."""
    lx, ly, lz = dims
    n = lx * ly * lz
    k = kappa.astype(np.float64).reshape(lz, ly, lx)
    t = vtype.reshape(lz, ly, lx)
    sig = np.zeros((6, lz, ly, lx), np.float64)
    offs = [(-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1)]
    for d, (dx, dy, dz) in enumerate(offs):
        kj = np.zeros_like(k)
        tj = np.zeros_like(t)
        src = [slice(None)] * 3
        dst = [slice(None)] * 3
        for ax, o in zip((2, 1, 0), (dx, dy, dz)):
            if o == -1:
                dst[ax] = slice(1, None); src[ax] = slice(0, -1)
            elif o == 1:
                dst[ax] = slice(0, -1); src[ax] = slice(1, None)
        kj[tuple(dst)] = k[tuple(src)]
        tj[tuple(dst)] = t[tuple(src)]
        ok = (t != AIR) & (tj != AIR)
        s = np.where(ok & (k + kj > 0), 2.0 * k * kj / np.where(k + kj > 0, k + kj, 1.0), 0.0)
        sig[d] = s
    return sig.reshape(6 * n).astype(np.float32)


def conductivity_reference(dims, vtype, rcomp, rtens, wind=(0.0, 0.0, 0.0), upwind_factor=0.30):
    """Face conductivity from compression/tension strength, restating
    L1-native/libpfsf/src/compute/conductivity.cpp (pfsf_compute_conductivity):
    vertical faces (+-Y) get min(rcomp); horizontal faces get
    min(rcomp) * min(1, avg(rtens) / max(min(rcomp), 1)), wind-biased."""
    lx, ly, lz = dims
    n = lx * ly * lz
    out = np.zeros(6 * n, np.float32)
    offs = [(-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1)]
    steps = {0: (-1, 0), 1: (1, 0), 4: (0, -1), 5: (0, 1)}
    ws = np.float32(1.0 + upwind_factor)
    rc = rcomp.astype(np.float32)
    rt = rtens.astype(np.float32)
    for d, (dx, dy, dz) in enumerate(offs):
        for z in range(lz):
            for y in range(ly):
                for x in range(lx):
                    i = x + lx * (y + ly * z)
                    if vtype[i] == AIR:
                        continue
                    nx, ny, nz = x + dx, y + dy, z + dz
                    if not (0 <= nx < lx and 0 <= ny < ly and 0 <= nz < lz):
                        continue
                    j = nx + lx * (ny + ly * nz)
                    if vtype[j] == AIR:
                        continue
                    base = min(rc[i], rc[j])
                    if not base > 0:
                        continue
                    if d in (2, 3):
                        out[d * n + i] = base
                        continue
                    avg = np.float32(0.5) * (rt[i] + rt[j])
                    denom = base if base > 1 else np.float32(1.0)
                    ratio = min(np.float32(avg / denom), np.float32(1.0))
                    s = np.float32(base * ratio)
                    sx, sz = steps[d]
                    dot = sx * wind[0] + sz * wind[2]
                    if dot > 0:
                        s = np.float32(s * ws)
                    elif dot < 0:
                        s = np.float32(s / ws)
                    out[d * n + i] = s if np.isfinite(s) else 0.0
    return out


def normalize_soa6(source, rcomp, rtens, cond):
    """L1-native/libpfsf/src/compute/normalize.cpp: divide source, rcomp,
    rtens and conductivity by sigma_max = max(1, max(cond)) when > 1."""
    smax = max(1.0, float(cond.max()) if cond.size else 1.0)
    if smax > 1.0:
        inv = np.float32(1.0 / np.float32(smax))
        return (source * inv).astype(np.float32), (rcomp * inv).astype(np.float32), \
            (rtens * inv).astype(np.float32), (cond * inv).astype(np.float32), smax
    return source, rcomp, rtens, cond, smax
