"""Input builders shared by the parity tests and the golden-vector script.

A "compat case" is the set of arrays the reference tick consumes through
pfsf_register_island_buffers: phi, source, SoA-6 conductivity, uint8 voxel
type, rcomp, rtens, max_phi (+ curing / hydration), normalised the way the
Java data builder does before handing them over
(PFSFDataBuilder.java:222-278 -> pfsf_normalize_soa6).
"""
from __future__ import annotations

import base64
import json
import math

import numpy as np

from pfsf_b200 import synth

GRAVITY = 9.81


def compat_from_kappa(isl: synth.IslandInputs, source_scale=1e-4):
    """Kappa-form synthetic island -> reference-style inputs: face sigma =
    harmonic mean of kappa, source scaled into the shader's working range,
    then the data builder's normalisation."""
    sig = synth.face_sigma_from_kappa(isl.dims, isl.vtype, isl.kappa)
    src = (isl.source * np.float32(source_scale)).astype(np.float32)
    rc = (isl.rcomp * np.float32(source_scale * 20.0)).astype(np.float32)
    rt = (isl.rtens * np.float32(source_scale * 20.0)).astype(np.float32)
    src, rc, rt, sig, _ = synth.normalize_soa6(src, rc, rt, sig)
    n = isl.n
    return {"dims": isl.dims, "phi": np.zeros(n, np.float32), "source": src, "conductivity": sig,
            "type": isl.vtype.copy(), "rcomp": rc, "rtens": rt,
            "max_phi": np.full(n, np.float32(np.inf), np.float32), "hydration": np.ones(n, np.float32)}


def compat_case(name: str):
    """Named small cases (all fit the CPU oracle in well under a second a tick)."""
    if name == "block8":
        return compat_from_kappa(synth.solid_block((8, 8, 8), seed=11))
    if name == "block16":
        return compat_from_kappa(synth.solid_block((16, 16, 16), seed=12))
    if name == "noise20":
        return compat_from_kappa(synth.noise_island((20, 18, 14), seed=13))
    if name == "slab":  # aspect 4 -> V-cycle every 2 steps
        return compat_from_kappa(synth.noise_island((32, 8, 6), seed=14, occupancy=0.8))
    if name == "rod":  # aspect 8 -> V-cycle every step + extra V-cycle
        return compat_from_kappa(synth.solid_block((4, 4, 34), seed=15))
    if name == "tiny":  # max side <= 4 -> no V-cycle
        return compat_from_kappa(synth.solid_block((3, 4, 2), seed=16))
    raise KeyError(name)


def isolated_voxel_case():
    """L16_NoSupportOrphanTest shape: one solid voxel with no live faces."""
    dims = (5, 5, 5)
    n = 125
    vt = np.zeros(n, np.uint8)
    vt[0:25] = 2  # anchor floor z=0
    centre = 2 + 5 * (2 + 5 * 3)
    vt[centre] = 1
    c = {"dims": dims, "phi": np.zeros(n, np.float32), "source": np.zeros(n, np.float32),
         "conductivity": np.zeros(6 * n, np.float32), "type": vt, "rcomp": np.ones(n, np.float32),
         "rtens": np.ones(n, np.float32), "max_phi": np.full(n, np.float32(np.inf)),
         "hydration": np.ones(n, np.float32)}
    c["source"][centre] = 0.5
    return c, centre


# ------------------------------------------------------------- reference fixtures
def load_fixture(path):
    """Schema-v1 fixture (Block Reality/api/src/test/resources/pfsf-fixtures,
    loader L1-native/libpfsf/src/example/fixture_loader.cpp) -> compat case.
    Voxel material id 0 is air; anchors from the anchor list or the
    registry's is_anchor; source = density * g; sigma from
    pfsf_compute_conductivity semantics; then normalisation."""
    d = json.load(open(path))
    lx, ly, lz = d["dims"]["lx"], d["dims"]["ly"], d["dims"]["lz"]
    n = lx * ly * lz
    mats = np.frombuffer(base64.b64decode(d["materials"]["voxels"]), dtype="<i4")[:n].copy()
    reg = {r["id"]: r for r in d["materials"]["registry"]}
    vt = np.zeros(n, np.uint8)
    src = np.zeros(n, np.float32)
    rc = np.zeros(n, np.float32)
    rt = np.zeros(n, np.float32)
    for i in range(n):
        m = int(mats[i])
        if m == 0 or m not in reg:
            continue
        r = reg[m]
        vt[i] = 2 if r.get("is_anchor", False) else 1
        src[i] = np.float32(r.get("density", 2400.0) * GRAVITY)
        rc[i] = r.get("rcomp", 30.0)
        rt[i] = r.get("rtens", 3.0)
    for a in d.get("anchors", []):
        i = a[0] + lx * (a[1] + ly * a[2])
        if vt[i] != 0:
            vt[i] = 2
    wind = d.get("wind", [0.0, 0.0, 0.0])
    cond = synth.conductivity_reference((lx, ly, lz), vt, rc, rt, wind=tuple(wind))
    src[vt != 1] = 0.0
    src, rc, rt, cond, _ = synth.normalize_soa6(src, rc, rt, cond)
    return {"dims": (lx, ly, lz), "phi": np.zeros(n, np.float32), "source": src, "conductivity": cond,
            "type": vt, "rcomp": rc, "rtens": rt, "max_phi": np.full(n, np.float32(np.inf)),
            "hydration": np.ones(n, np.float32), "name": d.get("fixture_id", "")}


def cantilever_column(L=12, q=1.0):
    """1 x 1 x L column, z = 0 anchored, unit vertical faces only: the
    discrete cantilever phi_k = q (k (L-1) - k (k-1) / 2) (README.md:208,
    phi(z) = qLz - qz^2/2 in the continuum)."""
    dims = (1, 1, L)
    n = L
    vt = np.ones(n, np.uint8)
    vt[0] = 2
    cond = np.zeros(6 * n, np.float32)
    for k in range(n):
        if k > 0:
            cond[4 * n + k] = 1.0
        if k < n - 1:
            cond[5 * n + k] = 1.0
    src = np.full(n, q, np.float32)
    src[0] = 0.0
    k = np.arange(n, dtype=np.float64)
    exact = q * (k * (L - 1) - k * (k - 1) / 2.0)
    exact[0] = 0.0
    c = {"dims": dims, "phi": np.zeros(n, np.float32), "source": src, "conductivity": cond, "type": vt,
         "rcomp": np.full(n, 1e9, np.float32), "rtens": np.full(n, 1e9, np.float32),
         "max_phi": np.full(n, np.float32(np.inf)), "hydration": np.ones(n, np.float32)}
    return c, exact
