"""Aggregation coarse correction of the oracle, pinned to the reference.

The oracle's builder (o_amg_build, a restatement of
L1-native/libpfsf/src/solver/amg_builder.cpp:9-63) is compared bit for bit
with the reference's own buildAMG, compiled from its source by oracle/ref.mk
into oracle/_ref/libpfsf_ref_amg.so, on seeded islands with air, anchors,
zero-conductivity voxels and odd sides.  The correction (o_amg_correct,
dispatcher_amg.cpp:83-161) is checked against its algebra restated in numpy,
and the PCG start with the correction against the start without it.
"""
import ctypes as C
import os

import numpy as np
import pytest

import cases
import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_AMG = os.path.join(ROOT, "oracle", "_ref", "libpfsf_ref_amg.so")

CASES = [((8, 8, 8), 1), ((7, 5, 9), 2), ((1, 1, 1), 3), ((2, 3, 1), 4), ((17, 13, 11), 5), ((32, 4, 3), 6)]


def _island(dims, seed):
    lx, ly, lz = dims
    n = lx * ly * lz
    rng = np.random.default_rng(seed)
    vtype = rng.choice(np.array([0, 1, 2], np.uint8), size=n, p=[0.2, 0.7, 0.1])
    sigma = rng.uniform(0.05, 2.0, size=(6, n)).astype(np.float32)
    sigma[:, vtype == 0] = 0.0
    # some solid voxels with every face conductivity zero (left out of their aggregate)
    zero = (rng.random(n) < 0.05) & (vtype == 1)
    sigma[:, zero] = 0.0
    # and a few faces zero at random
    sigma[rng.random((6, n)) < 0.1] = 0.0
    return sigma.reshape(-1), vtype


def _ref_build(dims, sigma, vtype):
    lib = C.CDLL(REF_AMG)
    f = lib.ref_build_amg
    f.restype = C.c_longlong
    lx, ly, lz = dims
    n = lx * ly * lz
    nc = ((lx + 1) // 2) * ((ly + 1) // 2) * ((lz + 1) // 2)
    agg = np.zeros(n, np.int32)
    w = np.zeros(n, np.float32)
    dc = np.zeros(max(nc, 1), np.float32)
    p = lambda a: a.ctypes.data_as(C.c_void_p)
    got = f(p(sigma), p(vtype), lx, ly, lz, p(agg), p(w), p(dc))
    return int(got), agg, w, dc[:nc]


@pytest.mark.parametrize("dims,seed", CASES)
def test_builder_matches_reference_bit_exact(dims, seed):
    if not os.path.exists(REF_AMG):
        pytest.skip("reference aggregation builder not built (make -C oracle -f ref.mk)")
    sigma, vtype = _island(dims, seed)
    nc, ragg, rw, rdc = _ref_build(dims, sigma, vtype)
    agg, w, dc = O.amg_build(dims, sigma, vtype)
    assert nc == dc.size
    np.testing.assert_array_equal(agg, ragg)
    assert np.array_equal(w.view(np.uint32), rw.view(np.uint32))
    assert np.array_equal(dc.view(np.uint32), rdc.view(np.uint32))


@pytest.mark.parametrize("dims,seed", CASES[:3])
def test_builder_invariants(dims, seed):
    """Weights of an aggregate sum to 1 (the builder's partition of unity),
    anchors and zero-conductivity voxels are left out, D_c >= 0."""
    sigma, vtype = _island(dims, seed)
    agg, w, dc = O.amg_build(dims, sigma, vtype)
    d6 = sigma.reshape(6, -1).sum(axis=0, dtype=np.float64)
    assert np.all(agg[vtype == 2] == -1)
    assert np.all(agg[d6 < 1e-20] == -1)
    assert np.all(w[agg < 0] == 0.0)
    sums = np.bincount(agg[agg >= 0], weights=w[agg >= 0].astype(np.float64), minlength=dc.size)
    used = np.bincount(agg[agg >= 0], minlength=dc.size) > 0
    np.testing.assert_allclose(sums[used], 1.0, rtol=1e-5)
    assert np.all(dc >= 0.0)


def test_correction_algebra():
    dims = (9, 7, 6)
    sigma, vtype = _island(dims, 11)
    agg, w, dc = O.amg_build(dims, sigma, vtype)
    rng = np.random.default_rng(12)
    r = rng.normal(size=agg.size).astype(np.float32)
    phi = rng.uniform(0, 1, size=agg.size).astype(np.float32)
    phi0 = phi.copy()
    O.amg_correct(dims, agg, w, dc, r, phi)
    m = agg >= 0
    rc = np.bincount(agg[m], weights=(w[m].astype(np.float64) * r[m]), minlength=dc.size)
    ec = np.where(dc > 1e-20, rc / np.where(dc > 1e-20, dc, 1.0), 0.0)
    want = phi0.astype(np.float64)
    want[m] += w[m] * ec[agg[m]]
    np.testing.assert_allclose(phi, want, rtol=1e-5, atol=1e-6)
    assert np.array_equal(phi[~m], phi0[~m])


def _oracle_island(case, amg):
    isl = O.Island(*case["dims"], amg=amg)
    isl.load(phi=case["phi"], source=case["source"], conductivity=case["conductivity"], type=case["type"],
             rcomp=case["rcomp"], rtens=case["rtens"], max_phi=case["max_phi"], hydration=case["hydration"])
    return isl


def test_tick_with_correction_runs_and_differs():
    """The oracle tick with the correction at the PCG start: finite, the same
    as the tick without it until PCG engages, different after."""
    case = cases.compat_case("block16")
    a, b = _oracle_island(case, False), _oracle_island(case, True)
    engaged = False
    for t in range(8):
        before = a.state()["pcg_allocated"] == 1
        a.tick()
        b.tick()
        pa, pb = a.view("phi"), b.view("phi")
        assert np.all(np.isfinite(pb))
        if not before and a.state()["pcg_allocated"] == 0:
            assert np.array_equal(pa, pb), f"tick {t}: no PCG yet, yet the two ticks differ"
        engaged |= a.state()["pcg_allocated"] == 1
    assert engaged
    assert not np.array_equal(a.view("phi"), b.view("phi"))
