"""The oracle's multigrid-preconditioned CG (oracle/kappa_mg.c) against its
FP64 Jacobi-PCG on the same operator.

The multigrid CG gives the FP64 reference solutions of the large benchmark
islands (256x256x128 and up), which the Jacobi-PCG cannot reach in a bounded
time; here both solve the same small islands and must agree to 1e-10
relative, single- and multi-threaded.  The FP32 variant (the timed CPU
baseline: FP32 V-cycle PCG inside FP64 residual refinement) must reach the
1e-6 relative residual and stay within 1e-5 of the FP64 solution.
"""
import numpy as np
import pytest

import oracle as O
from pfsf_b200 import synth


@pytest.mark.parametrize("dims,seed,kind", [((16, 14, 12), 3, "noise"), ((24, 20, 16), 4, "noise"),
                                            ((12, 12, 12), 5, "solid"), ((33, 9, 7), 6, "noise")])
def test_mgpcg64_matches_jacobi_pcg64(dims, seed, kind):
    isl = synth.noise_island(dims, seed=seed) if kind == "noise" else synth.solid_block(dims, seed=seed)
    k = isl.kappa.astype(np.float64)
    s = isl.source.astype(np.float64)
    xr, _, rr = O.kappa_solve64(dims, k, isl.vtype, s, tol=1e-13, maxit=200000)
    assert rr <= 1e-12
    x1, it1, r1 = O.kappa_mgpcg64(dims, k, isl.vtype, s, tol=1e-12, threads=1)
    x4, it4, r4 = O.kappa_mgpcg64(dims, k, isl.vtype, s, tol=1e-12, threads=4)
    assert r1 <= 1e-12 and r4 <= 1e-12
    sc = np.abs(xr).max()
    assert np.abs(x1 - xr).max() / sc <= 1e-10
    assert np.abs(x4 - xr).max() / sc <= 1e-10
    assert it1 < 60  # the V-cycle preconditioner does its job
    assert np.all(x1[isl.vtype != 1] == 0.0)


def test_mgpcg32_reaches_tolerance():
    isl = synth.noise_island((40, 30, 20), seed=7)
    k = isl.kappa.astype(np.float64)
    s = isl.source.astype(np.float64)
    xr, _, _ = O.kappa_mgpcg64(isl.dims, k, isl.vtype, s, tol=1e-12, threads=2)
    x, it, rel, outer = O.kappa_mgpcg32(isl.dims, k, isl.vtype, s, tol=1e-6, threads=2)
    assert rel <= 1e-6
    assert 1 <= outer <= 8
    assert np.abs(x - xr).max() / np.abs(xr).max() <= 1e-5
    # its residual is the FP64 operator's
    r = s - O.kappa_apply(isl.dims, k, isl.vtype, x)
    solid = isl.vtype == 1
    assert np.linalg.norm(r[solid]) / np.linalg.norm(s[solid]) == pytest.approx(rel, rel=1e-6)


def test_mgpcg_source_free_and_orphan():
    # source-free island: phi = 0 (debug/L12_SourceFreeIslandTest.java:98-104)
    isl = synth.noise_island((12, 10, 8), seed=8)
    zero = np.zeros(isl.n)
    x, it, rel = O.kappa_mgpcg64(isl.dims, isl.kappa.astype(np.float64), isl.vtype, zero, tol=1e-12)
    assert it == 0 and np.all(x == 0.0)
