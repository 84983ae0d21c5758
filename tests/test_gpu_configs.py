"""Parity of pfsf_tick_tolerance at the benchmark configurations' sizes
against the oracle's FP64 solution.

Each tick solves to a 1e-6 relative residual on the GPU, then runs the
reference tick's tail (history H = max(H, psi_e), phase field, failure scan)
on that phi.  The oracle solves the same system in FP64 (multigrid CG to
1e-11, oracle/kappa_mg.c) and runs its restatement of the tail on the FP64
phi rounded to FP32.  Checks:

* phi: max |phi_gpu - phi_fp64| <= 1e-5 max |phi_fp64| (FP64 accumulator);
* failure codes and the failure buffer: bit-exact on every voxel outside the
  tolerance margin.  The margin is found by perturbation: the oracle's tail
  also runs on four perturbed copies of phi_fp64 -- scaled by 1 +/- 1e-5
  and with independent per-voxel noise of 1e-5 max |phi| (ten times the
  solve's own error bound) -- each carrying its own history, damage and
  failure state.  A voxel where a perturbed run's code differs, or its H or
  damage differs by more than 1e-3 of the maximum (the psi_e switch of the
  history update, flux_in > 3 flux_out, scales psi_e by 100), sits within
  the solve tolerance of a decision threshold; since the phase field reads
  the damage of the six face neighbours, the margin grows by one voxel per
  tick.  The number of margin voxels is reported and bounded (0.5 % of the
  grid after one tick, 2 % after three);
* H and damage: within 1e-5 of their maxima outside the same margin.

Config 1: the 32^3 fully solid block, three-material mix.  Config 2: the
256 x 256 x 128 noise island (60 % occupancy).  Config 5, reduced: a
128 x 128 x 64 island at 55 % occupancy over 3 ticks with the load ramped,
the oracle carrying its own history, damage and failure state from tick to
tick.  Loads are scaled so max phi = 20 and resistances by 0.1 so the phase
field and the failure scan act on a share of the voxels.
"""
import json
import os

import numpy as np
import pytest

import oracle as O
from pfsf_b200 import capi, synth

pytestmark = pytest.mark.gpu

THREADS = os.cpu_count() or 1
DELTA = 1e-5


@pytest.fixture(scope="module")
def eng(lib_built):
    e = capi.Engine(capi.default_config(max_island_size=1 << 28, tick_budget_ms=1 << 30, vram=64 << 30))
    assert e.init() == capi.PFSF_OK, "CUDA device required"
    yield e
    e.close()


def _fp64(isl, source, x0=None):
    x, _, rel = O.kappa_mgpcg64(isl.dims, isl.kappa.astype(np.float64), isl.vtype, source.astype(np.float64),
                                tol=1e-11, maxit=5000, threads=THREADS, x0=x0)
    assert rel <= 1e-10
    return x


def _case(isl, phi_max=20.0, rscale=0.1):
    """Reference-layout inputs with the loads scaled so max phi = phi_max;
    also the FP64 solution per unit of that scaled load (a warm start for the
    per-tick FP64 solves: the system is linear in the load)."""
    phi = _fp64(isl, isl.source)
    scale = phi_max / np.abs(phi).max()
    case = {"conductivity": synth.face_sigma_from_kappa(isl.dims, isl.vtype, isl.kappa),
            "type": isl.vtype.copy(), "rcomp": (isl.rcomp * rscale).astype(np.float32),
            "rtens": (isl.rtens * rscale).astype(np.float32), "max_phi": np.full(isl.n, 1e9, np.float32),
            "hydration": np.ones(isl.n, np.float32), "source": (isl.source * scale).astype(np.float32)}
    return case, phi * scale


def _dilate6(m, dims):
    """m plus the six face neighbours of every voxel in it."""
    lx, ly, lz = dims
    g = m.reshape(lz, ly, lx)
    o = g.copy()
    o[1:] |= g[:-1]
    o[:-1] |= g[1:]
    o[:, 1:] |= g[:, :-1]
    o[:, :-1] |= g[:, 1:]
    o[:, :, 1:] |= g[:, :, :-1]
    o[:, :, :-1] |= g[:, :, 1:]
    return o.reshape(-1)


class Chain:
    """Oracle tail state (H, D, fail) carried from tick to tick."""

    def __init__(self, n):
        self.H = np.zeros(n, np.float32)
        self.D = np.zeros(n, np.float32)
        self.fail = np.zeros(n, np.uint32)

    def tick(self, dims, phi32, case):
        O.tolerance_tick_tail(dims, phi32, case, self.H, self.D, self.fail)


def _run(eng, iid, isl, case_x, ticks, prec, ramp=1.0, origin=(0, 0, 0)):
    case, x_unit = case_x
    eng.set_solve_mode(capi.SOLVE_BATCHED)
    eng.set_precision(prec)
    assert eng.add_island(iid, isl.dims, origin) == capi.PFSF_OK
    src = case["source"].copy()
    base = case["source"].copy()
    phi = np.zeros(isl.n, np.float32)
    phik = np.zeros(isl.n, np.float32)
    assert eng.register_buffers(iid, phi, src, case["conductivity"], case["type"], case["rcomp"], case["rtens"],
                                case["max_phi"]) == capi.PFSF_OK
    assert eng.register_kappa(iid, phik, src, isl.kappa, isl.vtype) == capi.PFSF_OK
    rng = np.random.default_rng(isl.n)
    solid = isl.vtype == 1
    noise = [rng.uniform(-1.0, 1.0, isl.n) * solid for _ in range(2)]
    chains = [Chain(isl.n) for _ in range(5)]
    margin = np.zeros(isl.n, bool)
    cap = 1 << 16
    report = []
    for t in range(ticks):
        f = 1.0 + (ramp - 1.0) * t / max(ticks - 1, 1)
        src[:] = base * np.float32(f)
        eng.L.pfsf_mark_full_rebuild(eng.h, iid)
        fb = np.zeros(1 + 4 * cap, np.int32)
        rc, st = eng.tick_tolerance([iid], fb, tol=1e-6)
        assert rc == capi.PFSF_OK and st.islands_converged == 1, st.max_rel_residual
        rc, x64 = eng.read_solution64(iid, isl.n)
        xr = _fp64(isl, src, x0=x_unit * f)
        err = float(np.abs(x64 - xr).max() / np.abs(xr).max())
        assert err <= 1e-5, f"tick {t}: phi error vs FP64 {err:.2e}"
        c = dict(case, source=src.copy())
        amp = DELTA * float(np.abs(xr).max())
        phis = [xr, xr * (1.0 + DELTA), xr * (1.0 - DELTA), xr + amp * noise[0], xr + amp * noise[1]]
        for ch, ph in zip(chains, phis):
            ch.tick(isl.dims, ph.astype(np.float32), c)
        ref = chains[0]
        fail_g = eng.debug_field(iid, 3)
        H_g = eng.debug_field(iid, 1)
        D_g = eng.debug_field(iid, 2)
        hs = max(float(np.abs(ref.H).max()), 1e-30)
        ds = max(float(np.abs(ref.D).max()), 1e-30)
        margin = _dilate6(margin, isl.dims) if t > 0 else margin
        for ch in chains[1:]:
            margin |= ch.fail != ref.fail
            margin |= np.abs(ch.H - ref.H) > 1e-3 * hs
            margin |= np.abs(ch.D - ref.D) > 1e-3 * ds
        fails = [ref.fail.astype(np.uint8)]
        out = ~margin
        bad = int(np.sum(fail_g[out] != fails[0][out]))
        assert bad == 0, f"tick {t}: {bad} failure codes differ outside the margin"
        assert float(np.abs(H_g - ref.H)[out].max(initial=0.0)) <= 1e-5 * hs, f"tick {t}: H"
        assert float(np.abs(D_g - ref.D)[out].max(initial=0.0)) <= 1e-5 * ds, f"tick {t}: damage"
        # the failure buffer: the GPU's tuples are its codes in voxel order
        nz = np.flatnonzero(fail_g)
        assert fb[0] == min(nz.size, cap)
        if nz.size:
            lx, ly, _ = isl.dims
            xs = nz[: fb[0]] % lx + origin[0]
            ys = (nz[: fb[0]] // lx) % ly + origin[1]
            zs = nz[: fb[0]] // (lx * ly) + origin[2]
            tup = fb[1: 1 + 4 * fb[0]].reshape(-1, 4)
            assert np.array_equal(tup[:, 0], xs) and np.array_equal(tup[:, 1], ys)
            assert np.array_equal(tup[:, 2], zs) and np.array_equal(tup[:, 3], fail_g[nz[: fb[0]]])
        report.append({"tick": t, "phi_err": err, "margin_voxels": int(margin.sum()),
                       "failures": int(np.count_nonzero(fails[0])), "relres": st.max_rel_residual})
    eng.L.pfsf_remove_island(eng.h, iid)
    print(json.dumps({"island": list(isl.dims), "precision": prec, "ticks": report}))
    return report


@pytest.mark.parametrize("prec", [capi.PREC_BF16, capi.PREC_FP32])
def test_config1_solid_block_32(eng, prec):
    isl = synth.solid_block((32, 32, 32), seed=1)
    rep = _run(eng, 9300 + prec, isl, _case(isl), ticks=1, prec=prec, origin=(4, 0, -2))
    assert rep[0]["failures"] > 0
    assert rep[0]["margin_voxels"] <= isl.n // 200, rep


def test_config2_noise_256x256x128(eng):
    isl = synth.noise_island((256, 256, 128), seed=11)
    rep = _run(eng, 9310, isl, _case(isl), ticks=1, prec=capi.PREC_BF16)
    assert rep[0]["failures"] > 0
    assert rep[0]["margin_voxels"] <= isl.n // 200, rep


def test_config5_fracture_reduced(eng):
    isl = synth.noise_island((128, 128, 64), seed=51, occupancy=0.55)
    rep = _run(eng, 9320, isl, _case(isl), ticks=3, prec=capi.PREC_BF16, ramp=2.0)
    assert rep[-1]["failures"] >= rep[0]["failures"] > 0
    assert max(r["margin_voxels"] for r in rep) <= isl.n // 50, rep
