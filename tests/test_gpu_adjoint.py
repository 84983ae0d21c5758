"""GPU adjoint of the tolerance solve, and the whole-GPU solve tier.

Bars:
  * pfsf_adjoint_to_tolerance (dL/dkappa, dL/ds for a given dL/dphi) agrees
    with the FP64 oracle adjoint to 1e-6 of its largest entry (solves at
    rel. tol 1e-10 vs 1e-14), in both execution modes and every precision;
  * the torch tooling (KappaSolve + calibration_loss) gives the oracle's total
    gradient to 1e-6, and central finite differences (h = 2^-10 on kappa, the
    config-4 step) to 1e-4 relative on voxels away from the inflow kinks;
  * per-tick losses over a ramped trajectory recompute evicted ticks from
    their checkpoints and still match the oracle;
  * the whole-GPU tier (islands >= PFSF_GRID_MIN_VOXELS, cooperative launch,
    software grid barrier) converges and matches the FP64 oracle solve.
"""
import os

import numpy as np
import pytest
import torch

import oracle as O
from pfsf_b200 import adjoint as AD
from pfsf_b200 import capi, synth

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _engine():
    e = capi.Engine(capi.default_config(max_island_size=1 << 26, tick_budget_ms=1 << 30))
    assert e.init() == capi.PFSF_OK, "CUDA device required"
    return e


@pytest.fixture(scope="module")
def eng(lib_built):
    e = _engine()
    yield e
    e.close()


_ids = [7000]


def _next_id():
    _ids[0] += 1
    return _ids[0]


def _problem(dims, seed):
    isl = synth.noise_island(dims, seed=seed)
    k = isl.kappa.astype(np.float64)
    s = isl.source.astype(np.float64)
    phi, _, _ = O.kappa_solve64(isl.dims, k, isl.vtype, s, tol=1e-14)
    rc = np.full(isl.n, float(np.median(np.abs(s[isl.vtype == 1]))) * 3.0)
    return isl, k, s, phi, rc, 0.9 * phi


@pytest.mark.parametrize("mode,prec", [(capi.SOLVE_PER_ISLAND, capi.PREC_FP32), (capi.SOLVE_BATCHED, capi.PREC_FP32),
                                       (capi.SOLVE_BATCHED, capi.PREC_BF16), (capi.SOLVE_BATCHED, capi.PREC_FP16)])
def test_adjoint_matches_oracle(eng, mode, prec):
    eng.set_solve_mode(mode)
    eng.set_precision(prec)
    isl, k, s, phi, rc, pt = _problem((20, 18, 14), seed=21)
    sess = AD.Session(eng, _next_id(), isl.dims, isl.vtype, tol=TOL)
    x = sess.solve(isl.kappa, isl.source)
    assert np.abs(x - phi).max() <= 1e-7 * np.abs(phi).max()
    _, g, _ = O.flux_loss64(isl.dims, k, isl.vtype, phi, rc, pt)
    gs, gk = sess.adjoint(g.astype(np.float32))
    gs_o, gk_o, _ = O.kappa_adjoint64(isl.dims, k, isl.vtype, x, g.astype(np.float32).astype(np.float64), tol=1e-14)
    assert np.abs(gs - gs_o).max() <= 1e-6 * np.abs(gs_o).max()
    assert np.abs(gk - gk_o).max() <= 1e-6 * np.abs(gk_o).max()
    assert np.all(gk[isl.vtype == 0] == 0) and np.all(gs[isl.vtype != 1] == 0)
    # the forward solution is still the arena's record after the adjoint
    rc2, x2 = eng.read_solution64(sess.iid, isl.n)
    assert np.array_equal(x, x2)


def test_torch_gradient_and_finite_differences(eng):
    eng.set_solve_mode(capi.SOLVE_BATCHED)
    eng.set_precision(capi.PREC_BF16)
    isl, k, s, phi, rc, pt = _problem((24, 20, 16), seed=4)
    sess = AD.Session(eng, _next_id(), isl.dims, isl.vtype, tol=TOL)
    kt = torch.tensor(isl.kappa.astype(np.float64), requires_grad=True)
    st = torch.tensor(isl.source.astype(np.float64), requires_grad=True)
    ph = AD.KappaSolve.apply(kt, st, sess, "base", None)
    L = AD.calibration_loss(ph, kt, isl.vtype, isl.dims, torch.tensor(rc), torch.tensor(pt))
    L.backward()
    # oracle total gradient at the float32 kappa / source the solve used
    k32, s32 = isl.kappa.astype(np.float64), isl.source.astype(np.float64)
    _, gphi, gkd = O.flux_loss64(isl.dims, k32, isl.vtype, ph.detach().numpy(), rc, pt)
    gs_o, gke, _ = O.kappa_adjoint64(isl.dims, k32, isl.vtype, ph.detach().numpy(), gphi, tol=1e-14)
    gk_o = gkd + gke
    assert np.abs(kt.grad.numpy() - gk_o).max() <= 1e-6 * np.abs(gk_o).max()
    assert np.abs(st.grad.numpy() - gs_o).max() <= 1e-6 * np.abs(gs_o).max()

    def loss_np(phv, kv):
        return float(AD.calibration_loss(torch.tensor(phv), torch.tensor(kv), isl.vtype, isl.dims,
                                         torch.tensor(rc), torch.tensor(pt)))

    rng = np.random.default_rng(1)
    vox = rng.choice(np.where(isl.vtype != 0)[0], 24, replace=False)
    fd, kink = AD.finite_difference_kappa(sess, isl.kappa, isl.source, ph.detach().numpy(), loss_np, vox)
    g = kt.grad.numpy()[vox]
    ok = ~kink
    assert ok.sum() >= 12
    rel = np.abs(g[ok] - fd[ok]) / np.abs(fd[ok])
    assert rel.max() <= 1e-4, (rel.max(), vox[ok][np.argmax(rel)])


def test_trajectory_recompute_from_checkpoints(eng):
    eng.set_solve_mode(capi.SOLVE_BATCHED)
    eng.set_precision(capi.PREC_BF16)
    isl, k, s, phi, rc, pt = _problem((16, 14, 12), seed=9)
    sess = AD.Session(eng, _next_id(), isl.dims, isl.vtype, tol=TOL)
    kt = torch.tensor(isl.kappa.astype(np.float64), requires_grad=True)
    st = torch.tensor(isl.source.astype(np.float64))
    phis, H, ck = AD.ramped_trajectory(sess, kt, st, ticks=6, ramp=2.0, checkpoint_every=2)
    assert sorted(ck) == [0, 2, 4]
    assert np.allclose(H, 0.5 * phis[-1].detach().numpy() ** 2)  # monotone ramp: last tick is the max
    L = sum(AD.calibration_loss(p, kt, isl.vtype, isl.dims, torch.tensor(rc), torch.tensor(pt)) for p in phis)
    L.backward()
    assert sess.recomputes == 5  # every tick but the last was evicted from the device
    # oracle: sum over ticks of the single-tick gradients
    k32 = isl.kappa.astype(np.float64)
    gk_o = np.zeros(isl.n)
    for t, p in enumerate(phis):
        pv = p.detach().numpy()
        _, gphi, gkd = O.flux_loss64(isl.dims, k32, isl.vtype, pv, rc, pt)
        _, gke, _ = O.kappa_adjoint64(isl.dims, k32, isl.vtype, pv, gphi, tol=1e-14)
        gk_o += gkd + gke
    assert np.abs(kt.grad.numpy() - gk_o).max() <= 1e-6 * np.abs(gk_o).max()


def test_adjoint_argument_errors(eng):
    eng.set_solve_mode(capi.SOLVE_BATCHED)
    eng.set_precision(capi.PREC_FP32)
    isl = synth.noise_island((12, 10, 8), seed=1)
    iid = _next_id()
    assert eng.add_island(iid, isl.dims) == capi.PFSF_OK
    phi = np.zeros(isl.n, np.float32)
    assert eng.register_kappa(iid, phi, isl.source, isl.kappa, isl.vtype) == capi.PFSF_OK
    assert eng.solve([iid], tol=1e-6)[0] == capi.PFSF_OK
    # no adjoint buffers registered
    assert eng.adjoint([iid])[0] == capi.PFSF_ERROR_INVALID_ARG
    g = np.zeros(isl.n, np.float32)
    short = np.zeros(isl.n - 1, np.float32)
    assert eng.register_adjoint(iid, g, g.copy(), short) == capi.PFSF_ERROR_INVALID_ARG
    assert eng.register_adjoint(iid, g, g.copy(), g.copy()) == capi.PFSF_OK
    # an island set the arena has not solved
    other = _next_id()
    assert eng.add_island(other, isl.dims) == capi.PFSF_OK
    assert eng.register_kappa(other, phi.copy(), isl.source, isl.kappa, isl.vtype) == capi.PFSF_OK
    assert eng.register_adjoint(other, g.copy(), g.copy(), g.copy()) == capi.PFSF_OK
    assert eng.adjoint([other])[0] == capi.PFSF_ERROR_INVALID_ARG
    # zero dL/dphi -> zero gradients
    assert eng.adjoint([iid])[0] == capi.PFSF_OK


def test_whole_gpu_tier_matches_oracle(lib_built):
    old = os.environ.get("PFSF_GRID_MIN_VOXELS")
    os.environ["PFSF_GRID_MIN_VOXELS"] = "6000"
    try:
        e = _engine()
    finally:
        if old is None:
            del os.environ["PFSF_GRID_MIN_VOXELS"]
        else:
            os.environ["PFSF_GRID_MIN_VOXELS"] = old
    try:
        e.set_solve_mode(capi.SOLVE_BATCHED)
        for prec in (capi.PREC_BF16, capi.PREC_FP32):
            e.set_precision(prec)
            # two giant islands (whole-GPU tier, one after the other) and two
            # small ones (persistent kernel) in one solve
            # (45 x 37 x 35: several plane-marching work items, odd sides)
            isls = [synth.noise_island((45, 37, 35), seed=31), synth.solid_block((20, 20, 20), seed=2),
                    synth.noise_island((12, 10, 9), seed=33), synth.noise_island((9, 8, 7), seed=34)]
            isls = [i for i in isls if i.n_active > 0]
            ids, hosts = [], []
            for isl in isls:
                iid = _next_id()
                assert e.add_island(iid, isl.dims) == capi.PFSF_OK
                h = np.zeros(isl.n, np.float32)
                assert e.register_kappa(iid, h, isl.source, isl.kappa, isl.vtype) == capi.PFSF_OK
                ids.append(iid)
                hosts.append(h)
            rc, st = e.solve(ids, tol=1e-6)
            assert rc == capi.PFSF_OK and st.islands_converged == len(isls), st.max_rel_residual
            for isl, iid, h in zip(isls, ids, hosts):
                rc, x64 = e.read_solution64(iid, isl.n)
                k64 = isl.kappa.astype(np.float64)
                r = isl.source.astype(np.float64) - O.kappa_apply(isl.dims, k64, isl.vtype, x64)
                sol = isl.vtype == 1
                assert np.linalg.norm(r[sol]) <= 1e-6 * np.linalg.norm(isl.source[sol].astype(np.float64))
                xr, _, _ = O.kappa_solve64(isl.dims, k64, isl.vtype, isl.source.astype(np.float64), tol=1e-12)
                assert np.abs(x64 - xr).max() <= 1e-4 * np.abs(xr).max()
                np.testing.assert_array_equal(h, x64.astype(np.float32))
            # adjoint through the whole-GPU tier
            isl = isls[0]
            g = np.random.default_rng(0).normal(size=isl.n).astype(np.float32)
            gbufs = [np.zeros(i.n, np.float32) for i in isls for _ in range(3)]
            for q, (i2, iid) in enumerate(zip(isls, ids)):
                gp = g if q == 0 else gbufs[3 * q]
                assert e.register_adjoint(iid, gp, gbufs[3 * q + 1], gbufs[3 * q + 2]) == capi.PFSF_OK
            rc, st = e.adjoint(ids, tol=1e-10)
            assert rc == capi.PFSF_OK and st.islands_converged == len(isls)
            rc, x64 = e.read_solution64(ids[0], isl.n)
            gs_o, gk_o, _ = O.kappa_adjoint64(isl.dims, isl.kappa.astype(np.float64), isl.vtype, x64,
                                              g.astype(np.float64), tol=1e-14)
            assert np.abs(gbufs[2] - gk_o).max() <= 1e-6 * np.abs(gk_o).max()
            assert np.abs(gbufs[1] - gs_o).max() <= 1e-6 * np.abs(gs_o).max()
    finally:
        e.close()


def test_trajectory_loss_gradient_matches_fp64_oracle_and_fd(eng):
    """The config-4 trajectory loss (per-tick flux and target terms plus the
    history term over H = max_t psi_e, psi_e with the Amor split) on a
    reduced island over 6 ramped ticks, checkpoint every 2: the torch
    gradient through every tick's device adjoint (5 ticks recomputed from
    their checkpoints) matches the FP64 oracle's trajectory gradient to 1e-6
    of its largest entry, and central differences to 1e-4 relative on
    voxels away from kinks."""
    eng.set_solve_mode(capi.SOLVE_BATCHED)
    eng.set_precision(capi.PREC_BF16)
    isl, k, s, phi, rc, pt = _problem((24, 20, 12), seed=31)
    k64 = isl.kappa.astype(np.float64)
    psi, _ = O.amor_psi64(isl.dims, k64, isl.vtype, 2.0 * phi)
    hs = 0.5 * float(psi.max())  # the history term acts on the most loaded voxels
    sess = AD.Session(eng, _next_id(), isl.dims, isl.vtype, tol=TOL)
    kt = torch.tensor(k64, requires_grad=True)
    st = torch.tensor(isl.source.astype(np.float64))
    L, phis, H = AD.trajectory_loss(sess, kt, st, rc, pt, ticks=6, ramp=2.0, checkpoint_every=2, h_scale=hs)
    L.backward()
    assert sess.recomputes == 5
    Lo, gko, phis_o, arg = O.trajectory_grad64(isl.dims, k64, isl.vtype, isl.source.astype(np.float64), rc, pt,
                                               6, 2.0, hs)
    assert abs(float(L) - Lo) <= 1e-6 * abs(Lo)
    g = kt.grad.detach().cpu().numpy()
    assert np.abs(g - gko).max() <= 1e-6 * np.abs(gko).max()
    assert len(set(arg[arg >= 0].tolist())) >= 1
    # central differences of the whole trajectory's loss
    rng = np.random.default_rng(31)
    vox = rng.choice(np.flatnonzero(isl.vtype != 0), 12, replace=False)
    phis0 = [p.detach().numpy() for p in phis]
    fd, kink = AD.trajectory_finite_difference(sess, isl.kappa.astype(np.float32), isl.source, phis0, rc, pt, vox,
                                               ramp=2.0, h_scale=hs)
    ok = ~kink
    assert ok.sum() >= 6
    rel = np.abs(g[vox][ok] - fd[ok]) / np.maximum(np.abs(fd[ok]), 1e-30)
    assert rel.max() <= 1e-4, rel
