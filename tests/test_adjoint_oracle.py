"""The FP64 adjoint calculus of the oracle, pinned against central finite
differences of FP64 oracle solves (CPU only).

No reference gradient exists (the reference has no adjoint code), so the
oracle's adjoint is itself checked here: dL/dkappa (solid and anchor voxels)
and dL/ds from one adjoint solve + the edge product agree with central
differences to 1e-6 relative.  The torch loss of the tooling
(pfsf_b200.adjoint.calibration_loss) is checked against the oracle's FP64 loss
and its partials.
"""
import numpy as np
import torch

import oracle as O
from pfsf_b200 import adjoint as AD
from pfsf_b200 import synth


def _setup(dims=(10, 9, 8), seed=3):
    isl = synth.noise_island(dims, seed=seed)
    k = isl.kappa.astype(np.float64)
    s = isl.source.astype(np.float64)
    phi, _, rr = O.kappa_solve64(isl.dims, k, isl.vtype, s, tol=1e-14)
    assert rr < 1e-13
    rc = np.full(isl.n, float(np.median(np.abs(s[isl.vtype == 1]))) * 3.0)
    pt = 0.9 * phi
    return isl, k, s, phi, rc, pt


def test_oracle_adjoint_matches_finite_differences():
    isl, k, s, phi, rc, pt = _setup()
    dims, vt = isl.dims, isl.vtype

    def total(kk, ss):
        ph, _, _ = O.kappa_solve64(dims, kk, vt, ss, tol=1e-14, x0=phi)
        return O.flux_loss64(dims, kk, vt, ph, rc, pt)[0]

    L, gphi, gk_direct = O.flux_loss64(dims, k, vt, phi, rc, pt)
    gs, gk_edge, rr = O.kappa_adjoint64(dims, k, vt, phi, gphi, tol=1e-14)
    gk = gk_direct + gk_edge
    rng = np.random.default_rng(0)
    nonair = np.where(vt != 0)[0]
    solid = np.where(vt == 1)[0]
    assert np.any(vt[nonair] == 2)
    for i in rng.choice(nonair, 10, replace=False):
        h = 1e-5 * k[i]
        kp, km = k.copy(), k.copy()
        kp[i] += h
        km[i] -= h
        fd = (total(kp, s) - total(km, s)) / (2 * h)
        assert abs(gk[i] - fd) <= 1e-6 * abs(fd), (i, vt[i], gk[i], fd)
    for i in rng.choice(solid, 6, replace=False):
        h = 1e-5 * abs(s[i]) + 1e-3
        sp, sm = s.copy(), s.copy()
        sp[i] += h
        sm[i] -= h
        fd = (total(k, sp) - total(k, sm)) / (2 * h)
        assert abs(gs[i] - fd) <= 1e-6 * abs(fd), (i, gs[i], fd)
    assert np.all(gk[vt == 0] == 0) and np.all(gs[vt != 1] == 0)


def test_torch_loss_matches_oracle():
    isl, k, s, phi, rc, pt = _setup((9, 8, 7), seed=5)
    L, gphi, gk = O.flux_loss64(isl.dims, k, isl.vtype, phi, rc, pt)
    kt = torch.tensor(k, requires_grad=True)
    pht = torch.tensor(phi, requires_grad=True)
    Lt = AD.calibration_loss(pht, kt, isl.vtype, isl.dims, torch.tensor(rc), torch.tensor(pt))
    Lt.backward()
    assert abs(float(Lt.detach()) - L) <= 1e-12 * abs(L)
    np.testing.assert_allclose(pht.grad.numpy(), gphi, rtol=0, atol=1e-12 * np.abs(gphi).max())
    np.testing.assert_allclose(kt.grad.numpy(), gk, rtol=0, atol=1e-12 * np.abs(gk).max())


def test_flux_in_is_the_failure_scan_inflow():
    """flux_in_i = sum_j w_ij max(phi_j - phi_i, 0) by direct summation."""
    isl = synth.noise_island((6, 5, 4), seed=8)
    rng = np.random.default_rng(2)
    phi = rng.normal(size=isl.n)
    k = isl.kappa.astype(np.float64)
    f = AD.flux_in(torch.tensor(phi), torch.tensor(k), isl.vtype, isl.dims).numpy()
    lx, ly, lz = isl.dims
    vt = isl.vtype
    p = np.where(vt == 1, phi, 0.0)
    want = np.zeros(isl.n)
    for z in range(lz):
        for y in range(ly):
            for x in range(lx):
                i = x + lx * (y + ly * z)
                if vt[i] == 0:
                    continue
                for dz in (-1, 0, 1):
                    for dy in (-1, 0, 1):
                        for dx in (-1, 0, 1):
                            m = abs(dx) + abs(dy) + abs(dz)
                            if m == 0 or not (0 <= x + dx < lx and 0 <= y + dy < ly and 0 <= z + dz < lz):
                                continue
                            j = (x + dx) + lx * ((y + dy) + ly * (z + dz))
                            if vt[j] == 0:
                                continue
                            w = [1.0, 0.5, 1 / 6][m - 1] * 2 * k[i] * k[j] / (k[i] + k[j])
                            want[i] += w * max(p[j] - p[i], 0.0)
    np.testing.assert_allclose(f, want, rtol=1e-12, atol=1e-12 * np.abs(want).max())


def test_amor_psi_is_the_history_update():
    """The torch and FP64 psi_e used by the trajectory loss are the history
    update of the tick (oracle o_history, the restatement of
    SH/rbgs_smooth.comp.glsl:177-191 on the face conductivity)."""
    import torch
    from pfsf_b200 import adjoint as AD
    isl = synth.noise_island((14, 12, 10), seed=23)
    rng = np.random.default_rng(23)
    phi = (rng.uniform(0.0, 2.0, isl.n) * (isl.vtype == 1)).astype(np.float32)
    sig = synth.face_sigma_from_kappa(isl.dims, isl.vtype, isl.kappa)
    H = np.zeros(isl.n, np.float32)
    O.history(isl.dims, phi, sig, isl.vtype, H)
    k64 = isl.kappa.astype(np.float64)
    psi64, _ = O.amor_psi64(isl.dims, k64, isl.vtype, phi.astype(np.float64))
    pt = AD.amor_psi(torch.tensor(phi.astype(np.float64)), torch.tensor(k64), isl.vtype, isl.dims).numpy()
    sc = float(np.abs(H).max())
    assert np.abs(psi64 - H).max() <= 1e-5 * sc
    assert np.abs(pt - psi64).max() <= 1e-12 * sc
