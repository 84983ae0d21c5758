"""Differentiable tolerance solve for material calibration (torch tooling).

The solve A(kappa) phi = s runs on the GPU through the C ABI
(pfsf_solve_to_tolerance); its gradient is the hand-written adjoint
(pfsf_adjoint_to_tolerance: one more solve with the same symmetric operator
plus an edge-product kernel giving dL/dkappa and dL/ds).  ``KappaSolve`` wraps
the pair as a torch.autograd.Function; the loss terms around it (the failure
scan's compressive inflow, a target misfit) are plain torch so autograd
supplies their direct partials.

Multi-tick trajectories (loads ramped over ticks, phase-field history
H = max(H, psi_e) carried along) keep a checkpoint of phi every
``checkpoint_every`` ticks; a tick whose solution is no longer the one held
on the device is re-solved from the nearest checkpoint during backward.

The reference has no gradient code: there is nothing to be bit-compatible
with; the calculus is checked against central finite differences and an FP64
CPU adjoint.
"""
from __future__ import annotations

import numpy as np
import torch

from . import capi


# --------------------------------------------------------------- operator links
def _dirs13():
    """Link directions counted once, with the group scale c (1, 1/2, 1/6)."""
    out = []
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                if (dz, dy, dx) > (0, 0, 0):
                    m = abs(dx) + abs(dy) + abs(dz)
                    out.append((dx, dy, dz, (1.0, 0.5, 1.0 / 6.0)[m - 1]))
    return out


_DIRS13 = _dirs13()


def _span(d, n):
    if d == 0:
        return slice(0, n), slice(0, n)
    return (slice(0, n - 1), slice(1, n)) if d == 1 else (slice(1, n), slice(0, n - 1))


def _pairs(dims, with_offset=False):
    lx, ly, lz = dims
    for dx, dy, dz, c in _DIRS13:
        (zi, zj), (yi, yj), (xi, xj) = _span(dz, lz), _span(dy, ly), _span(dx, lx)
        if with_offset:
            yield (zi, yi, xi), (zj, yj, xj), c, (dx, dy, dz)
        else:
            yield (zi, yi, xi), (zj, yj, xj), c


def _grow(v, off, side):
    """Zero-pads a per-link array (the i or j side of one direction) back to
    the full (lz, ly, lx) grid."""
    pads = []
    for d in off:  # x, y, z: torch pads the last dimension first
        if d == 0:
            pads += [0, 0]
        elif (d == 1) == (side == "i"):
            pads += [0, 1]
        else:
            pads += [1, 0]
    return torch.nn.functional.pad(v, pads)


def flux_in(phi, kappa, vtype, dims):
    """Compressive inflow of every voxel, sum_j w_ij max(phi_j - phi_i, 0)
    over the operator's links (w_ij = c 2 k_i k_j / (k_i + k_j)), as in the
    failure scan (SH/failure_scan.comp.glsl:89-158) on kappa link weights.
    phi is taken as 0 off the solid voxels.  Differentiable in phi and kappa."""
    lx, ly, lz = dims
    t = torch.as_tensor(vtype, device=phi.device).reshape(lz, ly, lx)
    solid = t == 1
    nonair = t != 0
    k = kappa.reshape(lz, ly, lx)
    zero = torch.zeros((), dtype=phi.dtype, device=phi.device)
    one = torch.ones((), dtype=k.dtype, device=phi.device)
    p = torch.where(solid, phi.reshape(lz, ly, lx), zero)
    f = torch.zeros_like(p)
    for si, sj, c, off in _pairs(dims, with_offset=True):
        ki, kj = k[si], k[sj]
        ok = nonair[si] & nonair[sj]
        s = torch.where(ok, ki + kj, one)
        w = torch.where(ok, 2.0 * c * ki * kj / s, zero)
        u = p[sj] - p[si]
        f = f + _grow(w * torch.relu(u), off, "i") + _grow(w * torch.relu(-u), off, "j")
    return f.reshape(-1)


def calibration_loss(phi, kappa, vtype, dims, rcomp, phi_target):
    """L = sum_solid softplus(flux_in / rcomp - 1) + 1/2 sum_solid (phi - phi_target)^2."""
    solid = torch.as_tensor(np.asarray(vtype) == 1, device=phi.device)
    f = flux_in(phi, kappa, vtype, dims)
    z = f / rcomp - 1.0
    d = phi - phi_target
    zero = torch.zeros((), dtype=phi.dtype, device=phi.device)
    return torch.where(solid, torch.nn.functional.softplus(z) + 0.5 * d * d, zero).sum()


# ------------------------------------------------------------------- session
class Session:
    """One island on an engine, registered for differentiable solves."""

    def __init__(self, eng: capi.Engine, iid: int, dims, vtype, tol=1e-10, max_iter=2000):
        self.eng, self.iid, self.dims, self.tol, self.max_iter = eng, iid, tuple(dims), tol, max_iter
        n = int(np.prod(dims))
        self.n = n
        self.vtype = np.ascontiguousarray(vtype, np.uint8)
        self.phi = np.zeros(n, np.float32)
        self.source = np.zeros(n, np.float32)
        self.kappa = np.zeros(n, np.float32)
        self.g_phi = np.zeros(n, np.float32)
        self.g_src = np.zeros(n, np.float32)
        self.g_kap = np.zeros(n, np.float32)
        assert eng.add_island(iid, self.dims) == capi.PFSF_OK
        assert eng.register_kappa(iid, self.phi, self.source, self.kappa, self.vtype) == capi.PFSF_OK
        assert eng.register_adjoint(iid, self.g_phi, self.g_src, self.g_kap) == capi.PFSF_OK
        self.current = None  # tag of the forward solution held on the device
        self.solves = 0
        self.recomputes = 0
        self.last_stats = None

    def solve(self, kappa, source, tag=None, warm=None):
        """FP64 solution of A(kappa) phi = source (kappa, source: float32 arrays)."""
        self.kappa[:] = kappa
        self.source[:] = source
        flags = capi.SOLVE_COLD_START
        if warm is not None:
            self.phi[:] = warm
            flags = 0
        rc, st = self.eng.solve([self.iid], tol=self.tol, max_iter=self.max_iter, flags=flags)
        if rc != capi.PFSF_OK or st.islands_converged != 1:
            raise RuntimeError(f"solve failed rc={rc} relres={st.max_rel_residual:.3e}")
        rc, x = self.eng.read_solution64(self.iid, self.n)
        self.current = tag
        self.solves += 1
        self.last_stats = st
        return x

    def adjoint(self, grad_phi):
        """(dL/ds, dL/dkappa) for dL/dphi = grad_phi at the solution on the device."""
        self.g_phi[:] = grad_phi
        rc, st = self.eng.adjoint([self.iid], tol=self.tol, max_iter=self.max_iter)
        if rc != capi.PFSF_OK or st.islands_converged != 1:
            raise RuntimeError(f"adjoint failed rc={rc} relres={st.max_rel_residual:.3e}")
        self.last_stats = st
        return self.g_src.astype(np.float64), self.g_kap.astype(np.float64)


class KappaSolve(torch.autograd.Function):
    """phi = A(kappa)^-1 source on the GPU; backward = the device adjoint.

    kappa and source are 1-D CPU tensors (any float dtype; the solve uses their
    float32 values); phi is float64 (the solver's FP64 accumulator)."""

    @staticmethod
    def forward(ctx, kappa, source, session: Session, tag=None, checkpoint=None):
        k = kappa.detach().cpu().numpy().astype(np.float32)
        s = source.detach().cpu().numpy().astype(np.float32)
        x = session.solve(k, s, tag=tag, warm=checkpoint)
        ctx.session, ctx.tag, ctx.checkpoint = session, tag, checkpoint
        ctx.k, ctx.s = k, s
        ctx.dtypes = (kappa.dtype, source.dtype)
        return torch.from_numpy(x)

    @staticmethod
    def backward(ctx, grad_phi):
        sess = ctx.session
        if sess.current is None or sess.current != ctx.tag:
            # the device holds another tick's solution: recompute this one
            # (warm-started from its checkpoint) before the adjoint
            sess.solve(ctx.k, ctx.s, tag=ctx.tag, warm=ctx.checkpoint)
            sess.recomputes += 1
        gs, gk = sess.adjoint(grad_phi.detach().cpu().numpy())
        return (torch.from_numpy(gk).to(ctx.dtypes[0]), torch.from_numpy(gs).to(ctx.dtypes[1]), None, None, None)


def ramped_trajectory(session: Session, kappa, source, ticks=32, ramp=2.0, checkpoint_every=8):
    """Runs `ticks` ticks with the load ramped linearly from 1x to `ramp`x.
    Returns (phi of every tick (list of tensors, differentiable), history H
    (numpy, max over ticks of psi_e = phi^2 / 2), checkpoints {tick: phi})."""
    checkpoints = {}
    H = np.zeros(session.n)
    phis = []
    warm = None
    for t in range(ticks):
        f = 1.0 + (ramp - 1.0) * t / max(ticks - 1, 1)
        base = checkpoints.get(checkpoint_every * (t // checkpoint_every))
        phi = KappaSolve.apply(kappa, source * f, session, t, warm if base is None else base)
        x = phi.detach().numpy()
        if t % checkpoint_every == 0:
            checkpoints[t] = x.astype(np.float32)
        H = np.maximum(H, 0.5 * x * x)
        warm = x.astype(np.float32)
        phis.append(phi)
    return phis, H, checkpoints


# --------------------------------------------------------- finite differences
def _local_rhs(dims, kappa64, vtype, phi0, i, kappa_i_new):
    """-(A(kappa') - A(kappa)) phi0 for kappa' = kappa with voxel i changed:
    nonzero only at i and its 26 neighbours (FP64)."""
    lx, ly, lz = dims
    x, y, z = i % lx, (i // lx) % ly, i // (lx * ly)
    rows = {}
    ki0, ki1 = kappa64[i], kappa_i_new
    pi = phi0[i] if vtype[i] == 1 else 0.0
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                if dx == dy == dz == 0:
                    continue
                nx, ny, nz = x + dx, y + dy, z + dz
                if not (0 <= nx < lx and 0 <= ny < ly and 0 <= nz < lz):
                    continue
                j = nx + lx * (ny + ly * nz)
                if vtype[j] == 0 or vtype[i] == 0:
                    continue
                c = (1.0, 0.5, 1.0 / 6.0)[abs(dx) + abs(dy) + abs(dz) - 1]
                kj = kappa64[j]
                w0 = 2.0 * c * ki0 * kj / (ki0 + kj) if ki0 + kj > 0 else 0.0
                w1 = 2.0 * c * ki1 * kj / (ki1 + kj) if ki1 + kj > 0 else 0.0
                dw = w1 - w0
                pj = phi0[j] if vtype[j] == 1 else 0.0
                if vtype[i] == 1:
                    rows[i] = rows.get(i, 0.0) - dw * (pi - pj)
                if vtype[j] == 1:
                    rows[j] = rows.get(j, 0.0) - dw * (pj - pi)
    return rows


def finite_difference_kappa(session: Session, kappa32, source32, phi0, loss_fn, voxels, h=2.0 ** -10):
    """Central differences dL/dkappa_i = (L(kappa + h e_i) - L(kappa - h e_i)) / (2h)
    of L(phi(kappa), kappa) for each voxel i.

    Each perturbed solution is phi0 + delta with A(kappa') delta =
    -(A(kappa') - A(kappa)) phi0 -- the same perturbed system written for
    the (small) change of phi, so the solver's relative tolerance applies to
    the change and not to phi; the step is taken in float32 (the solve's
    kappa precision) and the exact float32 step is the denominator.
    Returns (fd values, kink flags): a kink flag marks a voxel whose +/-
    solutions put some link on different sides of the failure-scan inflow's
    max(., 0), where the loss is not differentiable."""
    k64 = kappa32.astype(np.float64)
    vt = session.vtype
    out, kinks = [], []
    sign0 = None
    for i in voxels:
        vals, signs = [], []
        steps = []
        for sgn in (1.0, -1.0):
            kp = kappa32.copy()
            kp[i] = np.float32(kappa32[i] + np.float32(sgn * h))
            steps.append(float(kp[i]) - float(kappa32[i]))
            rows = _local_rhs(session.dims, k64, vt, phi0, i, float(kp[i]))
            rhs = np.zeros(session.n, np.float32)
            for r, v in rows.items():
                rhs[r] = v
            delta = session.solve(kp, rhs, tag=("fd", i, sgn))
            ph = phi0 + delta
            vals.append(loss_fn(ph, kp.astype(np.float64)))
            signs.append(ph)
        out.append((vals[0] - vals[1]) / (steps[0] - steps[1]))
        kinks.append(_kink(session.dims, vt, signs[0], signs[1]))
    return np.array(out), np.array(kinks)


def _kink(dims, vtype, pa, pb):
    lx, ly, lz = dims
    t = np.asarray(vtype).reshape(lz, ly, lx)
    A = np.where(t == 1, pa.reshape(lz, ly, lx), 0.0)
    B = np.where(t == 1, pb.reshape(lz, ly, lx), 0.0)
    for si, sj, _ in _pairs(dims):
        ok = (t[si] != 0) & (t[sj] != 0)
        ua, ub = A[sj] - A[si], B[sj] - B[si]
        if np.any(ok & (np.sign(ua) != np.sign(ub))):
            return True
    return False
