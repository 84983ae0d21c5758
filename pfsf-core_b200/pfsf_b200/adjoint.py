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


_FACES = ((-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1))


def _shift(a, dx, dy, dz, fill=0.0):
    """b[z, y, x] = a[z + dz, y + dy, x + dx], fill outside the box."""
    b = torch.full_like(a, fill)
    lz, ly, lx = a.shape

    def rng(d, n):
        return (slice(0, n - 1), slice(1, n)) if d == 1 else ((slice(1, n), slice(0, n - 1)) if d == -1 else
                                                             (slice(0, n), slice(0, n)))
    (zo, zi), (yo, yi), (xo, xi) = rng(dz, lz), rng(dy, ly), rng(dx, lx)
    b[zo, yo, xo] = a[zi, yi, xi]
    return b


def amor_psi(phi, kappa, vtype, dims):
    """Elastic energy density with the Amor split, as the history update
    H = max(H, psi_e) computes it (SH/rbgs_smooth.comp.glsl:177-191, the
    library's k_history): psi_e = phi^2 / 2, times 0.01 where the face inflow
    exceeds three times the face outflow; flows over the six faces with the
    face conductivity = the harmonic-mean kappa link value; solid voxels with
    phi > 0 only (0 elsewhere).  Differentiable in phi (piecewise)."""
    lx, ly, lz = dims
    t = torch.as_tensor(np.asarray(vtype), device=phi.device).reshape(lz, ly, lx)
    k = kappa.reshape(lz, ly, lx).to(phi.dtype)
    p = torch.where(t == 1, phi.reshape(lz, ly, lx), torch.zeros((), dtype=phi.dtype, device=phi.device))
    fin = torch.zeros_like(p)
    fout = torch.zeros_like(p)
    for dx, dy, dz in _FACES:
        kj = _shift(k, dx, dy, dz)
        tj = _shift(t, dx, dy, dz, 0)
        pj = _shift(p, dx, dy, dz)
        ok = (t != 0) & (tj != 0) & ((k + kj) > 0)
        sig = torch.where(ok, 2.0 * k * kj / torch.where(ok, k + kj, torch.ones_like(k)), torch.zeros_like(k))
        flow = sig * (pj - p)
        fin = fin + torch.relu(flow)
        fout = fout + torch.relu(-flow)
    factor = torch.where(fin > 3.0 * fout, torch.full_like(p, 0.01), torch.ones_like(p))
    psi = 0.5 * p * p * factor
    return torch.where((t == 1) & (p > 0), psi, torch.zeros_like(psi)).reshape(-1)


def _device(device):
    if device is not None:
        return torch.device(device)
    return torch.device("cuda") if torch.cuda.is_available() else torch.device("cpu")


def trajectory_objective(phis, kappa, vtype, dims, rcomp, phi_target, ramp=2.0, h_scale=1.0, device=None):
    """The config-4 calibration loss of a given trajectory phi_0..phi_{T-1}
    (tick t under the load f_t, ramped linearly from 1 to `ramp`):

        L = sum_t [ sum_solid softplus(flux_in(phi_t) / rcomp - 1)
                    + 1/2 sum_solid (phi_t - f_t phi_target)^2 ]
          + sum_solid softplus(H / h_scale - 1),   H = max_t psi_e(phi_t)

    (psi_e: amor_psi, the history the phase field reads), as torch ops on
    `device` (the GPU by default).  Returns (L, H)."""
    dev = _device(device)
    ticks = len(phis)
    kd = torch.as_tensor(kappa, device=dev, dtype=torch.float64) if not torch.is_tensor(kappa) else kappa.to(dev)
    rc = torch.as_tensor(rcomp, device=dev, dtype=torch.float64)
    pt = torch.as_tensor(phi_target, device=dev, dtype=torch.float64)
    solid = torch.as_tensor(np.asarray(vtype) == 1, device=dev)
    L = torch.zeros((), dtype=torch.float64, device=dev)
    H = torch.zeros(int(np.prod(dims)), dtype=torch.float64, device=dev)
    for t, phi in enumerate(phis):
        f = 1.0 + (ramp - 1.0) * t / max(ticks - 1, 1)
        pd = (phi if torch.is_tensor(phi) else torch.as_tensor(phi, dtype=torch.float64)).to(dev)
        L = L + calibration_loss(pd, kd, vtype, dims, rc, f * pt)
        H = torch.maximum(H, amor_psi(pd, kd, vtype, dims))
    z = H / h_scale - 1.0
    L = L + torch.where(solid, torch.nn.functional.softplus(z), torch.zeros_like(z)).sum()
    return L, H


def trajectory_loss(session, kappa, source, rcomp, phi_target, ticks=32, ramp=2.0, checkpoint_every=8,
                    h_scale=1.0, device=None):
    """Solves the ramped trajectory (tick t: A(kappa) phi_t = f_t s, a
    checkpoint of phi every `checkpoint_every` ticks) and returns
    (trajectory_objective, phis, H).  Every tick enters the gradient:
    backward runs each tick's adjoint in reverse order, and the device holds
    only the last tick's solution, so every earlier tick is re-solved from
    its checkpoint first (Session.recomputes counts them)."""
    checkpoints = {}
    phis = []
    warm = None
    for t in range(ticks):
        f = 1.0 + (ramp - 1.0) * t / max(ticks - 1, 1)
        base = checkpoints.get(checkpoint_every * (t // checkpoint_every))
        phi = KappaSolve.apply(kappa, source * f, session, t, warm if base is None else base)
        x = phi.detach().numpy()
        if t % checkpoint_every == 0:
            checkpoints[t] = x.astype(np.float32)
        warm = x.astype(np.float32)
        phis.append(phi)
    L, H = trajectory_objective(phis, kappa, session.vtype, session.dims, rcomp, phi_target, ramp, h_scale, device)
    return L, phis, H


def trajectory_finite_difference(session, kappa32, source32, phis0, rcomp, phi_target, voxels, ramp=2.0,
                                 h_scale=1.0, h=2.0 ** -10, device=None):
    """Central differences of trajectory_objective w.r.t. kappa_i at each
    voxel i: every tick's perturbed solution is phi0_t + delta_t with
    A(kappa') delta_t = -(A(kappa') - A(kappa)) phi0_t (see
    finite_difference_kappa), the whole trajectory's loss evaluated at
    kappa +/- h e_i.  Returns (fd, kink flags): a kink flag marks a voxel
    whose +/- trajectories differ in a link's inflow side, a voxel's psi_e
    switch or the tick that attains the history maximum."""
    ticks = len(phis0)
    k64 = kappa32.astype(np.float64)
    vt = session.vtype
    out, kinks = [], []
    for i in voxels:
        vals, trajs, steps = [], [], []
        for sgn in (1.0, -1.0):
            kp = kappa32.copy()
            kp[i] = np.float32(kappa32[i] + np.float32(sgn * h))
            steps.append(float(kp[i]) - float(kappa32[i]))
            traj = []
            for t in range(ticks):
                rows = _local_rhs(session.dims, k64, vt, phis0[t], i, float(kp[i]))
                rhs = np.zeros(session.n, np.float32)
                for r, v in rows.items():
                    rhs[r] = v
                traj.append(phis0[t] + session.solve(kp, rhs, tag=("fd", i, sgn, t)))
            with torch.no_grad():
                L, H = trajectory_objective(traj, kp.astype(np.float64), vt, session.dims, rcomp, phi_target, ramp,
                                            h_scale, device)
            vals.append(float(L))
            trajs.append((traj, kp))
        out.append((vals[0] - vals[1]) / (steps[0] - steps[1]))
        kink = any(_kink(session.dims, vt, a, b) for a, b in zip(trajs[0][0], trajs[1][0]))
        if not kink:
            kink = _history_kink(session, trajs[0], trajs[1], device)
        kinks.append(kink)
    return np.array(out), np.array(kinks)


def _history_kink(session, ta, tb, device):
    """The +/- trajectories differ in a psi_e switch or the argmax tick."""
    pats = []
    for traj, kp in (ta, tb):
        kd = torch.as_tensor(kp.astype(np.float64), device=_device(device))
        psis = torch.stack([amor_psi(torch.as_tensor(p, dtype=torch.float64, device=kd.device), kd, session.vtype,
                                     session.dims) for p in traj])
        sq = torch.stack([0.5 * torch.as_tensor(p, dtype=torch.float64, device=kd.device) ** 2 for p in traj])
        switched = (psis < 0.5 * sq).cpu().numpy()
        pats.append((switched, torch.argmax(psis, dim=0).cpu().numpy()))
    return bool(np.any(pats[0][0] != pats[1][0]) or np.any(pats[0][1] != pats[1][1]))


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
