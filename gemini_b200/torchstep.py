"""A pure-tensor FP64 transcription of one fluid-advance step (torch ops only).

This is the differentiable stand-in of the CUDA step: the same discrete function
(advec.f90:21-447 boundaries, interface velocities and MC sweeps, multifluid.f90:179-233
conversions, 553-688 clean_param, 309-342 energy diffusion with collisions.f90:162-199
and PDEparabolic.f90:19-346, in the order of app/main.f90:280-355 without compression and
sources), written with out-of-place tensor operations so that torch.autograd can
differentiate it.  It serves two purposes: the checker of the hand-written adjoint (autograd
through this transcription on small grids) and, for pieces that have no CUDA adjoint
kernel, the step's vector-Jacobian product.

Conventions: a field is a tensor (S, X3, X2, X1) with X = l + 4 (two ghosts per side), the
C-order view of the reference's Fortran block (x1 fastest, species slowest).  Grids without
null points only (clean_param's null-cell overwrites are not differentiable data paths).
The time step is an input (a frozen schedule): dt_calc is not differentiated.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .state import AMU, ELCHRG, GAMMAS, KB, LSP, MS, QS

MINDENS, MINDENSNULL, MINDENSDIV = 1.0e-100, 1.0e-20, 1.0e-5
# collisions.f90:51-53 thermal_coeff: default-REAL literals widened to double
TCOEF = np.array([0.1019e-12, 0.0747e-12, 0.0754e-12, 0.0701e-12, 0.1068e-12, 0.3986e-12],
                 dtype=np.float32).astype(np.float64)


_CONST = {}


def _const(name, arr, device, shape):
    """Species constants as device tensors, created once per device (so that a captured
    CUDA graph of the step contains no host-to-device copy)."""
    import torch

    key = (name, str(device))
    t = _CONST.get(key)
    if t is None:
        t = torch.as_tensor(np.asarray(arr, dtype=np.float64), device=device).reshape(shape)
        _CONST[key] = t
    return t


@dataclass
class TGrid:
    """Grid metrics as tensors in the (X3, X2, X1) / face layouts."""

    lx1: int
    lx2: int
    lx3: int
    gridflag: int
    flagper: int
    dx: list       # per direction: dx(0..l+2)
    dxi: list      # per direction: dxi(1..l)
    h: list        # h1, h2, h3 ghosted (X3, X2, X1)
    hx: dict       # (metric k, family d) -> face tensor in the natural (i3, i2, i1) layout


def tgrid(grid, device="cpu") -> TGrid:
    import torch

    if grid.nullpts is not None and np.any(grid.nullpts):
        raise ValueError("the differentiable step supports grids without null points")

    def T(a):
        return torch.as_tensor(np.ascontiguousarray(np.asarray(a, dtype=np.float64).transpose()),
                               dtype=torch.float64, device=device)

    def V(a):
        return torch.as_tensor(np.asarray(a, dtype=np.float64), device=device)

    hx = {}
    for k in (1, 2, 3):
        for d in (1, 2, 3):
            hx[(k, d)] = T(getattr(grid, f"h{k}x{d}i"))
    return TGrid(grid.lx1, grid.lx2, grid.lx3, grid.gridflag, grid.flagper,
                 [V(grid.dx1), V(grid.dx2), V(grid.dx3)], [V(grid.dx1i), V(grid.dx2i), V(grid.dx3i)],
                 [T(grid.h1), T(grid.h2), T(grid.h3)], hx)


# ---- branch record ----------------------------------------------------------------------
# The step is piecewise smooth: it branches at the limiter (minmod), the upwind choice and the
# floors.  When BRANCHES is a list, every data-dependent branch decision of the step appends a
# digest of its mask (the count of taken branches and a sum of fixed pseudo-random 31-bit
# weights over them), so that two evaluations can be compared branch for branch: equal digest
# lists mean (barring a collision of ~2^-31 per site) that both took the same branches.
BRANCHES = None
_WEIGHTS = {}


def _digest(mask):
    import torch

    key = (mask.numel(), str(mask.device))
    w = _WEIGHTS.get(key)
    if w is None:
        g = torch.Generator(device="cpu").manual_seed(mask.numel())
        w = torch.randint(0, 2 ** 31, (mask.numel(),), generator=g, dtype=torch.int64).to(mask.device)
        _WEIGHTS[key] = w
    m = mask.reshape(-1).to(torch.int64)
    return int(m.sum()), int((m * w).sum())


def branch(mask):
    """Record a branch mask (when recording) and return it."""
    if BRANCHES is not None:
        BRANCHES.append(_digest(mask))
    return mask


def floor(x, lo):
    """torch.clamp(x, min=lo) with its branch recorded."""
    import torch

    branch(x < lo)
    return torch.clamp(x, min=lo)


# ---- helpers ---------------------------------------------------------------------------
def minmod(a, b):
    import torch

    z = torch.zeros_like(a)
    return torch.where(branch(a * b <= 0.0), z, torch.where(branch(a.abs() < b.abs()), a, b))


def _axis(dim):  # tensor axis of direction dim in (S, X3, X2, X1)
    return {1: 3, 2: 2, 3: 1}[dim]


def advec_line(f, v, dt, dx, dxi, ha1, ha2i, h1i, lx, axis):
    """advec.f90:384-435 along `axis` for every line at once.  f: ghosted along axis
    (-1..lx+2 at 0..lx+3); v, ha2i, h1i: faces 1..lx+1 along axis; ha1: cells (ghosted)."""
    import torch

    if lx <= 1:
        return f
    axis = axis - f.dim()  # right-aligned: the metric tensors have no species axis

    def sl(t, a, b):
        return t.narrow(axis, a, b - a)

    def bc(vec):  # 1-D tensor along axis -> broadcastable
        shape = [1] * (-axis)
        shape[0] = vec.numel()
        return vec.reshape(shape)

    F = lambda i0, i1: sl(f, i0 + 1, i1 + 1)  # f(i0 .. i1-1)
    dxv = bc(dx)
    # L(i) = (f(i)-f(i-1))/dx(i), R(i) = (f(i+1)-f(i))/dx(i+1), i = 0..lx+1
    Lsl = (F(0, lx + 2) - F(-1, lx + 1)) / sl(dxv, 0, lx + 2)
    Rsl = (F(1, lx + 3) - F(0, lx + 2)) / sl(dxv, 1, lx + 3)
    Csl = (F(1, lx + 3) - F(-1, lx + 1)) / (sl(dxv, 0, lx + 2) + sl(dxv, 1, lx + 3))
    slope = minmod(Csl, minmod(2 * Lsl, 2 * Rsl))  # slope(0..lx+1)
    # faces i = 1..lx+1
    dxf = sl(dxv, 1, lx + 2)
    s_i = sl(slope, 1, lx + 2)
    s_im1 = sl(slope, 0, lx + 1)
    f_i = F(1, lx + 2)
    f_im1 = F(0, lx + 1)
    neg = f_i * v - 0.5 * v * (dxf + v / h1i * dt) * s_i
    pos = f_im1 * v + 0.5 * v * (dxf - v / h1i * dt) * s_im1
    phi = torch.where(branch(v < 0), neg, pos)
    P = ha2i * phi
    upd = F(1, lx + 1) - dt * (sl(P, 1, lx + 1) - sl(P, 0, lx)) / bc(dxi) / sl(ha1, 2, lx + 2)
    return torch.cat([sl(f, 0, 2), upd, sl(f, lx + 2, lx + 4)], dim=axis)


def _rep(x, axis, lo, hi):
    """Write the edge values of a tensor ghosted along axis into its 2 ghost layers
    (copy of cell 1 into -1, 0 and of cell l into l+1, l+2)."""
    import torch

    n = x.shape[axis]
    e0 = x.narrow(axis, 2, 1)
    e1 = x.narrow(axis, n - 3, 1)
    mid = x.narrow(axis, 2, n - 4)
    return torch.cat([e0, e0, mid, e1, e1], dim=axis)


def _wrap3(x):
    """mpihalo.f90:147-151 self-wrap on x3 for the rows i2 = 1..lx2 (x1 including ghosts)."""
    import torch

    n3 = x.shape[1]
    lx3 = n3 - 4
    X2 = x.shape[2]
    core = x.narrow(2, 2, X2 - 4)
    lo = core.narrow(1, lx3, 2)      # i3 = lx3-1, lx3 -> ghosts -1, 0
    hi = core.narrow(1, 2, 2)        # i3 = 1, 2 -> ghosts lx3+1, lx3+2
    mid = core.narrow(1, 2, lx3)
    newcore = torch.cat([lo, mid, hi], dim=1)
    return torch.cat([x.narrow(2, 0, 2), newcore, x.narrow(2, X2 - 2, 2)], dim=2)


def sweep_field(G: TGrid, f, v, dim, frank, nsp, dt):
    """sweep{dim}_allspec of species 0..nsp-1 of the ghosted field f (S, X3, X2, X1) with the
    face velocities v (reference face layout as a tensor); the other species and every
    ghost cell pass through (advec.f90:283-381)."""
    import torch

    lx1, lx2, lx3 = G.lx1, G.lx2, G.lx3
    h1, h2, h3 = G.h
    hx = G.hx

    def ha1(fr):
        return (h1 * h1 * h2 * h3) if fr else (h1 * h2 * h3)

    if dim == 1:
        cell = ha1(0)[2:lx3 + 2, 2:lx2 + 2, :]
        ha2 = hx[(2, 1)] * hx[(3, 1)]
        h1i = hx[(1, 1)]
        core = f[:nsp, 2:lx3 + 2, 2:lx2 + 2, :]
        out = advec_line(core, v[:nsp], dt, G.dx[0], G.dxi[0], cell, ha2, h1i, lx1, 3)
        top = f[:nsp]
        mid = torch.cat([top[:, 2:lx3 + 2, :2], out, top[:, 2:lx3 + 2, lx2 + 2:]], 2)
        top = torch.cat([top[:, :2], mid, top[:, lx3 + 2:]], 1)
        return torch.cat([top, f[nsp:]], 0)
    if dim == 2:
        cell = ha1(frank)[2:lx3 + 2, :, 2:lx1 + 2]
        ha2 = (hx[(1, 2)] * hx[(1, 2)] * hx[(3, 2)]) if frank else (hx[(1, 2)] * hx[(3, 2)])
        h1i = hx[(2, 2)]
        core = f[:nsp, 2:lx3 + 2, :, 2:lx1 + 2]
        out = advec_line(core, v[:nsp], dt, G.dx[1], G.dxi[1], cell, ha2, h1i, lx2, 2)
        top = f[:nsp]
        mid = torch.cat([top[:, 2:lx3 + 2, :, :2], out, top[:, 2:lx3 + 2, :, lx1 + 2:]], 3)
        top = torch.cat([top[:, :2], mid, top[:, lx3 + 2:]], 1)
        return torch.cat([top, f[nsp:]], 0)
    cell = ha1(frank)[:, 2:lx2 + 2, 2:lx1 + 2]
    ha2 = (hx[(1, 3)] * hx[(1, 3)] * hx[(2, 3)]) if frank else (hx[(1, 3)] * hx[(2, 3)])
    h1i = hx[(3, 3)]
    core = f[:nsp, :, 2:lx2 + 2, 2:lx1 + 2]
    out = advec_line(core, v[:nsp], dt, G.dx[2], G.dxi[2], cell, ha2, h1i, lx3, 1)
    top = f[:nsp]
    mid = torch.cat([top[:, :, 2:lx2 + 2, :2], out, top[:, :, 2:lx2 + 2, lx1 + 2:]], 3)
    top = torch.cat([top[:, :, :2], mid, top[:, :, lx2 + 2:]], 2)
    return torch.cat([top, f[nsp:]], 0)


# ---- the step ------------------------------------------------------------------------
def step(G: TGrid, ns, vs1, vs2, vs3, Ts, v1i_lo, v1i_hi, nn, Tn, J1, dt, Teinf, Ttop=None,
         diffsolvetype=2, diffusion=None, sweep_impl=None):
    """One fused step.  ns, vs1, Ts: (7, X3, X2, X1); vs2, vs3 likewise (inputs only);
    v1i_lo / v1i_hi: the x1 boundary faces of vs1i from the previous step, (7, lx3, lx2);
    nn: (3, lx3, lx2, lx1); Tn: (lx3, lx2, lx1); J1: (X3, X2, X1); Ttop: optional per-column
    top Dirichlet temperature (lx3, lx2) replacing Teinf; diffusion: optional replacement of
    energy_diffusion, called as diffusion(n, T, Ttop) (e.g. a function with a hand-written
    adjoint); sweep_impl: optional replacement of the field sweeps, called as
    sweep_impl(f, v, dim, frank, nsp) with the face velocities v of direction dim.  Returns
    (ns, vs1, Ts, v1i_lo, v1i_hi) after the step."""
    import torch

    lx1, lx2, lx3 = G.lx1, G.lx2, G.lx3
    dev = ns.device
    ms = _const("ms", MS, dev, (7, 1, 1, 1))
    qs = _const("qs", QS, dev, (7, 1, 1, 1))
    gam = _const("gam", GAMMAS, dev, (7, 1, 1, 1))
    h1, h2, h3 = G.h
    # v12rhov1, T2rhoe (multifluid.f90:193-214)
    rv = ns * ms * vs1
    re = ns * KB * Ts / (gam - 1)

    # ---- set_global_boundaries (advec.f90:21-149) on n, rv, re, v2, v3
    I = slice(2, lx1 + 2)
    n_c = ns.narrow(3, 2, lx1)
    # x1 min: n ghosts by the ratio extrapolation (interior rows; the x2/x3 ghost rows follow
    # from the x2/x3 copies below)
    coeff_lo = ns[..., 3] / ns[..., 4]
    n0 = torch.minimum(coeff_lo * ns[..., 2], ns[..., 2])
    branch(coeff_lo * ns[..., 2] < ns[..., 2])
    nm1 = torch.minimum(coeff_lo * n0, n0)
    branch(coeff_lo * n0 < n0)
    coeff_hi = ns[..., lx1] / ns[..., lx1 - 1]
    nl1 = torch.minimum(coeff_hi * ns[..., lx1 + 1], ns[..., lx1 + 1])
    branch(coeff_hi * ns[..., lx1 + 1] < ns[..., lx1 + 1])
    nl2 = torch.minimum(coeff_hi * nl1, nl1)
    branch(coeff_hi * nl1 < nl1)
    n = torch.cat([nm1.unsqueeze(3), n0.unsqueeze(3), n_c, nl1.unsqueeze(3), nl2.unsqueeze(3)], dim=3)
    # rho v1 ghosts: reflection of the stale boundary faces, times n ms
    pad = lambda t: torch.nn.functional.pad(t, (2, 2, 2, 2))  # (7, lx3, lx2) -> (7, X3, X2)
    v1_1 = vs1[..., 2]
    v1_l = vs1[..., lx1 + 1]
    inner = torch.zeros_like(v1_1, dtype=torch.bool)
    inner[:, 2:lx3 + 2, 2:lx2 + 2] = True
    rv0 = torch.where(inner, 2 * pad(v1i_lo) - v1_1, rv[..., 1])
    rvm1 = rv0 + rv0 - v1_1
    rvl1 = torch.where(inner, 2 * pad(v1i_hi) - v1_l, rv[..., lx1 + 2])
    rvl2 = rvl1 + rvl1 - v1_l
    rv = torch.cat([(rvm1 * n[..., 0] * ms[..., 0]).unsqueeze(3), (rv0 * n[..., 1] * ms[..., 0]).unsqueeze(3),
                    rv.narrow(3, 2, lx1),
                    (rvl1 * n[..., lx1 + 2] * ms[..., 0]).unsqueeze(3), (rvl2 * n[..., lx1 + 3] * ms[..., 0]).unsqueeze(3)],
                   dim=3)
    Tb0 = re[..., 2] / n[..., 2]
    Tbl = re[..., lx1 + 1] / n[..., lx1 + 1]
    re = torch.cat([(Tb0 * n[..., 0]).unsqueeze(3), (Tb0 * n[..., 1]).unsqueeze(3), re.narrow(3, 2, lx1),
                    (Tbl * n[..., lx1 + 2]).unsqueeze(3), (Tbl * n[..., lx1 + 3]).unsqueeze(3)], dim=3)
    # x2 copies (never periodic), then x3 copies or the periodic self-wrap
    v2 = _rep(vs2, 2, 0, 0)
    n = _rep(n, 2, 0, 0)
    rv = _rep(rv, 2, 0, 0)
    re = _rep(re, 2, 0, 0)
    v3 = vs3
    if not G.flagper:
        v3 = _rep(v3, 1, 0, 0)
        n = _rep(n, 1, 0, 0)
        rv = _rep(rv, 1, 0, 0)
        re = _rep(re, 1, 0, 0)
    else:  # halo_fluidvars: the self-wrap of n, rv, re, v2, v3
        n, rv, re, v2, v3 = (_wrap3(t) for t in (n, rv, re, v2, v3))

    # ---- interface_vels (advec.f90:155-229)
    v1c = vs1[:, 2:lx3 + 2, 2:lx2 + 2, 2:lx1 + 2]
    mid = 0.5 * (v1c[..., :-1] + v1c[..., 1:])            # faces 2..lx1
    if G.gridflag == 1:
        f1 = torch.minimum(mid[..., :1], torch.zeros_like(mid[..., :1]))
        branch(mid[..., :1] < 0)
    else:
        f1 = v1c[..., :1]
    if G.gridflag == 2:
        fN = torch.maximum(mid[..., -1:], torch.zeros_like(mid[..., -1:]))
        branch(mid[..., -1:] > 0)
    else:
        fN = v1c[..., -1:]
    v1i = torch.cat([f1, mid, fN], dim=3)                   # (7, lx3, lx2, lx1+1)
    v2c = v2[:, 2:lx3 + 2, :, 2:lx1 + 2]
    v2i = 0.5 * (v2c[:, :, 1:lx2 + 2] + v2c[:, :, 2:lx2 + 3])  # (7, lx3, lx2+1, lx1)
    v3c = v3[:, :, 2:lx2 + 2, 2:lx1 + 2]
    v3i = 0.5 * (v3c[:, 1:lx3 + 2] + v3c[:, 2:lx3 + 3])    # (7, lx3+1, lx2, lx1)

    def sweep(f, dim, frank, nsp):
        return sweep_field(G, f, {1: v1i, 2: v2i, 3: v3i}[dim], dim, frank, nsp, dt)

    if sweep_impl is not None:
        vel = {1: v1i, 2: v2i, 3: v3i}

        def sweep(f, dim, frank, nsp):  # noqa: F811 -- the replacement
            return sweep_impl(f, vel[dim], dim, frank, nsp)

    n = sweep(n, 3, 0, 6)
    rv = sweep(rv, 3, 1, 6)
    re = sweep(re, 3, 0, 7)
    n = sweep(n, 1, 0, 6)
    rv = sweep(rv, 1, 0, 6)
    re = sweep(re, 1, 0, 7)
    if G.flagper:
        n, rv, re = _wrap3(n), _wrap3(rv), _wrap3(re)
    n = sweep(n, 2, 0, 6)
    rv = sweep(rv, 2, 1, 6)
    re = sweep(re, 2, 0, 7)

    # ---- rhov12v1 (multifluid.f90:218-233)
    v1 = rv[:6] / (ms[:6] * floor(n[:6], MINDENSDIV))
    chrg = (n[:6] * qs[:6] * v1)
    csum = chrg[0]
    for s in range(1, 6):
        csum = csum + chrg[s]
    nsum = n[0]
    for s in range(1, 6):
        nsum = nsum + n[s]
    ve = -1 / floor(nsum, MINDENSDIV) / qs[6] * csum
    v1 = torch.cat([v1, ve.unsqueeze(0)], 0)
    # clean_param(1): floors, electron sum, ghosts := 1e-5
    ni = floor(n[:6], MINDENS)
    ne = ni[0]
    for s in range(1, 6):
        ne = ne + ni[s]
    n = torch.cat([ni, ne.unsqueeze(0)], 0)
    ghost = torch.ones_like(n[0], dtype=torch.bool)
    ghost[2:lx3 + 2, 2:lx2 + 2, 2:lx1 + 2] = False
    n = torch.where(ghost, torch.full_like(n, MINDENSDIV), n)
    # rhoe2T + clean_param(3)
    T = floor((gam - 1) / KB * re / floor(n, MINDENSDIV), 100.0)
    T = torch.where(ghost, torch.full_like(T, 100.0), T)

    # ---- energy diffusion (multifluid.f90:309-342)
    if diffusion is None:
        T = energy_diffusion(G, n, T, J1, nn, Tn, dt, Teinf, Ttop, diffsolvetype)
    else:
        T = diffusion(n, T, Ttop)
    T = torch.where(ghost, torch.full_like(T, 100.0), floor(T, 100.0))
    return n, v1, T, v1i[..., 0], v1i[..., -1]


def pow25(x):
    import torch

    return torch.pow(x, 2.5)


def energy_diffusion(G: TGrid, n, T, J1, nn, Tn, dt, Teinf, Ttop=None, diffsolvetype=2):
    """thermal_conduct + diffusion_prep + TRBDF2/backward Euler per column, all species.
    Returns T (7, X3, X2, X1) with the interior replaced and max(T,100) applied."""
    import torch

    lx1, lx2, lx3 = G.lx1, G.lx2, G.lx3
    h1, h2, h3 = (h[2:lx3 + 2, 2:lx2 + 2, 2:lx1 + 2] for h in G.h)
    Tc = T[:, 2:lx3 + 2, 2:lx2 + 2, 2:lx1 + 2]
    nc = n[:, 2:lx3 + 2, 2:lx2 + 2, 2:lx1 + 2]
    tco = _const("tcoef", TCOEF, T.device, (6, 1, 1, 1))
    lam_i = tco * pow25(Tc[:6])
    te = Tc[6]
    X = nn[0] * 1.1e-16 * (1 + 5.7e-4 * te) + nn[1] * 2.82e-17 * torch.sqrt(te) * (1 - 1.21e-4 * te) + \
        nn[2] * 2.2e-16 * (1 + 3.6e-2 * torch.sqrt(te))
    lam_e = ELCHRG * 100 * 7.7e5 * pow25(te) / (1 + 3.22e4 * (te * te) / nc[6] * X)
    lam = torch.cat([lam_i, lam_e.unsqueeze(0)], 0)
    beta = torch.zeros_like(lam)
    beta = torch.cat([beta[:6], (5.0 / 2 * KB / ELCHRG * J1[2:lx3 + 2, 2:lx2 + 2, 2:lx1 + 2]).unsqueeze(0)], 0)
    gam = _const("gam", GAMMAS, T.device, (7, 1, 1, 1))
    C = (gam - 1.0) / KB / floor(nc, MINDENSDIV) / (h1 * h2 * h3)
    B = C * beta / h1
    D = lam * h2 * h3 / h1
    # Dirichlet values (diffusion.f90:54-79)
    tn1, tnl = Tn[..., 0], Tn[..., -1]
    top = Ttop if Ttop is not None else torch.full_like(tn1, float(Teinf))
    if G.gridflag == 0:
        tmin, tmax = tn1, tnl
    elif G.gridflag == 1:
        tmin, tmax = top, tnl
    else:
        tmin, tmax = tn1, top
    tmin = tmin.unsqueeze(0).expand(7, lx3, lx2)
    tmax = tmax.unsqueeze(0).expand(7, lx3, lx2)
    dx = G.dx[0]
    dxi = G.dxi[0]
    # rows i = 2..lx1-1 (1-based): Dh(i) = 0.5*(D(i-1)+D(i))
    Dh = 0.5 * (D[..., :-1] + D[..., 1:])                  # Dh(2..lx1)
    Ci = C[..., 1:lx1 - 1]
    Bi = B[..., 1:lx1 - 1]
    Dhm = Dh[..., 0:lx1 - 2]                               # Dh(i)
    Dhp = Dh[..., 1:lx1 - 1]                               # Dh(i+1)
    dxm = dx[2:lx1]                                        # dx(i)
    dxp = dx[3:lx1 + 1]                                    # dx(i+1)
    dxii = dxi[1:lx1 - 1]
    qm = Ci * Dhm / dxii / dxm
    qp = Ci * Dhp / dxii / dxp
    bq = Bi / (dxp + dxm)
    Tin = Tc[..., 1:lx1 - 1]
    Tm = Tc[..., 0:lx1 - 2]
    Tp = Tc[..., 2:lx1]

    def solve(a, b, c, r):
        """Tridiagonal solve over x1 with Dirichlet (identity) rows 1 and lx1."""
        one = torch.ones_like(tmin).unsqueeze(-1)
        zero = torch.zeros_like(one)
        A = torch.cat([zero, a, zero], -1)
        Bd = torch.cat([one, b, one], -1)
        Cd = torch.cat([zero, c, zero], -1)
        R = torch.cat([tmin.unsqueeze(-1), r, tmax.unsqueeze(-1)], -1)
        return thomas(A, Bd, Cd, R)

    if diffsolvetype == 2:
        a = -(qm / 2) + bq / 2
        b = 1 / (dt / 2) + qp / 2 + qm / 2
        c = -(qp / 2) - bq / 2
        Pd = qp / 2 + qm / 2
        r = Tin / (dt / 2) - a * Tm - Pd * Tin - c * Tp
        TR = solve(a, b, c, r)
        a2 = -qm + bq
        b2 = 1 / (dt / 3) + qp + qm
        c2 = -qp - bq
        r2 = -(1 / 3.0 * Tin / (dt / 3)) + 4 / 3.0 * TR[..., 1:lx1 - 1] / (dt / 3)
        out = solve(a2, b2, c2, r2)
    else:
        a = -qm + bq
        b = 1 / dt + qp + qm
        c = -qp - bq
        out = solve(a, b, c, Tin / dt)
    # place the x1 Dirichlet ghosts (layers 0, lx1+1) and the interior
    lo = tmin.unsqueeze(-1)
    hi = tmax.unsqueeze(-1)
    rows = torch.cat([T[:, 2:lx3 + 2, 2:lx2 + 2, 0:1], lo, out, hi, T[:, 2:lx3 + 2, 2:lx2 + 2, lx1 + 3:]], -1)
    mid = torch.cat([T[:, 2:lx3 + 2, :2], rows, T[:, 2:lx3 + 2, lx2 + 2:]], 2)
    Tfull = torch.cat([T[:, :2], mid, T[:, lx3 + 2:]], 1)
    return floor(Tfull, 100.0)


def thomas(a, b, c, r):
    """Tridiagonal solve along the last axis (no pivoting), differentiable."""
    import torch

    n = r.shape[-1]
    cp = [None] * n
    dp = [None] * n
    cp[0] = c[..., 0] / b[..., 0]
    dp[0] = r[..., 0] / b[..., 0]
    for i in range(1, n):
        den = b[..., i] - a[..., i] * cp[i - 1]
        cp[i] = c[..., i] / den
        dp[i] = (r[..., i] - a[..., i] * dp[i - 1]) / den
    x = [None] * n
    x[n - 1] = dp[n - 1]
    for i in range(n - 2, -1, -1):
        x[i] = dp[i] - cp[i] * x[i + 1]
    return torch.stack(x, -1)
