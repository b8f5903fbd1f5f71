"""The oracle's source/loss solves (multifluid.f90:474-549 with ETD_uncoupled,
calculus.in.f90:174-196), given production and loss rates, checked on the CPU: the
exponential-time-differencing limits, a numpy statement of the update, and the bookkeeping
each routine does after it (electron density, velocities, temperatures).  The rates come
from sources.f90, which is not restated yet; the reference ships no test of these solves."""
import math

import numpy as np

import oracle as O
from gemini_b200 import grid as G
from gemini_b200 import state as S

LSP = 7


def test_etd_limits_and_statement():
    rng = np.random.default_rng(2)
    n = 4000
    f = rng.uniform(1e8, 1e12, n)
    P = rng.uniform(0, 1e9, n)
    L = np.where(rng.uniform(size=n) < 0.3, 0.0, 10 ** rng.uniform(-14, 2, n))
    dt = 0.25
    out = O.etd_uncoupled(f, P, L, dt)
    Ldt = L * dt
    # the C library's exp, as the oracle (and gfortran) call it: 1 - exp(-Ldt) cancels just
    # above the 1e-10 cut, so an exp one ulp apart moves the result by ~1e-9 there
    e = np.array([math.exp(-1.0 * x) for x in Ldt])
    want = np.where(Ldt > 1e-10, f * e + P / np.where(L > 0, L, 1.0) * (1 - e), f + P * dt)
    assert np.array_equal(out, want)
    small = Ldt <= 1e-10
    assert np.array_equal(out[small], f[small] + P[small] * dt)  # explicit Euler below the cut
    big = Ldt > 50
    np.testing.assert_allclose(out[big], P[big] / L[big], rtol=1e-14)  # equilibrium P/L


def _rates(g, seed):
    rng = np.random.default_rng(seed)
    shp = (g.lx1, g.lx2, g.lx3, LSP)
    Pr = np.asfortranarray(rng.uniform(0, 1e6, shp))
    Lo = np.asfortranarray(10 ** rng.uniform(-6, 0, shp))
    return Pr, Lo, rng


def test_mass_source_loss_solve():
    g = G.dipole_grid(14, 5, 4)
    st = S.init_state(g, seed=3, perturb=0.2)
    Pr, Lo, rng = _rates(g, 5)
    Prp = np.asfortranarray(rng.uniform(0, 1e5, (g.lx1, g.lx2, g.lx3, LSP - 1)))
    ns0 = st.fluidvars[..., 0:LSP].copy()
    dt = 0.1
    Pr_out = O.mass_source_loss_solve(g, st, dt, Pr, Lo, Prp)
    ns = st.fluidvars[..., 0:LSP]
    I = (slice(2, g.lx1 + 2), slice(2, g.lx2 + 2), slice(2, g.lx3 + 2))
    assert np.array_equal(Pr_out[..., :LSP - 1], Pr[..., :LSP - 1] + Prp)
    for s in range(LSP - 1):
        want = O.etd_uncoupled(ns0[I + (s,)], Pr_out[..., s], Lo[..., s], dt)
        assert np.array_equal(np.ascontiguousarray(ns[I + (s,)]).ravel(), want)
    # ghosts of the ions untouched; electrons are the ion sum everywhere (ghosts included)
    ghost = np.ones(ns.shape[:3], bool)
    ghost[I] = False
    assert np.array_equal(ns[ghost][:, :LSP - 1], ns0[ghost][:, :LSP - 1])
    esum = ns[..., 0].copy()
    for s in range(1, LSP - 1):
        esum = esum + ns[..., s]
    assert np.array_equal(ns[..., LSP - 1], esum)


def test_momentum_source_loss_solve():
    g = G.cartesian_grid(12, 4, 5)
    st = S.init_state(g, seed=4, perturb=0.1)
    O.v12rhov1(g, st)
    Pr, Lo, _ = _rates(g, 6)
    O.momentum_source_loss_solve(g, st, 0.05, Pr * 1e-20, Lo)
    ms, qs, _, _ = O.constants()
    ns = st.fluidvars[..., 0:LSP]
    vs1 = st.fluidvars[..., LSP:2 * LSP]
    rv = st.fluidauxvars[..., 0:LSP]
    for s in range(LSP - 1):
        assert np.array_equal(vs1[..., s], rv[..., s] / (ms[s] * np.maximum(ns[..., s], 1e-5)))
    chrg = ns[..., 0] * qs[0] * vs1[..., 0]
    for s in range(1, LSP - 1):
        chrg = chrg + ns[..., s] * qs[s] * vs1[..., s]
    ve = -1 / np.maximum(ns[..., LSP - 1], 1e-5) / qs[LSP - 1] * chrg
    assert np.array_equal(vs1[..., LSP - 1], ve)
    assert np.array_equal(rv[..., LSP - 1], ns[..., LSP - 1] * ms[LSP - 1] * ve)


def test_energy_source_loss_solve():
    g = G.dipole_grid(12, 4, 4)
    st = S.init_state(g, seed=8, perturb=0.2)
    O.T2rhoe(g, st)
    Pr, Lo, rng = _rates(g, 9)
    Pr *= 1e-12
    Qe = np.asfortranarray(rng.uniform(0, 1e-13, (g.lx1, g.lx2, g.lx3)))
    re0 = st.fluidauxvars[..., LSP:2 * LSP].copy()
    Pr_out = O.energy_source_loss_solve(g, st, 0.1, Pr, Lo, Qe)
    assert np.array_equal(Pr_out[..., LSP - 1], Pr[..., LSP - 1] + Qe)
    assert np.array_equal(Pr_out[..., :LSP - 1], Pr[..., :LSP - 1])
    _, _, gam, _ = O.constants()
    kB = 1.38064852e-23
    ns = st.fluidvars[..., 0:LSP]
    re = st.fluidauxvars[..., LSP:2 * LSP]
    Ts = st.fluidvars[..., 4 * LSP:5 * LSP]
    for s in range(LSP):
        assert np.array_equal(Ts[..., s], np.maximum((gam[s] - 1) / kB * re[..., s] / np.maximum(ns[..., s], 1e-5), 100.0))
    assert not np.array_equal(re, re0)
    assert (Ts >= 100.0).all()


def _neutrals(g, seed, scale=1.0):
    rng = np.random.default_rng(seed)
    shp = (g.lx1, g.lx2, g.lx3)
    nn = np.asfortranarray(np.stack([10 ** rng.uniform(10, 16, shp) for _ in range(7)], axis=-1) * scale)
    vn = [np.asfortranarray(rng.uniform(-100, 100, shp)) for _ in range(3)]
    Tn = np.asfortranarray(rng.uniform(200, 1500, shp))
    return nn, vn, Tn


def _recombination(ns, Ts):
    """The five electron recombination rates of srcsContinuity (per ion density), with the C
    library's pow."""
    pw = np.vectorize(math.pow)
    ne, Te = ns[..., LSP - 1], Ts[..., LSP - 1]
    o2 = np.where(Te <= 1200, 1.95e-7 * pw(300 / Te, 0.70), 7.38e-8 * pw(1200 / Te, 0.56))
    return {0: 3.7e-12 * pw(250 / Te, 0.7) * ne * 1e-6, 1: 4.2e-7 * pw(300 / Te, 0.85) * ne * 1e-6,
            2: 1.8e-7 * pw(300 / Te, 0.39) * ne * 1e-6, 3: o2 * ne * 1e-6,
            5: 3.7e-12 * pw(250 / Te, 0.7) * ne * 1e-6}


def test_srcs_continuity_with_no_neutrals_is_recombination_alone():
    g = G.dipole_grid(10, 4, 3)
    st = S.init_state(g, seed=2, perturb=0.3)
    nn, vn, Tn = _neutrals(g, 1, scale=0.0)
    Pr, Lo = O.srcs_continuity(g, st, nn, *vn, Tn)
    I = (slice(2, g.lx1 + 2), slice(2, g.lx2 + 2), slice(2, g.lx3 + 2))
    rec = _recombination(st.fluidvars[I + (slice(0, LSP),)], st.fluidvars[I + (slice(4 * LSP, 5 * LSP),)])
    assert not Pr.any()
    for s in range(LSP):
        assert np.array_equal(Lo[..., s], rec.get(s, np.zeros_like(Lo[..., s])))


def test_srcs_continuity_n_atoms_alone():
    """With only atomic nitrogen, O2+ + N --> NO+ + O is the one ion-neutral reaction."""
    g = G.cartesian_grid(9, 4, 3)
    st = S.init_state(g, seed=5, perturb=0.2)
    nn, vn, Tn = _neutrals(g, 2)
    nn[..., [0, 1, 2, 3, 5, 6]] = 0.0
    Pr, Lo = O.srcs_continuity(g, st, nn, *vn, Tn)
    I = (slice(2, g.lx1 + 2), slice(2, g.lx2 + 2), slice(2, g.lx3 + 2))
    ns = st.fluidvars[I + (slice(0, LSP),)]
    beta = 1.2e-10 * nn[..., 4] * 1e-6
    assert np.array_equal(Pr[..., 1], 0.0 + beta * ns[..., 3])
    rec = _recombination(ns, st.fluidvars[I + (slice(4 * LSP, 5 * LSP),)])
    assert np.array_equal(Lo[..., 3], (0.0 + beta) + rec[3])
    assert not Pr[..., [0, 2, 3, 4, 5, 6]].any()


def test_srcs_continuity_conserves_ions_up_to_recombination():
    """Every ion-neutral reaction moves density from one ion species to another, so the
    ions' total production minus loss is minus the electron recombination alone."""
    for mk, seed in ((lambda: G.dipole_grid(16, 5, 4), 3), (lambda: G.cartesian_grid(12, 5, 4), 4)):
        g = mk()
        st = S.init_state(g, seed=seed, perturb=0.3)
        I = (slice(2, g.lx1 + 2), slice(2, g.lx2 + 2), slice(2, g.lx3 + 2))
        fv = st.fluidvars
        rng = np.random.default_rng(seed)
        fv[I + (slice(LSP, 2 * LSP),)] = rng.uniform(-2000, 2000, fv[I + (slice(LSP, 2 * LSP),)].shape)
        nn, vn, Tn = _neutrals(g, seed)
        Pr, Lo = O.srcs_continuity(g, st, nn, *vn, Tn)
        ns = fv[I + (slice(0, LSP),)]
        rec = _recombination(ns, fv[I + (slice(4 * LSP, 5 * LSP),)])
        net = np.zeros(ns.shape[:3])
        scale = np.zeros(ns.shape[:3])
        for s in range(LSP - 1):
            net = net + Pr[..., s] - Lo[..., s] * ns[..., s]
            scale = scale + Pr[..., s] + Lo[..., s] * ns[..., s]
        for s, r in rec.items():
            net = net + r * ns[..., s]
        assert (np.abs(net) <= 1e-13 * scale).all()
        assert (Pr >= 0).all() and (Lo >= 0).all()


# ---- srcsEnergy: an independent, vectorised numpy statement (C library functions) ----------

_F32 = lambda rows: np.array(rows, dtype=np.float32).astype(np.float64)
_CSN = _F32([[-1, 6.82e-10, 6.64e-10, -1], [2.44e-10, 4.34e-10, 4.27e-10, 0.69e-10],
             [2.58e-10, -1, 4.49e-10, 0.74e-10], [2.31e-10, 4.13e-10, -1, 0.65e-10],
             [4.42e-10, 7.47e-10, 7.25e-10, 1.45e-10], [-1, 33.6e-10, 32.0e-10, -1], [-1, -1, -1, -1]])
_C2SN1 = _F32([[3.67e-11, 0, 0, 4.63e-12], [0, 0, 0, 0], [0, 5.14e-11, 0, 0], [0, 0, 2.59e-11, 0],
               [0, 0, 0, 0], [6.61e-11, 0, 0, 2.65e-10], [-1, -1, -1, -1]])
_C2SN2 = _F32([[0.064, 0, 0, -1], [0, 0, 0, 0], [0, 0.069, 0, 0], [0, 0, 0.073, 0], [0, 0, 0, 0],
               [0.047, 0, 0, 0.083], [-1, -1, -1, -1]])
_CSJ = _F32([[0.22, 0.26, 0.25, 0.26, 0.22, 0.077, 1.87e-3], [0.14, 0.16, 0.16, 0.17, 0.13, 0.042, 9.97e-4],
             [0.15, 0.17, 0.17, 0.18, 0.14, 0.045, 1.07e-3], [0.13, 0.16, 0.15, 0.16, 0.12, 0.039, 9.347e-4],
             [0.25, 0.28, 0.28, 0.28, 0.24, 0.088, 2.136e-3], [1.23, 1.25, 1.25, 1.25, 1.23, 0.90, 29.7e-3],
             [54.5, 54.5, 54.5, 54.5, 54.5, 54.5, 38.537]])
_AMU, _KB, _EL = 1.660539040e-27, 1.38064852e-23, 1.60217662e-19
_MN = np.array([16.0, 28.0, 32.0, 1.0]) * _AMU
_V = {n: np.vectorize(getattr(math, n)) for n in ("pow", "erf", "log10", "exp", "tanh", "sin", "sqrt")}


def _np_maxwell(isp, j, nnj, tn, ts):
    pw = _V["pow"]
    if isp < LSP - 1:
        if _CSN[isp, j] < 0:
            if isp == 0 and j == 3:
                return _C2SN1[isp, j] * pw(tn + ts / 16, 0.5) * nnj * 1e-6
            te = 0.5 * (tn + ts)
            a = 1 - _C2SN2[isp, j] * _V["log10"](te)
            return _C2SN1[isp, j] * (a * a) * pw(te, 0.5) * nnj * 1e-6
        return _CSN[isp, j] * nnj * 1e-6
    te = ts
    r = [lambda: 8.9e-11 * (1.0 + 5.7e-4 * te) * pw(te, 0.5), lambda: 2.33e-11 * (1.0 - 1.21e-4 * te) * te,
         lambda: 1.82e-10 * (1.0 + 3.6e-2 * pw(te, 0.5)) * pw(te, 0.5),
         lambda: 4.5e-9 * (1.0 - 1.35e-4 * te) * pw(te, 0.5)][j]()
    return r * nnj * 1e-6


def _np_coulomb(isp, t, ms, ns2, ts1, ts2, v1, v2):
    if isp == t:
        z = np.zeros_like(ts1)
        return z, z, z
    te = (ms[t] * ts1 + ms[isp] * ts2) / (ms[t] + ms[isp])
    nu = _CSJ[isp, t] * ns2 * 1e-6 / _V["pow"](te, 1.5)
    mred = ms[isp] * ms[t] / (ms[isp] + ms[t])
    W = np.abs(v1 - v2) / _V["sqrt"](2 * _KB * te / mred)
    psi = _V["exp"](-(W * W))
    with np.errstate(divide="ignore", invalid="ignore"):
        phi = np.where(W < 0.1, 1.0, 3.0 / 4 * math.sqrt(math.pi) * _V["erf"](W) / (W * W * W) - 3.0 / 2 / (W * W) * psi)
    return nu, phi, psi


def _np_srcs_energy(g, st, nn, vn1, vn2, vn3, Tn):
    ms, _, gam, _ = O.constants()
    I = (slice(2, g.lx1 + 2), slice(2, g.lx2 + 2), slice(2, g.lx3 + 2))
    fv = st.fluidvars
    ns, v1, v2, v3, Ts = (fv[I + (slice(k * LSP, (k + 1) * LSP),)] for k in range(5))
    Pr = np.zeros(ns.shape)
    Lo = np.zeros(ns.shape)
    for s in range(LSP):
        for j in range(4):
            nu = _np_maxwell(s, j, nn[..., j], Tn, Ts[..., s])
            fact = 2 * nu / (ms[s] + _MN[j])
            Pr[..., s] = Pr[..., s] + ns[..., s] * ms[s] * _KB / (gam[s] - 1) * fact * Tn
            Lo[..., s] = Lo[..., s] + ms[s] * fact
            fact = fact * _MN[j] / 3
            d = ((v1[..., s] - vn1) * (v1[..., s] - vn1) + (v2[..., s] - vn2) * (v2[..., s] - vn2)
                 + (v3[..., s] - vn3) * (v3[..., s] - vn3))
            Pr[..., s] = Pr[..., s] + ns[..., s] * ms[s] / (gam[s] - 1) * d * fact
        for t in range(LSP):
            nu, phi, psi = _np_coulomb(s, t, ms, ns[..., t], Ts[..., s], Ts[..., t], v1[..., s], v1[..., t])
            fact = 2 * nu * psi / (ms[s] + ms[t])
            Pr[..., s] = Pr[..., s] + ns[..., s] * ms[s] * _KB / (gam[s] - 1) * fact * Ts[..., t]
            Lo[..., s] = Lo[..., s] + ms[s] * fact
            fact = 2 * nu * phi / (ms[s] + ms[t]) * ms[t] / 3
            d = ((v1[..., s] - v1[..., t]) * (v1[..., s] - v1[..., t]) + (v2[..., s] - v2[..., t]) * (v2[..., s] - v2[..., t])
                 + (v3[..., s] - v3[..., t]) * (v3[..., s] - v3[..., t]))
            Pr[..., s] = Pr[..., s] + ns[..., s] * ms[s] / (gam[s] - 1) * d * fact
    sf = _EL / _KB * (gam[LSP - 1] - 1)
    Te = Ts[..., LSP - 1]
    nu = sf * 6.9e-14 * nn[..., 2] * 1e-6 / _V["sqrt"](Te)
    pT, lT = nu * Tn, nu
    nu = sf * 2.9e-14 * nn[..., 1] * 1e-6 / _V["sqrt"](Te)
    pT, lT = pT + nu * Tn, lT + nu
    f = 1.06e4 + 7.51e3 * _V["tanh"](1.10e-3 * (Te - 1800))
    gg = 3300 + 1.233 * (Te - 1000) - 2.056e-4 * (Te - 1000) * (Te - 4000)
    fact = (sf * 2.99e-12 * nn[..., 1] * 1e-6 * _V["exp"](f * (Te - 2000) / Te / 2000)
            * (_V["exp"](-gg * (Te - Tn) / Te / Tn) - 1))
    pT = pT - np.maximum(fact, 0.0)
    f = 3300 - 839 * _V["sin"](1.91e-4 * (Te - 2700))
    fact = (sf * 5.196e-13 * nn[..., 2] * 1e-6 * _V["exp"](f * (Te - 700) / Te / 700)
            * (_V["exp"](-2770 * (Te - Tn) / Te / Tn) - 1))
    pT = pT - np.maximum(fact, 0.0)
    Pr[..., LSP - 1] = Pr[..., LSP - 1] + pT * ns[..., LSP - 1] * _KB / (gam[LSP - 1] - 1)
    Lo[..., LSP - 1] = Lo[..., LSP - 1] + lT
    return Pr, Lo


def test_srcs_energy_matches_numpy_statement():
    g = G.dipole_grid(10, 4, 3)
    st = S.init_state(g, seed=12, perturb=0.3)
    rng = np.random.default_rng(12)
    fv = st.fluidvars
    I = (slice(2, g.lx1 + 2), slice(2, g.lx2 + 2), slice(2, g.lx3 + 2))
    for k in (1, 2, 3):  # velocities of every species, some pairs far apart (Phi branch)
        fv[I + (slice(k * LSP, (k + 1) * LSP),)] = rng.uniform(-3000, 3000, fv[I + (slice(0, LSP),)].shape)
    nn, vn, Tn = _neutrals(g, 12)
    Pr, Lo = O.srcs_energy(g, st, nn, *vn, Tn)
    Pw, Lw = _np_srcs_energy(g, st, nn, *vn, Tn)
    assert np.array_equal(Lo, Lw)
    assert np.array_equal(Pr, Pw)
    # finite everywhere; Lo is not sign-definite: the electron-N2 and electron-H collision
    # fits (1 - 1.21e-4 Te, 1 - 1.35e-4 Te) turn negative above ~8300 K and ~7400 K
    assert np.isfinite(Lo).all() and np.isfinite(Pr).all()


def test_srcs_energy_electron_rotational_cooling_alone():
    """With only O2 as neutral and no ions in motion, the electrons' loss rate holds the O2
    rotational term and the ion-neutral / Coulomb terms."""
    g = G.cartesian_grid(8, 3, 3)
    st = S.init_state(g, seed=3, perturb=0.1)
    nn, vn, Tn = _neutrals(g, 3)
    nn[..., [0, 1, 3]] = 0.0
    Pr, Lo = O.srcs_energy(g, st, nn, *vn, Tn)
    Pw, Lw = _np_srcs_energy(g, st, nn, *vn, Tn)
    assert np.array_equal(Lo, Lw) and np.array_equal(Pr, Pw)
    assert (Lo[..., LSP - 1] > 0).all()


# ---- srcsMomentum_curv (single rank): numpy statement and a plasma at rest -----------------

def _np_grad1(f, h1, dx1):
    """grad3D1_curv_23 along axis 0 (the first point divides by dx1[0], as the reference)."""
    out = np.empty_like(f)
    out[0] = (f[1] - f[0]) / dx1[0] / h1[0]
    out[1:-1] = (f[2:] - f[:-2]) / (dx1[2:] + dx1[1:-1])[:, None, None] / h1[1:-1]
    out[-1] = (f[-1] - f[-2]) / dx1[-1] / h1[-1]
    return out


def _np_srcs_momentum(g, st, nn, vn1, Tn, E1, Q, g1):
    ms, qs, _, _ = O.constants()
    n1 = g.lx1
    I = (slice(2, n1 + 2), slice(2, g.lx2 + 2), slice(2, g.lx3 + 2))
    J = (slice(1, n1 + 3), slice(2, g.lx2 + 2), slice(2, g.lx3 + 2))  # x1 indices 0..lx1+1
    fv = st.fluidvars
    ns, v1, v2, v3, Ts = (fv[I + (slice(k * LSP, (k + 1) * LSP),)] for k in range(5))
    h1, h2, h3 = g.h1[I], g.h2[I], g.h3[I]
    dh2 = _np_grad1(g.h2[J], g.h1[J], g.dx1[0:n1 + 2])[1:-1]
    dh3 = _np_grad1(g.h3[J], g.h1[J], g.dx1[0:n1 + 2])[1:-1]
    dxi = g.dx1[1:n1 + 1]
    lg = np.vectorize(math.log)
    Te = Ts[..., LSP - 1]
    epol = _KB * Te / qs[LSP - 1] * _np_grad1(lg(ns[..., LSP - 1] * _KB * Te), h1, dxi)
    alt = g.alt[I]
    e1f = np.where(alt < 100e3, 0.0, E1[I])
    Pr = np.zeros(ns.shape)
    Lo = np.zeros(ns.shape)
    for s in range(LSP):
        for j in range(4):
            nu = _np_maxwell(s, j, nn[..., j], Tn, Ts[..., s])
            Lo[..., s] = Lo[..., s] + nu
            Pr[..., s] = Pr[..., s] + ns[..., s] * ms[s] * nu * vn1
        for t in range(LSP):
            nu, phi, _ = _np_coulomb(s, t, ms, ns[..., t], Ts[..., s], Ts[..., t], v1[..., s], v1[..., t])
            Lo[..., s] = Lo[..., s] + nu * phi
            Pr[..., s] = Pr[..., s] + ns[..., s] * ms[s] * nu * phi * v1[..., t]
        p = ns[..., s] * _KB * Ts[..., s]
        ionpress = p * _np_grad1(lg(p), h1, dxi)
        gq = _np_grad1(Q[..., s], h1, dxi)
        geom = (v2[..., s] * v2[..., s] * h3 * dh2 + v3[..., s] * v3[..., s] * h2 * dh3) * ns[..., s] * ms[s] / (h1 * h2 * h3)
        Pr[..., s] = Pr[..., s] + ns[..., s] * qs[s] * (e1f + epol) - ionpress - gq + geom + ns[..., s] * ms[s] * g1
    return Pr, Lo


def _momentum_inputs(g, seed):
    rng = np.random.default_rng(seed)
    shp = (g.lx1, g.lx2, g.lx3)
    nn, vn, Tn = _neutrals(g, seed)
    E1 = np.asfortranarray(rng.uniform(-1e-3, 1e-3, (g.lx1 + 4, g.lx2 + 4, g.lx3 + 4)))
    Q = np.asfortranarray(rng.uniform(0, 1e-12, shp + (LSP,)))
    g1 = np.asfortranarray(rng.uniform(-9.8, -8.0, shp))
    return nn, vn[0], Tn, E1, Q, g1


def test_srcs_momentum_matches_numpy_statement():
    g = G.dipole_grid(12, 4, 3)
    st = S.init_state(g, seed=21, perturb=0.3)
    rng = np.random.default_rng(21)
    fv = st.fluidvars
    I = (slice(2, g.lx1 + 2), slice(2, g.lx2 + 2), slice(2, g.lx3 + 2))
    for k in (1, 2, 3):
        fv[I + (slice(k * LSP, (k + 1) * LSP),)] = rng.uniform(-3000, 3000, fv[I + (slice(0, LSP),)].shape)
    args = _momentum_inputs(g, 21)
    Pr, Lo = O.srcs_momentum(g, st, *args)
    Pw, Lw = _np_srcs_momentum(g, st, *args)
    assert np.array_equal(Lo, Lw)
    assert np.array_equal(Pr, Pw)
    assert np.isfinite(Pr).all() and (g.alt[I] < 100e3).any() and (g.alt[I] >= 100e3).any()


def test_srcs_momentum_of_a_uniform_plasma_at_rest_is_zero():
    """No flow, no neutral wind, no field, no gravity, uniform density and temperature:
    every force term vanishes, while the collision loss rates do not."""
    g = G.cartesian_grid(10, 4, 3)
    st = S.init_state(g, seed=1, perturb=0.0)
    fv = st.fluidvars
    for s in range(LSP):
        fv[..., s] = 1e11 if s < LSP - 1 else 6e11
        fv[..., 4 * LSP + s] = 1500.0
    fv[..., LSP:4 * LSP] = 0.0
    nn, vn1, Tn, E1, Q, g1 = _momentum_inputs(g, 2)
    Pr, Lo = O.srcs_momentum(g, st, nn, np.zeros_like(vn1), Tn, np.zeros_like(E1), np.zeros_like(Q),
                             np.zeros_like(g1))
    assert (Pr == 0).all()
    assert (Lo > 0).all()


def test_srcs_energy_balances_at_thermal_equilibrium():
    """Every species at the neutral temperature and moving with the neutral wind: heat
    transfer, friction and the electrons' inelastic terms all vanish, so each species'
    production equals its loss times its energy density."""
    g = G.dipole_grid(12, 4, 3)
    st = S.init_state(g, seed=4, perturb=0.2)
    nn, vn, Tn = _neutrals(g, 4)
    fv = st.fluidvars
    I = (slice(2, g.lx1 + 2), slice(2, g.lx2 + 2), slice(2, g.lx3 + 2))
    for s in range(LSP):
        fv[I + (4 * LSP + s,)] = Tn
        for k in range(3):
            fv[I + ((1 + k) * LSP + s,)] = vn[k]
    O.T2rhoe(g, st)
    Pr, Lo = O.srcs_energy(g, st, nn, *vn, Tn)
    re = st.fluidauxvars[I + (slice(LSP, 2 * LSP),)]
    np.testing.assert_allclose(Pr, Lo * re, rtol=1e-12, atol=0)
    assert (Lo > 0).all()


def test_full_step_runs_and_stays_physical():
    """fluid_adv with compression and the source/loss sub-step (synthetic neutral state and
    ionization): finite, densities above the floor, temperatures at or above 100 K, and a
    different state from the step without sources."""
    g = G.dipole_grid(20, 5, 4)
    a = S.init_state(g, seed=6, perturb=0.2)
    b = a.copy()
    rng = np.random.default_rng(6)
    shp = (g.lx1, g.lx2, g.lx3)
    nn = np.asfortranarray(np.concatenate([a.nn, np.stack([10 ** rng.uniform(9, 12, shp) for _ in range(4)], -1)], -1))
    vn = [np.asfortranarray(rng.uniform(-50, 50, shp)) for _ in range(3)]
    g1 = np.asfortranarray(np.full(shp, -9.0))
    Pi = np.asfortranarray(rng.uniform(0, 1e8, shp + (LSP - 1,)))
    Qe = np.asfortranarray(rng.uniform(0, 1e-12, shp))
    dt = 0.05
    O.fluid_adv_full(g, a, dt, nn, *vn, g1, Pi, Qe)
    O.fluid_adv_compression(g, b, dt)
    fv = a.fluidvars
    assert np.isfinite(fv).all() and np.isfinite(a.fluidauxvars[..., :2 * LSP]).all()
    I = (slice(2, g.lx1 + 2), slice(2, g.lx2 + 2), slice(2, g.lx3 + 2))
    assert (fv[I + (slice(0, LSP),)] > 0).all()
    assert (fv[I + (slice(4 * LSP, 5 * LSP),)] >= 100.0).all()
    assert not np.array_equal(fv, b.fluidvars)
