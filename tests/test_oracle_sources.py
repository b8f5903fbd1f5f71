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
