"""The CPU oracle pinned to the reference's own tests and to LAPACK, plus oracle-side
properties (no GPU needed)."""
import json
import os

import numpy as np
import pytest

import oracle as O
from gemini_b200 import grid as G
from gemini_b200 import state as S

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _diffusion1d(npts=256, nsteps=13):
    """test/diffusion/test_diffusion1D.f90:33-110 on the oracle's 1-D solvers."""
    ix = np.arange(-1, npts + 3)
    x1 = (ix - 1).astype(np.float64) / float(npts - 1)
    lx1 = npts
    dx1 = x1[1:] - x1[:-1]
    x1i = 0.5 * (x1[1:lx1 + 2] + x1[2:lx1 + 3])
    dx1i = x1i[1:] - x1i[:-1]
    T0 = np.sin(2 * np.pi * x1) + np.sin(8 * np.pi * x1)
    TE, TB = T0[2:lx1 + 2].copy(), T0[2:lx1 + 2].copy()
    # dt=0.05/8**2/pi**2/maxval(lambda): 0.05 and 8**2 are default REAL, so the first
    # quotient is single precision
    dt = float(np.float32(0.05) / np.float32(64)) / (np.pi * np.pi) / 1.0
    Z, ONE = np.zeros(lx1), np.ones(lx1)
    t = 0.0
    for _ in range(nsteps):
        TE = O.backeuler_1d(TE, Z, Z, ONE, ONE, Z, 0.0, 0.0, dt, dx1, dx1i)
        TB = O.trbdf2_1d(TB, Z, Z, ONE, ONE, Z, 0.0, 0.0, dt, dx1, dx1i)
        t = t + dt
    xi = x1[2:lx1 + 2]
    true = np.exp(-4 * np.pi ** 2 * t) * np.sin(2 * np.pi * xi) + np.exp(-64 * np.pi ** 2 * t) * np.sin(8 * np.pi * xi)
    return TE, TB, true


def test_diffusion1d_golden():
    g = json.load(open(os.path.join(GOLDEN, "diffusion1d.json")))
    TE, TB, true = _diffusion1d(g["npts"], g["step_0based"] + 1)
    k = g["index_interior_0based"]
    # backward Euler reproduces all 15 printed digits
    assert TE[k] == pytest.approx(g["TsEuler"], rel=1e-14)
    # TRBDF2: 7e-13 from the printed value; scipy's OpenBLAS dgbsv lands 8e-13 away -- the
    # pivoted band LU on this stiff system is only reproducible to ~1e-12 across BLAS builds
    assert TB[k] == pytest.approx(g["TsBDF2"], rel=2e-12)
    assert true[k] == pytest.approx(g["Tstrue"], rel=1e-14)


def test_diffusion1d_accuracy_bound():
    """test_diffusion1D.f90:102-109: |numerical - analytic| <= 0.05 at every step."""
    TE, TB, true = _diffusion1d(256, 100)
    assert np.max(np.abs(TE - true)) < 0.05
    assert np.max(np.abs(TB - true)) < 0.05


def test_dgbsv_restatement_vs_openblas():
    d = np.load(os.path.join(GOLDEN, "dgbsv_cases.npz"))
    for ab, b, x, piv, n in zip(d["ab"], d["b"], d["x"], d["piv"], d["n"]):
        n = int(n)
        lu, ipiv, xo, info = O.dgbsv(ab[:, :n], b[:n], 2, 2)
        assert info == 0
        assert np.array_equal(ipiv - 1, piv[:n]), "row interchanges must match LAPACK's"
        scale = np.max(np.abs(x[:n]))
        assert np.max(np.abs(xo - x[:n])) <= 1e-11 * scale


def test_oracle_step_runs_finite():
    g = G.cartesian_grid(24, 6, 5)
    st = S.init_state(g, seed=3)
    dts = O.run_steps(g, st, 3)
    assert all(dt > 0 for dt in dts)
    assert np.isfinite(st.fluidvars).all() and np.isfinite(st.fluidauxvars[..., :14]).all()
    assert (st.Ts >= 100).all() and (st.ns[2:-2, 2:-2, 2:-2] > 0).all()


@pytest.mark.parametrize("dim", [1, 2, 3])
def test_advection_conserves_with_closed_ends(dim):
    """Flux-difference form: with zero velocity on the two end faces of every line,
    sum(f * ha1 * dxi) along the line is conserved to round-off."""
    g = G.dipole_grid(20, 6, 5)
    st = S.init_state(g, seed=9, perturb=0.2)
    O.v12rhov1(g, st); O.T2rhoe(g, st)
    rng = np.random.default_rng(1)
    vsi = {1: st.vs1i, 2: st.vs2i, 3: st.vs3i}[dim]
    vsi[...] = rng.uniform(-200, 200, vsi.shape)
    sl = [slice(None)] * 4
    for end in (0, -1):
        sl[dim - 1] = end
        vsi[tuple(sl)] = 0.0
    lx1, lx2, lx3 = g.lx1, g.lx2, g.lx3
    inner = (slice(2, lx1 + 2), slice(2, lx2 + 2), slice(2, lx3 + 2))
    vol = (g.h1 * g.h2 * g.h3)[inner]
    dxi = {1: g.dx1i[:, None, None], 2: g.dx2i[None, :, None], 3: g.dx3i[None, None, :]}[dim]
    before = np.array([(st.ns[inner + (s,)] * vol * dxi).sum(axis=dim - 1) for s in range(6)])
    O.sweep(g, st, dim, "mass", 2.0)
    after = np.array([(st.ns[inner + (s,)] * vol * dxi).sum(axis=dim - 1) for s in range(6)])
    assert np.max(np.abs(after - before) / np.abs(before)) < 1e-13


def test_extended_solver_vs_lapack_spread():
    """The two oracle band solvers differ only by LAPACK's pivoting round-off."""
    g = G.dipole_grid(96, 4, 3)
    st = S.init_state(g, seed=4, perturb=0.2)
    a, b = st.copy(), st.copy()
    dt, _ = O.dt_calc(g, st, 0.5)
    try:
        O.set_diffusion_solver(0)
        O.energy_diffusion(g, a, dt)
        O.set_diffusion_solver(1)
        O.energy_diffusion(g, b, dt)
    finally:
        O.set_diffusion_solver(0)
    rel = np.max(np.abs(a.Ts - b.Ts) / b.Ts)
    assert rel < 1e-8


def test_markstein_division_is_ieee_division():
    """The device divides a/b as q0=a*y, r=fma(-q0,b,a), q=fma(r,y,q0) with y=RN(1/b) inside
    its exponent guards; that must be the IEEE quotient bit for bit (random operands and
    near-representable quotients, signed zeros)."""
    bad, checked = O.markstein_mismatches(3_000_000, seed=7)
    assert checked > 2_500_000
    assert bad == 0
