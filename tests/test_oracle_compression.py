"""The oracle's compression sub-step (app/main.f90:320-338): VNRicht_artvisc, the RK2
zero-order-hold ghosts, div3D_curv_23 and the two-stage energy update, checked on the CPU
against exact cases (the divergence of linear fields, a flow at rest) and against a second,
numpy statement of the same formulas.  The reference ships no test of this sub-step, so
these restate rather than pin it."""
import numpy as np
import pytest

import oracle as O
from gemini_b200 import grid as G
from gemini_b200 import state as S

LSP = 7


def _np_div3D(g, f1, f2, f3):
    """div3D_curv_23 on the slab 0..lx+1, vectorised (calculus/div.f90:110-200)."""
    # ghosted arrays start at grid index -1; slab index j <-> grid index j-1
    L1, L2, L3 = g.lx1 + 2, g.lx2 + 2, g.lx3 + 2
    h1 = g.h1[1:1 + L1, 1:1 + L2, 1:1 + L3]
    h2 = g.h2[1:1 + L1, 1:1 + L2, 1:1 + L3]
    h3 = g.h3[1:1 + L1, 1:1 + L2, 1:1 + L3]
    a1, a2, a3 = (f[1:1 + L1, 1:1 + L2, 1:1 + L3] for f in (f1, f2, f3))
    dx1, dx2, dx3 = g.dx1[0:L1], g.dx2[0:L2], g.dx3[0:L3]
    d = np.empty((L1, L2, L3))
    t = h2 * h3 * a1
    d[0] = (t[1] - t[0]) / dx1[1]
    d[1:-1] = (t[2:] - t[:-2]) / (dx1[2:] + dx1[1:-1])[:, None, None]
    d[-1] = (t[-1] - t[-2]) / dx1[-1]
    if g.lx2 > 1:
        t = h1 * h3 * a2
        d[:, 0] = d[:, 0] + (t[:, 1] - t[:, 0]) / dx2[1]
        d[:, 1:-1] = d[:, 1:-1] + (t[:, 2:] - t[:, :-2]) / (dx2[2:] + dx2[1:-1])[None, :, None]
        d[:, -1] = d[:, -1] + (t[:, -1] - t[:, -2]) / dx2[-1]
    if g.lx3 > 1:
        t = h1 * h2 * a3
        d[:, :, 0] = d[:, :, 0] + (t[:, :, 1] - t[:, :, 0]) / dx3[1]
        d[:, :, 1:-1] = d[:, :, 1:-1] + (t[:, :, 2:] - t[:, :, :-2]) / (dx3[2:] + dx3[1:-1])[None, None, :]
        d[:, :, -1] = d[:, :, -1] + (t[:, :, -1] - t[:, :, -2]) / dx3[-1]
    return d / (h1 * h2 * h3)


def test_div3D_exact_for_linear_fields():
    """Centred and one-sided differences are exact for linear fields: on a Cartesian grid
    div(a x1, b x2, c x3) = a + b + c at every slab point."""
    g = G.cartesian_grid(12, 7, 5)
    x1, x2, x3 = np.meshgrid(g.x1, g.x2, g.x3, indexing="ij")
    a, b, c = 2.5e-3, -1.25e-3, 0.5e-3
    d = O.div3D(g, a * x1, b * x2, c * x3)
    np.testing.assert_allclose(d, a + b + c, rtol=1e-9, atol=1e-15)


@pytest.mark.parametrize("mk", [lambda: G.dipole_grid(20, 6, 5), lambda: G.cartesian_grid(14, 5, 6, flagper=1),
                                lambda: G.cartesian_grid(10, 1, 6)], ids=["dipole", "cart_periodic", "cart_2d"])
def test_div3D_matches_numpy_statement(mk):
    g = mk()
    rng = np.random.default_rng(3)
    shp = (g.lx1 + 4, g.lx2 + 4, g.lx3 + 4)
    f1, f2, f3 = (np.asfortranarray(rng.standard_normal(shp)) for _ in range(3))
    d = O.div3D(g, f1, f2, f3)
    assert np.array_equal(d, _np_div3D(g, f1, f2, f3))


def test_artvisc_matches_numpy_statement():
    g = G.dipole_grid(18, 5, 4)
    st = S.init_state(g, seed=5, perturb=0.2)
    rng = np.random.default_rng(8)
    st.fluidvars[..., LSP:2 * LSP] = rng.uniform(-300, 300, st.fluidvars[..., LSP:2 * LSP].shape)
    Q = O.vnricht_artvisc(g, st)
    ms = O.constants()[0]
    ns = st.fluidvars[..., 0:LSP]
    vs1 = st.fluidvars[..., LSP:2 * LSP]
    I2, I3 = slice(2, g.lx2 + 2), slice(2, g.lx3 + 2)
    for s in range(LSP - 1):
        v1i = 0.5 * (vs1[1:g.lx1 + 2, I2, I3, s] + vs1[2:g.lx1 + 3, I2, I3, s])  # faces 1..lx1+1
        dv = v1i[1:] - v1i[:-1]
        m = np.minimum(dv, 0.0)
        want = ns[2:g.lx1 + 2, I2, I3, s] * ms[s] * 0.25 * 9.0 * (m * m)
        assert np.array_equal(Q[..., s], want)
    assert not Q[..., LSP - 1].any()
    assert (Q >= 0).all() and Q[..., :LSP - 1].any()


@pytest.mark.parametrize("flagper", [0, 1])
def test_rk2_global_boundary_zero_order_hold(flagper):
    g = G.cartesian_grid(9, 5, 6, flagper=flagper)
    st = S.init_state(g, seed=2, perturb=0.1)
    rng = np.random.default_rng(1)
    fv = st.fluidvars
    fv[..., LSP:4 * LSP] = rng.standard_normal(fv[..., LSP:4 * LSP].shape)
    before = fv.copy()
    O.rk2_global_boundary(g, st)
    vs1, vs2, vs3 = (fv[..., k * LSP:(k + 1) * LSP] for k in (1, 2, 3))
    n1, n2, n3 = g.lx1, g.lx2, g.lx3
    # x1 (vs1), then x2 (all three), then x3 unless periodic: ghost 0 and lx+1 copy the edge
    for v in (vs1, vs2, vs3):
        assert np.array_equal(v[:, 1], v[:, 2]) and np.array_equal(v[:, n2 + 2], v[:, n2 + 1])
        if not flagper:
            assert np.array_equal(v[:, :, 1], v[:, :, 2]) and np.array_equal(v[:, :, n3 + 2], v[:, :, n3 + 1])
    assert np.array_equal(vs1[1, 3:n2 + 1, 3:n3 + 1], vs1[2, 3:n2 + 1, 3:n3 + 1])
    assert np.array_equal(vs1[n1 + 2, 3:n2 + 1, 3:n3 + 1], vs1[n1 + 1, 3:n2 + 1, 3:n3 + 1])
    if flagper:  # periodic x3 ghosts are left to the halo
        for k in (2, 3):
            v0 = before[..., k * LSP:(k + 1) * LSP]
            v = fv[..., k * LSP:(k + 1) * LSP]
            assert np.array_equal(v[2:n1 + 2, 2:n2 + 2, 1], v0[2:n1 + 2, 2:n2 + 2, 1])
    # interiors untouched
    assert np.array_equal(fv[2:n1 + 2, 2:n2 + 2, 2:n3 + 2], before[2:n1 + 2, 2:n2 + 2, 2:n3 + 2])


def test_compression_update_matches_numpy_statement():
    g = G.dipole_grid(16, 5, 4)
    st = S.init_state(g, seed=6, perturb=0.2)
    rng = np.random.default_rng(4)
    fv = st.fluidvars
    fv[..., LSP:4 * LSP] = rng.uniform(-200, 200, fv[..., LSP:4 * LSP].shape)
    Q = np.asfortranarray(rng.uniform(0, 1e-12, (g.lx1, g.lx2, g.lx3, LSP)))
    dt = 0.05
    O.T2rhoe(g, st)
    re0 = st.fluidauxvars[..., LSP:2 * LSP].copy()
    O.compression(g, st, dt, Q)
    gam = O.constants()[2]
    I = (slice(2, g.lx1 + 2), slice(2, g.lx2 + 2), slice(2, g.lx3 + 2))
    for s in range(LSP):
        d = _np_div3D(g, fv[..., LSP + s], fv[..., 2 * LSP + s], fv[..., 3 * LSP + s])[1:-1, 1:-1, 1:-1]
        p = re0[I + (s,)]
        half = p - dt / 2 * (p * (gam[s] - 1) + Q[..., s]) * d
        want = p - dt * (half * (gam[s] - 1) + Q[..., s]) * d
        assert np.array_equal(st.fluidauxvars[I + (LSP + s,)], want)
    # ghosts untouched
    ghost = np.ones(fv.shape[:3], bool)
    ghost[I] = False
    assert np.array_equal(st.fluidauxvars[ghost][:, LSP:2 * LSP], re0[ghost])


def test_step_with_compression_equals_step_without_at_rest():
    """With every velocity zero the divergence and the viscosity vanish, so the step with
    the compression sub-step gives the bits of the step without it."""
    g = G.dipole_grid(20, 5, 4)
    a = S.init_state(g, seed=7, perturb=0.2)
    a.fluidvars[..., LSP:4 * LSP] = 0.0
    b = a.copy()
    O.fluid_adv(g, a, 0.05)
    O.fluid_adv_compression(g, b, 0.05)
    assert np.array_equal(a.fluidvars, b.fluidvars)


def test_compression_heats_a_converging_flow():
    """A uniform converging flow along x1 (negative divergence) raises the energy density of
    every species; an expanding one lowers it."""
    g = G.cartesian_grid(16, 4, 4)
    for sign in (-1.0, 1.0):
        st = S.init_state(g, seed=1, perturb=0.0)
        fv = st.fluidvars
        x1 = g.x1[:, None, None]
        fv[..., LSP:2 * LSP] = (sign * 1e-3 * x1)[..., None]
        fv[..., 2 * LSP:4 * LSP] = 0.0
        O.T2rhoe(g, st)  # the energy densities the step carries into compression
        re0 = st.fluidauxvars[..., LSP:2 * LSP].copy()
        assert (re0[2:-2, 2:-2, 2:-2] > 0).all()
        Q = O.vnricht_artvisc(g, st)
        O.compression(g, st, 0.1, Q)
        I = (slice(2, g.lx1 + 2), slice(2, g.lx2 + 2), slice(2, g.lx3 + 2))
        d = st.fluidauxvars[I + (slice(LSP, 2 * LSP),)] - re0[I]
        assert (d > 0).all() if sign < 0 else (d < 0).all()
