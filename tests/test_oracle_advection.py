"""Properties of the oracle's MC-limited advection (advec.f90:384-435) that the scheme
implies: at CFL 1 with uniform velocity the flux-form update is an exact one-cell shift,
and a smooth profile converges at about second order.  The reference ships no advection
test; these check the restatement against the mathematics of the scheme."""
import numpy as np

import oracle as O


def _uniform_line(lx, dxv=1.0):
    return dict(dx=np.full(lx + 3, dxv), dxi=np.full(lx, dxv), ha1=np.ones(lx + 4), ha2i=np.ones(lx + 1),
                h1i=np.ones(lx + 1))


def test_cfl_one_is_an_exact_shift():
    """v dt / dx = 1: phi(i) is the upwind cell's value, so each cell takes its upwind
    neighbour's value exactly (integers keep every subtraction exact)."""
    rng = np.random.default_rng(0)
    lx = 40
    f = rng.integers(0, 1000, lx + 4).astype(np.float64)
    g = _uniform_line(lx)
    out = O.advec1D_MC_curv(f, np.ones(lx + 1), 1.0, **g)
    assert np.array_equal(out[2:lx + 2], f[1:lx + 1])       # shift right by one cell
    out = O.advec1D_MC_curv(f, -np.ones(lx + 1), 1.0, **g)
    assert np.array_equal(out[2:lx + 2], f[3:lx + 3])       # shift left by one cell
    assert np.array_equal(out[[0, 1, lx + 2, lx + 3]], f[[0, 1, lx + 2, lx + 3]])  # ghosts pass through


def _advect_bump(lx, cfl=0.5, T=0.25):
    L = 1.0
    dx = L / lx
    x = (np.arange(-1, lx + 3) - 0.5) * dx  # cell centres of indices -1..lx+2
    f = np.exp(-((x - 0.3) / 0.05) ** 2)
    v = 1.0
    dt = cfl * dx / v
    nsteps = int(round(T / dt))
    g = _uniform_line(lx, dx)
    for _ in range(nsteps):
        f = O.advec1D_MC_curv(f, np.full(lx + 1, v), dt, **g)
    exact = np.exp(-((x - 0.3 - v * nsteps * dt) / 0.05) ** 2)
    return np.abs(f[2:lx + 2] - exact[2:lx + 2]).sum() * dx


def test_smooth_bump_converges_at_about_second_order():
    e = [_advect_bump(n) for n in (100, 200, 400)]
    assert e[0] > e[1] > e[2]
    assert e[0] / e[1] > 3.0 and e[1] / e[2] > 3.0   # order > 1.58 in L1 (the limiter clips the peak)


def test_constant_field_stays_constant_on_a_curvilinear_line():
    """A constant field with a face flux that is constant once the metric is included
    (ha2i v = const) and cell volumes ha1 dxi matching the face spacing stays constant."""
    rng = np.random.default_rng(3)
    lx = 30
    dx = rng.uniform(0.5, 1.5, lx + 3)
    dxi = rng.uniform(0.5, 1.5, lx)
    ha1 = rng.uniform(1.0, 2.0, lx + 4)
    ha2i = rng.uniform(1.0, 2.0, lx + 1)
    h1i = rng.uniform(1.0, 2.0, lx + 1)
    v = 0.3 / ha2i                      # ha2i * v uniform: no divergence of the flux
    f = np.full(lx + 4, 7.0)
    out = O.advec1D_MC_curv(f, v, 0.1, dx, dxi, ha1, ha2i, h1i)
    np.testing.assert_allclose(out, 7.0, rtol=1e-14)
