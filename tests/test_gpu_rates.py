"""GPU parity of the production/loss rates (sources.f90 srcsContinuity, srcsEnergy,
srcsMomentum_curv with collisions.f90) through the device C ABI against the oracle.

The device evaluates every expression in the reference's order with the same IEEE
operations; only pow, exp, log, log10, erf, tanh and sin are the device's own (a few ulp
from the C library's), and x**0.5, x**1.5 are sqrt(x), x*sqrt(x) there (within 1.5 ulp).  Tolerance, written here, for Pr and Lo alike:
  |gpu - oracle| <= 1e-12 (|oracle| + max over the species' cells of |oracle|),
i.e. relative where a rate is a sum of like-signed terms and norm-wise per species where
terms of both signs cancel: the Coulomb Phi near W = 0.1 (two terms of ~150 cancel to ~1,
so a 2-ulp erf moves it by ~1e-13 relative), the electron-N2 and electron-H collision fits
(negative above ~8300 K and ~7400 K, so the electrons' Lo is a signed sum), the momentum
sources (drag, fields and gradients of both signs).  Checked against the host bodies with
every device math function moved by 2 ulp (passes) and by 1e5 ulp (fails).
The same bodies compiled for the host reproduce the oracle bit for bit
(test_rates_host.py), so any larger difference here is the device's, not the formula's."""
import numpy as np
import pytest

import oracle as O
from gemini_b200 import fluid as F
from gemini_b200 import grid as G

from helpers import LSP, rate_inputs

pytestmark = pytest.mark.gpu

GRIDS = [
    ("cart", lambda: G.cartesian_grid(20, 10, 8)),
    ("cart_2d", lambda: G.cartesian_grid(24, 9, 1)),
    ("cart_periodic", lambda: G.cartesian_grid(16, 5, 7, flagper=1)),
    ("dipole", lambda: G.dipole_grid(40, 8, 6)),
    ("dipole_nulls", lambda: G.dipole_grid(40, 8, 5, q_extent=0.5)),
]
RTOL = 1e-12


def _dev(a):
    import torch
    return torch.from_numpy(np.asfortranarray(a, dtype=np.float64).ravel(order="F").copy()).cuda()


def _cmp(what, got, want):
    Pa, La = want
    P, L = (t.cpu().numpy().reshape(Pa.shape, order="F") for t in got)
    assert np.isfinite(P).all() and np.isfinite(L).all(), what
    for nm, got_, want_ in (("Lo", L, La), ("Pr", P, Pa)):
        scale = np.abs(want_).reshape(-1, LSP, order="F").max(axis=0)
        err = np.abs(got_ - want_)
        ok = err <= RTOL * (np.abs(want_) + scale)
        assert ok.all(), f"{what} {nm}: {np.count_nonzero(~ok)} cells beyond tolerance, worst {err[~ok].max()!r}"


@pytest.mark.parametrize("name,mk", GRIDS, ids=[c[0] for c in GRIDS])
def test_rates(name, mk):
    g = mk()
    st, nn, vn, Tn, E1, Q, g1, alt = rate_inputs(g, 41)
    st.electrovars[..., 0] = E1
    ds = F.DeviceState.from_host(F.DeviceGrid(g), st.copy())
    try:
        d = [_dev(a) for a in (nn, vn[0], vn[1], vn[2], Tn)]
        _cmp("continuity", F.srcs_continuity(ds, *d), O.srcs_continuity(g, st, nn, *vn, Tn))
        _cmp("energy", F.srcs_energy(ds, *d), O.srcs_energy(g, st, nn, *vn, Tn))
        _cmp("momentum", F.srcs_momentum(ds, d[0], d[1], d[4], _dev(Q), _dev(alt), _dev(g1)),
             O.srcs_momentum(g, st, nn, vn[0], Tn, E1, Q, g1))
    finally:
        ds.close()
