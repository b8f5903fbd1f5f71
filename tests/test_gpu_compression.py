"""GPU parity of the compression sub-step (app/main.f90:320-338): VNRicht_artvisc, the
zero-order-hold velocity ghosts of RK2_global_boundary and the compression update of rhoes,
each through the device C ABI against the oracle, bit for bit (the device restates the
reference's operation order with IEEE divisions and no FMA contraction)."""
import numpy as np
import pytest

import oracle as O
from gemini_b200 import fluid as F
from gemini_b200 import state as S

from helpers import LSP, assert_identical, cases

pytestmark = pytest.mark.gpu

CASES = cases()
IDS = [c[0] for c in CASES]
DT = 0.07


def _state(case):
    name, g, kw = case
    st = S.init_state(g, **kw)
    rng = np.random.default_rng(kw.get("seed", 0) + 100)
    fv = st.fluidvars
    fv[..., LSP:4 * LSP] = rng.uniform(-800, 800, fv[..., LSP:4 * LSP].shape)  # ghosts too
    O.T2rhoe(g, st)
    return g, st


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_compression_substep_exact(case):
    g, st = _state(case)
    a = st.copy()
    Qa = O.vnricht_artvisc(g, a)
    O.halo_fluidvars(g, a)
    O.rk2_global_boundary(g, a)
    O.compression(g, a, DT, Qa)

    dg = F.DeviceGrid(g)
    ds = F.DeviceState.from_host(dg, st.copy())
    try:
        Q = F.vnricht_artvisc(ds)
        assert np.array_equal(Q.cpu().numpy(), Qa.ravel(order="F")), "artvisc"
        F.halo_fluidvars(ds)
        F.rk2_global_boundary_allspec(ds)
        b = ds.to_host(st)
        assert np.array_equal(b.fluidvars, a.fluidvars), "rk2_global_boundary"
        F.compression(ds, Q, DT)
        b = ds.to_host(st)
        assert_identical(b, a, "compression")
        assert not np.array_equal(b.fluidauxvars[..., LSP:2 * LSP], st.fluidauxvars[..., LSP:2 * LSP])
    finally:
        ds.close()


def test_compression_dt_from_device_slot():
    """dt is read on the device: a step with the slot holding 2*dt equals the oracle's."""
    name, g, kw = CASES[0]
    g, st = _state(CASES[0])
    a = st.copy()
    Qa = O.vnricht_artvisc(g, a)
    O.compression(g, a, 2 * DT, Qa)
    ds = F.DeviceState.from_host(F.DeviceGrid(g), st.copy())
    try:
        Q = F.vnricht_artvisc(ds)
        ds.dt.fill_(2 * DT)
        F.compression(ds, Q, ds.dt)
        assert np.array_equal(ds.to_host(st).fluidauxvars, a.fluidauxvars)
    finally:
        ds.close()
