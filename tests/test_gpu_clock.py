"""Device-resident time stepping through the C ABI: gem_dt_select_dev against the oracle's
dt_select (libgemini_mpi.f90:450-483) bit for bit over its clip, floor and throttle cases,
and a loop of steps with dt and the clock kept on the device against the same loop driven
from the host with the oracle."""
import ctypes

import numpy as np
import pytest

import oracle as O
from gemini_b200 import _lib
from gemini_b200 import fluid as F
from gemini_b200 import grid as G
from gemini_b200 import state as S

from test_clock_host import select_cases

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _exact_dependencies():
    O.set_device_semantics(True)
    yield
    O.set_device_semantics(False)


def _clock(t, tout, tglowout, it):
    """a gem_clock in device memory: four doubles and the iteration counter"""
    import torch
    c = torch.tensor([t, tout, tglowout, 0.0, 0.0], dtype=torch.float64)
    c.view(torch.int64)[4] = it
    return c.cuda()


def _select(cfg, ds, clock, dt):
    c = cfg.c()
    _lib.check(_lib.lib().gem_dt_select_dev(ctypes.byref(c), ds.g, F._ptr(ds.fluidvars), ds.work, F._ptr(clock),
                                            F._ptr(dt), None))


def test_dt_select_exact():
    import torch
    g = G.dipole_grid(16, 5, 4)
    st = S.init_state(g, seed=2, perturb=0.2)
    ds = F.DeviceState.from_host(F.DeviceGrid(g), st.copy())
    try:
        dtcfl = O.dt_calc(g, st)[0]
        for t, tout, tglow, flag, it, prev in select_cases(dtcfl):
            cfg = F.FluidCfg(st.Teinf)
            cfg.flagglow = flag
            clock = _clock(t, tout, tglow, it)
            dt = torch.tensor([prev], dtype=torch.float64, device="cuda")
            _select(cfg, ds, clock, dt)
            want = O.dt_select(g, st, t=t, tout=tout, it=it, dtprev=prev, tglowout=tglow, flagglow=flag)
            assert dt.item() == want, (t, tout, tglow, flag, it, prev)
            assert clock[3].item() == dtcfl
    finally:
        ds.close()


def test_step_loop_keeps_dt_on_the_device():
    import torch
    g = G.cartesian_grid(20, 10, 8)
    st = S.init_state(g, seed=1)
    ds = F.DeviceState.from_host(F.DeviceGrid(g), st.copy())
    try:
        cfg = F.FluidCfg(st.Teinf)
        ref = st.copy()
        t, tout, dtprev = 0.0, 1e12, 1.0
        dts = []
        for it in range(1, 5):
            dtr = O.dt_select(g, ref, t=t, tout=tout, it=it, dtprev=dtprev)
            O.fluid_adv(g, ref, dtr)
            t, dtprev = t + dtr, dtr
            dts.append(dtr)
        clock = _clock(0.0, tout, float("inf"), 1)
        dt = torch.tensor([1.0], dtype=torch.float64, device="cuda")
        got = []
        for _ in range(4):
            _select(cfg, ds, clock, dt)
            F.fluid_adv(cfg, ds, dt)
            _lib.check(_lib.lib().gem_clock_advance_dev(F._ptr(clock), F._ptr(dt), None))
            got.append(dt.item())
        np.testing.assert_allclose(got, dts, rtol=1e-11)
        assert got[0] == dts[0]
        assert clock.view(torch.int64)[4].item() == 5
        assert abs(clock[0].item() - t) <= 1e-11 * t
    finally:
        ds.close()
