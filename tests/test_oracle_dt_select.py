"""The oracle's dt_select (libgemini_mpi.f90:449-482 with temporal_mpi.f90:26-66, single
rank): the CFL step, the GLOW-output and output clips, the 1e-6 floor and the growth
throttle (dtscale = 2), each case checked against the CFL step alone."""
import oracle as O
from gemini_b200 import grid as G
from gemini_b200 import state as S


def _case():
    g = G.dipole_grid(16, 5, 4)
    st = S.init_state(g, seed=2, perturb=0.2)
    return g, st, O.dt_calc(g, st)[0]


def test_no_clip_first_iteration_is_the_cfl_step():
    g, st, dt = _case()
    assert O.dt_select(g, st, t=0.0, tout=1e9, it=1, dtprev=1e-12) == dt  # no throttle on iteration 1


def test_growth_throttled_to_twice_the_previous_step():
    g, st, dt = _case()
    assert O.dt_select(g, st, t=0.0, tout=1e9, it=2, dtprev=dt / 4) == 2 * (dt / 4)
    assert O.dt_select(g, st, t=0.0, tout=1e9, it=2, dtprev=dt / 2) == dt      # exactly 2x: kept
    assert O.dt_select(g, st, t=0.0, tout=1e9, it=2, dtprev=dt * 10) == dt     # shrinking is free


def test_output_clip_and_floor():
    g, st, dt = _case()
    t = 100.0
    assert O.dt_select(g, st, t=t, tout=t + dt / 3, it=1, dtprev=dt) == (t + dt / 3) - t
    assert O.dt_select(g, st, t=t, tout=t + 1e-9, it=1, dtprev=dt) == 1e-6   # never below 1e-6
    assert O.dt_select(g, st, t=t, tout=t + 5 * dt, it=1, dtprev=dt) == dt


def test_glow_output_clips_first_when_enabled():
    g, st, dt = _case()
    t = 10.0
    tg, to = t + dt / 5, t + dt / 2
    assert O.dt_select(g, st, t=t, tout=to, it=1, dtprev=dt, tglowout=tg, flagglow=1) == tg - t
    assert O.dt_select(g, st, t=t, tout=to, it=1, dtprev=dt, tglowout=tg, flagglow=0) == to - t
