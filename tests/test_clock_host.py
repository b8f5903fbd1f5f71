"""The device dt_select body (gem_clock.cuh: the output clips, the 1e-6 floor and the growth
throttle after the CFL step), compiled for the host, against the oracle's dt_select
(libgemini_mpi.f90:450-483 with temporal_mpi.f90:27-84) bit for bit over clip, floor and
throttle cases."""
import ctypes
import itertools
import os
import shutil
import subprocess

import pytest

import oracle as O
from gemini_b200 import grid as G
from gemini_b200 import state as S

from helpers import harness_flags

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    cxx = shutil.which("g++")
    if not cxx:
        pytest.skip("no g++")
    out = str(tmp_path_factory.mktemp("clock") / "libclock.so")
    subprocess.check_call([cxx, "-O2", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", *harness_flags(), "-o", out,
                           os.path.join(HERE, "clock_harness.cpp")])
    L = ctypes.CDLL(out)
    d = ctypes.c_double
    L.hc_dt_select.argtypes = [d, d, d, d, ctypes.c_int, ctypes.c_longlong, d]
    L.hc_dt_select.restype = d
    return L


def select_cases(dt):
    """(t, tout, tglowout, flagglow, it, dtprev) around every branch of the selection."""
    ts = (0.0, 100.0, 3.3e5)
    outs = (lambda t: 1e12, lambda t: t + dt / 3, lambda t: t + 1e-9, lambda t: t + dt)
    glows = (lambda t: float("inf"), lambda t: t + dt / 7, lambda t: t)
    for t, fo, fg, flag, it, prev in itertools.product(ts, outs, glows, (0, 1), (1, 2, 50),
                                                       (dt / 4, dt / 2, dt, 10 * dt, 1e-7)):
        yield t, fo(t), fg(t), flag, it, prev


def test_dt_select_body_equals_the_oracle(harness):
    g = G.dipole_grid(16, 5, 4)
    st = S.init_state(g, seed=2, perturb=0.2)
    dtcfl = O.dt_calc(g, st)[0]
    n = 0
    for t, tout, tglow, flag, it, prev in select_cases(dtcfl):
        want = O.dt_select(g, st, t=t, tout=tout, it=it, dtprev=prev, tglowout=tglow, flagglow=flag)
        got = harness.hc_dt_select(dtcfl, t, tout, tglow, flag, it, prev)
        assert got == want or (got != got and want != want), (t, tout, tglow, flag, it, prev, got, want)
        n += 1
    assert n == 3 * 4 * 3 * 2 * 3 * 5
