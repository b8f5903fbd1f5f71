"""The device production/loss rate kernels' bodies (gem_rates.cuh: srcsContinuity,
srcsEnergy, srcsMomentum_curv), compiled for the host with the C library's math functions
and run over every index of their ranges, against the oracle's restatement bit for bit.  The
metric tables are laid out as the device holds them (none on unit-metric grids, one x3 slice
with stride 0 when they do not vary along x3)."""
import ctypes
import math
import os
import shutil
import subprocess

import numpy as np
import pytest

import oracle as O
from gemini_b200 import grid as G
from gemini_b200 import state as S

from helpers import rate_inputs, harness_flags

LSP = 7
HERE = os.path.dirname(os.path.abspath(__file__))
_D = ctypes.POINTER(ctypes.c_double)


class HRView(ctypes.Structure):
    _fields_ = [("lx1", ctypes.c_int), ("lx2", ctypes.c_int), ("lx3", ctypes.c_int), ("c3", ctypes.c_longlong)] + \
               [(n, _D) for n in ("h1", "h2", "h3", "dx1", "ms", "qs", "gam")] + [("pi", ctypes.c_double)]


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    cxx = shutil.which("g++")
    if not cxx:
        pytest.skip("no g++")
    out = str(tmp_path_factory.mktemp("rates") / "librates.so")
    subprocess.check_call([cxx, "-O2", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", *harness_flags(), "-o", out,
                           os.path.join(HERE, "rates_harness.cpp")])
    L = ctypes.CDLL(out)
    P = ctypes.POINTER(HRView)
    L.hr_continuity.argtypes = [P] + [_D] * 8
    L.hr_energy.argtypes = [P] + [_D] * 8
    L.hr_momentum.argtypes = [P] + [_D] * 10
    L.hr_coulomb_pair.argtypes = [P, ctypes.c_int, ctypes.c_int] + [ctypes.c_double] * 4 + [_D]
    return L


def _p(a):
    return a.ctypes.data_as(_D)


def _view(g, keep):
    """The metric layout the device uses (gem_grid_create)."""
    lx1, lx2, lx3 = g.lx1, g.lx2, g.lx3
    ms, qs, gam, _ = O.constants()
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (g.dx1, ms, qs, gam)]
    hs = [np.asfortranarray(getattr(g, n)) for n in ("h1", "h2", "h3")]
    c3 = (lx1 + 4) * (lx2 + 4)
    if g.unit_metrics:
        hs = [None, None, None]
    elif all(np.array_equal(h[:, :, k], h[:, :, 2]) for h in hs for k in range(2, lx3 + 2)):
        hs = [np.asfortranarray(h[:, :, 2]) for h in hs]
        c3 = 0
    keep.extend([h for h in hs if h is not None] + arrs)
    hp = [(_p(h) if h is not None else _D()) for h in hs]
    return HRView(lx1, lx2, lx3, c3, *hp, *[_p(a) for a in arrs], 4 * math.atan(1.0))


GRIDS = [
    ("cart", lambda: G.cartesian_grid(14, 6, 5)),
    ("cart_2d", lambda: G.cartesian_grid(12, 1, 6)),
    ("dipole", lambda: G.dipole_grid(18, 6, 5)),
    ("dipole_nulls", lambda: G.dipole_grid(16, 6, 4, q_extent=0.5)),
]


@pytest.mark.parametrize("name,mk", GRIDS, ids=[c[0] for c in GRIDS])
def test_rate_bodies_equal_the_oracle_on_the_host(harness, name, mk):
    g = mk()
    st, nn, vn, Tn, E1, Q, g1, alt = rate_inputs(g, 31)
    keep = []
    v = _view(g, keep)
    shp = (g.lx1, g.lx2, g.lx3, LSP)
    fv = np.asfortranarray(st.fluidvars)
    for which in ("continuity", "energy", "momentum"):
        Pr, Lo = np.full(shp, np.nan, order="F"), np.full(shp, np.nan, order="F")
        if which == "continuity":
            Pa, La = O.srcs_continuity(g, st, nn, *vn, Tn)
            harness.hr_continuity(ctypes.byref(v), _p(nn), *[_p(a) for a in vn], _p(Tn), _p(fv), _p(Pr), _p(Lo))
        elif which == "energy":
            Pa, La = O.srcs_energy(g, st, nn, *vn, Tn)
            harness.hr_energy(ctypes.byref(v), _p(nn), *[_p(a) for a in vn], _p(Tn), _p(fv), _p(Pr), _p(Lo))
        else:
            Pa, La = O.srcs_momentum(g, st, nn, vn[0], Tn, E1, Q, g1)
            harness.hr_momentum(ctypes.byref(v), _p(nn), _p(vn[0]), _p(Tn), _p(fv), _p(E1), _p(Q), _p(alt), _p(g1),
                                _p(Pr), _p(Lo))
        assert np.array_equal(Lo, La), which
        assert np.array_equal(Pr, Pa), which


def test_coulomb_pair_is_symmetric_to_the_bit(harness):
    """The device rate kernels evaluate each unordered charged pair's Teff**1.5, Phi and Psi
    once and hand both species the same bits; that is exact because, with no contraction,
    swapping the species (and their temperatures and drifts) gives the same bits.  Checked on
    every pair over temperatures of 100..40000 K and drifts of up to 3 km/s (both branches
    of Phi, W below and above 0.1)."""
    g = G.cartesian_grid(6, 2, 2)
    keep = []
    v = _view(g, keep)
    rng = np.random.default_rng(17)
    a, b = np.zeros(3), np.zeros(3)
    branches = set()
    for _ in range(400):
        i, j = (int(x) for x in rng.choice(LSP, 2, replace=False))
        t1, t2 = rng.uniform(100, 40000, 2)
        u1, u2 = rng.uniform(-3000, 3000, 2) * rng.choice([1e-3, 1.0])
        harness.hr_coulomb_pair(ctypes.byref(v), i, j, t1, t2, u1, u2, _p(a))
        harness.hr_coulomb_pair(ctypes.byref(v), j, i, t2, t1, u2, u1, _p(b))
        assert a.tobytes() == b.tobytes(), (i, j, t1, t2, u1, u2, a, b)
        branches.add(a[1] == 1.0)
    assert branches == {True, False}

