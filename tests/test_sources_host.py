"""The device source/loss solves' per-cell bodies (gem_sources.cuh), compiled for the host
and run over every cell of the ghosted block, against the oracle's mass, momentum and
energy source/loss solves (multifluid.f90:474-549) bit for bit: on the host both call the
C library's exp, so any difference is in the index arithmetic or the operation order."""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

import oracle as O
from gemini_b200 import grid as G
from gemini_b200 import state as S

from helpers import harness_flags

LSP = 7
HERE = os.path.dirname(os.path.abspath(__file__))
_D = ctypes.POINTER(ctypes.c_double)


class HSView(ctypes.Structure):
    _fields_ = [("lx1", ctypes.c_int), ("lx2", ctypes.c_int), ("lx3", ctypes.c_int),
                ("ms", _D), ("qs", _D), ("gam", _D)]


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    cxx = shutil.which("g++")
    if not cxx:
        pytest.skip("no g++")
    out = str(tmp_path_factory.mktemp("src") / "libsrc.so")
    subprocess.check_call([cxx, "-O2", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", *harness_flags(), "-o", out,
                           os.path.join(HERE, "sources_harness.cpp")])
    L = ctypes.CDLL(out)
    P = ctypes.POINTER(HSView)
    d = ctypes.c_double
    L.hs_mass.argtypes = [P, d, _D, _D, _D, _D]
    L.hs_momentum.argtypes = [P, d, _D, _D, _D, _D, _D]
    L.hs_energy.argtypes = [P, d, _D, _D, _D, _D, _D, _D]
    return L


def _p(a):
    return a.ctypes.data_as(_D)


def _view(g, keep):
    ms, qs, gam, _ = O.constants()
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (ms, qs, gam)]
    keep.extend(arrs)
    return HSView(g.lx1, g.lx2, g.lx3, *[_p(a) for a in arrs])


def _blk(a, k):
    """pointer to species block k of a ghosted Fortran-ordered state array"""
    ng = a.shape[0] * a.shape[1] * a.shape[2]
    return ctypes.cast(a.ctypes.data + 8 * k * LSP * ng, _D)


def _rates(g, seed, scale):
    """Production in [0, scale), loss rates over 1e-14..1 with a fifth of them zero, so that
    L dt falls on both sides of the 1e-10 cut."""
    rng = np.random.default_rng(seed)
    shp = (g.lx1, g.lx2, g.lx3, LSP)
    Pr = np.asfortranarray(rng.uniform(0, scale, shp))
    Lo = np.asfortranarray(np.where(rng.uniform(size=shp) < 0.2, 0.0, 10 ** rng.uniform(-14, 0, shp)))
    return Pr, Lo, rng


GRIDS = [
    ("cart", lambda: G.cartesian_grid(14, 6, 5)),
    ("cart_2d", lambda: G.cartesian_grid(12, 1, 6)),
    ("dipole", lambda: G.dipole_grid(18, 6, 5)),
]


@pytest.mark.parametrize("name,mk", GRIDS, ids=[c[0] for c in GRIDS])
def test_solve_bodies_equal_the_oracle_on_the_host(harness, name, mk):
    g = mk()
    st = S.init_state(g, seed=21, perturb=0.2)
    O.v12rhov1(g, st)
    O.T2rhoe(g, st)
    keep = []
    v = _view(g, keep)
    dt = 0.1
    # energy
    Pr, Lo, rng = _rates(g, 1, 1e-12)
    Qe = np.asfortranarray(rng.uniform(0, 1e-13, (g.lx1, g.lx2, g.lx3)))
    a, b = st.copy(), st.copy()
    Pa = O.energy_source_loss_solve(g, a, dt, Pr, Lo, Qe)
    Pb = Pr.copy(order="F")
    harness.hs_energy(ctypes.byref(v), dt, _p(Pb), _p(Lo), _p(Qe), _blk(b.fluidauxvars, 1), _blk(b.fluidvars, 4),
                      _blk(b.fluidvars, 0))
    assert np.array_equal(Pb, Pa)
    assert np.array_equal(b.fluidvars, a.fluidvars) and np.array_equal(b.fluidauxvars, a.fluidauxvars)
    # momentum
    Pr, Lo, _ = _rates(g, 2, 1e-20)
    O.momentum_source_loss_solve(g, a, dt, Pr, Lo)
    harness.hs_momentum(ctypes.byref(v), dt, _p(Pr), _p(Lo), _blk(b.fluidvars, 0), _blk(b.fluidauxvars, 0),
                        _blk(b.fluidvars, 1))
    assert np.array_equal(b.fluidvars, a.fluidvars) and np.array_equal(b.fluidauxvars, a.fluidauxvars)
    # mass
    Pr, Lo, rng = _rates(g, 3, 1e6)
    Pp = np.asfortranarray(rng.uniform(0, 1e5, (g.lx1, g.lx2, g.lx3, LSP - 1)))
    Pa = O.mass_source_loss_solve(g, a, dt, Pr, Lo, Pp)
    Pb = Pr.copy(order="F")
    harness.hs_mass(ctypes.byref(v), dt, _p(Pb), _p(Lo), _p(Pp), _blk(b.fluidvars, 0))
    assert np.array_equal(Pb, Pa)
    assert np.array_equal(b.fluidvars, a.fluidvars) and np.array_equal(b.fluidauxvars, a.fluidauxvars)
    assert not np.array_equal(b.fluidvars, st.fluidvars)
