"""The device compression kernels' per-index bodies (gem_compression.cuh), compiled for the
host and run over every index of their ranges, against the oracle's compression sub-step
(VNRicht_artvisc, RK2_global_boundary, compression) bit for bit: the same check the GPU
parity test makes, with the index arithmetic exercised over the whole grid on the CPU.
The metric tables are laid out as the device holds them (none on unit-metric grids, one
x3 slice with stride 0 when they do not vary along x3)."""
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


class HView(ctypes.Structure):
    _fields_ = [("lx1", ctypes.c_int), ("lx2", ctypes.c_int), ("lx3", ctypes.c_int), ("flagper", ctypes.c_int),
                ("c3", ctypes.c_longlong)] + [(n, _D) for n in ("h1", "h2", "h3", "dx1", "dx2", "dx3", "ms", "gm1")]


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    cxx = shutil.which("g++")
    if not cxx:
        pytest.skip("no g++")
    out = str(tmp_path_factory.mktemp("cmp") / "libcmp.so")
    subprocess.check_call([cxx, "-O2", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", *harness_flags(), "-o", out,
                           os.path.join(HERE, "compression_harness.cpp")])
    L = ctypes.CDLL(out)
    P = ctypes.POINTER(HView)
    L.hc_artvisc.argtypes = [P, _D, _D, _D]
    L.hc_rk2.argtypes = [P, _D, _D, _D]
    L.hc_compression.argtypes = [P, _D, _D, _D, _D, _D, ctypes.c_double]
    return L


def _p(a):
    return a.ctypes.data_as(_D)


def _view(g, keep):
    """The metric layout the device uses (gem_grid_create)."""
    lx1, lx2, lx3 = g.lx1, g.lx2, g.lx3
    ms, _, gam, _ = O.constants()
    arrs = {"ms": np.ascontiguousarray(ms), "gm1": np.ascontiguousarray(gam - 1)}
    for n in ("dx1", "dx2", "dx3"):
        arrs[n] = np.ascontiguousarray(getattr(g, n), dtype=np.float64)
    hs = [np.asfortranarray(getattr(g, n)) for n in ("h1", "h2", "h3")]
    c3 = (lx1 + 4) * (lx2 + 4)
    if g.unit_metrics:
        hp = [None, None, None]
    else:
        inv = all(np.array_equal(h[:, :, k], h[:, :, 2]) for h in hs for k in range(2, lx3 + 2))
        if inv:  # one slice (ghosted x3 index 2) and x3 stride 0
            hs = [np.asfortranarray(h[:, :, 2]) for h in hs]
            c3 = 0
        hp = hs
    keep.extend([a for a in hp if a is not None] + list(arrs.values()))
    v = HView(lx1=lx1, lx2=lx2, lx3=lx3, flagper=g.flagper, c3=c3,
              **{n: (_p(a) if a is not None else _D()) for n, a in zip(("h1", "h2", "h3"), hp)},
              **{n: _p(a) for n, a in arrs.items()})
    return v, c3


CASES = [
    ("cart", lambda: G.cartesian_grid(14, 6, 5)),
    ("cart_periodic", lambda: G.cartesian_grid(12, 5, 6, flagper=1)),
    ("cart_2d", lambda: G.cartesian_grid(12, 1, 6)),
    ("dipole", lambda: G.dipole_grid(18, 6, 5)),
    ("cart_inverted", lambda: G.cartesian_grid(10, 4, 4, inverted=True)),
]


@pytest.mark.parametrize("name,mk", CASES, ids=[c[0] for c in CASES])
def test_device_bodies_equal_the_oracle_on_the_host(harness, name, mk):
    g = mk()
    st = S.init_state(g, seed=11, perturb=0.2)
    rng = np.random.default_rng(11)
    fv = st.fluidvars
    fv[..., LSP:4 * LSP] = rng.uniform(-800, 800, fv[..., LSP:4 * LSP].shape)  # ghosts too
    O.T2rhoe(g, st)
    a = st.copy()   # oracle
    b = st.copy()   # device bodies on the host
    dt = 0.07
    Qa = O.vnricht_artvisc(g, a)
    O.halo_fluidvars(g, a)
    O.rk2_global_boundary(g, a)
    O.compression(g, a, dt, Qa)
    keep = []
    v, _ = _view(g, keep)
    O.halo_fluidvars(g, b)  # the reference's halo (the device has gem_halo_fluidvars_dev)
    ng = (g.lx1 + 4) * (g.lx2 + 4) * (g.lx3 + 4)
    base = b.fluidvars.ctypes.data
    vs = [ctypes.cast(base + 8 * k * LSP * ng, _D) for k in (1, 2, 3)]
    Qb = np.zeros((g.lx1, g.lx2, g.lx3, LSP), order="F")
    # Q from the state before the halo and the zero-order hold, as the oracle
    c = st.copy()
    harness.hc_artvisc(ctypes.byref(v), _p(c.fluidvars), ctypes.cast(c.fluidvars.ctypes.data + 8 * LSP * ng, _D),
                       _p(Qb))
    assert np.array_equal(Qb, Qa)
    harness.hc_rk2(ctypes.byref(v), *vs)
    assert np.array_equal(b.fluidvars, a.fluidvars)
    re = ctypes.cast(b.fluidauxvars.ctypes.data + 8 * LSP * ng, _D)
    harness.hc_compression(ctypes.byref(v), *vs, _p(Qb), re, dt)
    assert np.array_equal(b.fluidauxvars[..., LSP:2 * LSP], a.fluidauxvars[..., LSP:2 * LSP])
    assert not np.array_equal(a.fluidauxvars[..., LSP:2 * LSP], st.fluidauxvars[..., LSP:2 * LSP])
