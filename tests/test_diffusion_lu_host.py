"""The device diffusion kernel's per-column body (gem_diffusion_lu.cuh: thermal_conduct,
diffusion_prep and the TRBDF2 / backward-Euler band systems in registers, factored and solved
in LAPACK dgbsv's operation order), compiled for the host and run over every column and
species, against the oracle's energy_diffusion with the restated LAPACK solve
(PDEparabolic.f90:142,216,337 -> gbsv.in.f90:90) bit for bit.

The oracle runs with its correctly rounded T**2.5 (pow mode 1), the one dependency the device
evaluates differently from the reference's C-library pow.  The stiff cases pivot on the
Dirichlet identity rows and inside the columns; their LAPACK-order results sit ~1e-10 away
from an exact solve of the same systems, so agreement to the last bit shows the solve follows
LAPACK's order, not merely its solution."""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

import oracle as O
from gemini_b200 import grid as G
from gemini_b200 import state as S

from helpers import cases, harness_flags

LSP = 7
HERE = os.path.dirname(os.path.abspath(__file__))
_D = ctypes.POINTER(ctypes.c_double)


class HDiff(ctypes.Structure):
    _fields_ = [("lx1", ctypes.c_int), ("lx2", ctypes.c_int), ("lx3", ctypes.c_int), ("gridflag", ctypes.c_int),
                ("solver", ctypes.c_int), ("unit", ctypes.c_int), ("dt", ctypes.c_double),
                ("Teinf", ctypes.c_double)] + [(n, _D) for n in ("h1", "h2", "h3", "dx1", "dx1i", "Ttop")]


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    cxx = shutil.which("g++")
    if not cxx:
        pytest.skip("no g++")
    out = str(tmp_path_factory.mktemp("dlu") / "libdlu.so")
    subprocess.check_call([cxx, "-O2", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", *harness_flags(),
                           "-o", out, os.path.join(HERE, "diffusion_lu_harness.cpp")])
    L = ctypes.CDLL(out)
    L.hd_energy_diffusion.argtypes = [ctypes.POINTER(HDiff), _D, _D, _D, _D, _D]
    L.hd_energy_diffusion.restype = ctypes.c_int
    return L


@pytest.fixture(autouse=True)
def _lapack_order_oracle():
    O.set_diffusion_solver(0)  # the restated LAPACK dgbsv
    O.set_pow_mode(1)          # correctly rounded T**2.5, as the device
    yield
    O.set_exact_dependencies(False)


def _p(a):
    return a.ctypes.data_as(_D)


def run_harness(L, g, st, dt, solver, Ttop=None):
    keep = [np.asfortranarray(getattr(g, n), dtype=np.float64) for n in ("h1", "h2", "h3")]
    dx1 = np.ascontiguousarray(g.dx1, dtype=np.float64)
    dx1i = np.ascontiguousarray(g.dx1i, dtype=np.float64)
    keep += [dx1, dx1i]
    h = HDiff(g.lx1, g.lx2, g.lx3, g.gridflag, solver, int(g.unit_metrics), float(dt), float(st.Teinf),
              _p(keep[0]), _p(keep[1]), _p(keep[2]), _p(dx1), _p(dx1i),
              _p(Ttop) if Ttop is not None else ctypes.cast(None, _D))
    fv = st.fluidvars
    ng = fv.shape[0] * fv.shape[1] * fv.shape[2]
    base = fv.ctypes.data
    ns = ctypes.cast(base, _D)
    Ts = ctypes.cast(base + 8 * 4 * LSP * ng, _D)
    J1 = np.asfortranarray(st.electrovars[..., 3])
    rc = L.hd_energy_diffusion(ctypes.byref(h), ns, Ts, _p(J1), _p(st.nn), _p(st.Tn))
    assert rc == 0
    # the ghost cells other than the x1 boundary layers take max(T,100) (multifluid.f90:340)
    fv[..., 4 * LSP:5 * LSP] = np.maximum(fv[..., 4 * LSP:5 * LSP], 100.0)


GRIDS = cases() + [
    ("dipole384", G.dipole_grid(384, 4, 3), dict(seed=21, perturb=0.2)),
    ("cart96", G.cartesian_grid(96, 6, 4), dict(seed=22)),
    ("dipole_j1", G.dipole_grid(64, 5, 4), dict(seed=23, perturb=0.2, J1_amp=2e-5)),
]


@pytest.mark.parametrize("solver", [2, 1])
@pytest.mark.parametrize("dtscale", [1.0, 30.0])
@pytest.mark.parametrize("case", GRIDS, ids=[c[0] for c in GRIDS])
def test_body_equals_lapack_order_oracle(harness, case, dtscale, solver):
    name, g, kw = case
    st = S.init_state(g, **kw)
    dt, _ = O.dt_calc(g, st, 0.5)
    dt *= dtscale
    ref = st.copy()
    O.energy_diffusion(g, ref, dt, solver)
    got = st.copy()
    run_harness(harness, g, got, dt, solver)
    a, b = got.fluidvars[..., 4 * LSP:], ref.fluidvars[..., 4 * LSP:]
    if not np.array_equal(a, b):
        bad = np.argwhere(a != b)
        i = tuple(bad[0])
        rel = np.max(np.abs(a - b) / np.abs(b))
        raise AssertionError(f"{name}: {len(bad)} cells differ (max rel {rel:.3g}), first {i}: {a[i]!r} vs {b[i]!r}")


def test_stiff_columns_pivot_and_differ_from_an_exact_solve(harness):
    """On the stiff dipole column set the LAPACK-order solution is measurably not the exact
    one, so bit equality with it is a statement about the operation order."""
    g = G.dipole_grid(384, 4, 3)
    st = S.init_state(g, seed=21, perturb=0.2)
    dt, _ = O.dt_calc(g, st, 0.5)
    lap = st.copy()
    O.energy_diffusion(g, lap, dt, 2)
    O.set_diffusion_solver(1)
    ex = st.copy()
    O.energy_diffusion(g, ex, dt, 2)
    O.set_diffusion_solver(0)
    T_l, T_e = lap.fluidvars[..., 4 * LSP:], ex.fluidvars[..., 4 * LSP:]
    spread = float(np.max(np.abs(T_l - T_e) / T_e))
    assert spread > 1e-12, spread
    got = st.copy()
    run_harness(harness, g, got, dt, 2)
    assert np.array_equal(got.fluidvars[..., 4 * LSP:], T_l)


def test_per_column_top_temperature_equals_scalar(harness):
    g = G.cartesian_grid(20, 5, 4)
    st = S.init_state(g, seed=3)
    dt, _ = O.dt_calc(g, st, 0.5)
    a, b = st.copy(), st.copy()
    run_harness(harness, g, a, dt, 2)
    run_harness(harness, g, b, dt, 2, Ttop=np.full(g.lx2 * g.lx3, st.Teinf))
    assert np.array_equal(a.fluidvars, b.fluidvars)
