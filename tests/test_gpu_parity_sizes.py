"""GPU parity at the sizes the benchmarks use, bit for bit against the oracle (restated
LAPACK band solve, correctly rounded T**2.5):

- the Cartesian 96x32x32 workload (field-aligned x1 from 80 to 1000 km, gridflag 2) for its
  100 steps of dt_calc + the fused step;
- full-length dipole columns (lx1 = 384, the benchmark's field lines, +-20 % lognormal
  perturbation) for 10 steps;
- one step for column lengths from the 4-row minimum up to 512 rows;
- one step of the whole 384x192x192 dipole workload.

Each step's dt and the whole state after the last step must be identical.  The oracle runs
multithreaded; the full-size case needs about 30 GB of host memory.
"""
import numpy as np
import pytest

import oracle as O
from gemini_b200 import fluid as F
from gemini_b200 import grid as G
from gemini_b200 import state as S

from helpers import assert_identical

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _device_semantics():
    O.set_device_semantics(True)
    yield
    O.set_device_semantics(False)


def _run(g, kw, nsteps, solver=2):
    st = S.init_state(g, **kw)
    dg = F.DeviceGrid(g)
    ds = F.DeviceState.from_host(dg, st.copy())
    cfg = F.FluidCfg(st.Teinf, solver)
    ref = st.copy()
    dts = O.run_steps(g, ref, nsteps, diffsolvetype=solver)
    for k in range(nsteps):
        dt = F.dt_calc(ds, 0.5)
        got = float(dt.item())
        assert got == dts[k], f"step {k}: dt {got!r} vs {dts[k]!r}"
        F.fluid_adv(cfg, ds, dt)
    assert F.check_finite(ds) == 0
    return ds.to_host(st), ref


def test_cartesian_96x32x32_100_steps():
    g = G.cartesian_grid(96, 32, 32)
    assert g.gridflag == 2
    got, ref = _run(g, dict(seed=0), 100)
    assert_identical(got, ref, "Cartesian 96x32x32, 100 steps")


@pytest.mark.parametrize("lx2,lx3,seed", [(8, 6, 11), (16, 8, 12)])
def test_dipole_full_columns_10_steps(lx2, lx3, seed):
    g = G.dipole_grid(384, lx2, lx3)
    got, ref = _run(g, dict(seed=seed, perturb=0.2), 10)
    assert_identical(got, ref, f"dipole 384x{lx2}x{lx3}, 10 steps")


@pytest.mark.parametrize("lx1", [4, 5, 7, 31, 32, 33, 63, 97, 128, 255, 256, 384, 512])
@pytest.mark.parametrize("solver", [2, 1])
def test_column_lengths_one_step(lx1, solver):
    g = G.dipole_grid(lx1, 3, 2) if lx1 >= 16 else G.cartesian_grid(lx1, 3, 2)
    got, ref = _run(g, dict(seed=lx1, perturb=0.2), 1, solver)
    assert_identical(got, ref, f"lx1={lx1}, solver {solver}")


def test_full_size_dipole_one_step():
    g = G.dipole_grid(384, 192, 192)
    got, ref = _run(g, dict(seed=1, perturb=0.2), 1)
    assert_identical(got, ref, "dipole 384x192x192, one step")
