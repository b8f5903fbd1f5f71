"""GPU parity: every reference routine on the device against the CPU oracle.

Advection, ghost fill, interface velocities, conversions, clean_param and dt_calc are
restated with the reference's operation order and no FMA.  The diffusion forms its band
systems in the reference's order and factors/solves them in LAPACK dgbsv's order
(dgbtf2 partial pivoting, dgbtrs/dtbsv), so every routine and the fused step must match the
oracle bit for bit.  The oracle runs its restated LAPACK solve with the correctly rounded
T**2.5 (the device's one departure from the reference's C-library pow; the spread that a
one-ulp change of pow causes is measured in test_gpu_parity_sizes.py).
"""
import numpy as np
import pytest

import oracle as O
from gemini_b200 import fluid as F
from gemini_b200 import state as S

from helpers import assert_identical, cases, randomize_interface_vels

pytestmark = pytest.mark.gpu

CASES = cases()
IDS = [c[0] for c in CASES]


@pytest.fixture(scope="module", autouse=True)
def _device_semantics():
    O.set_device_semantics(True)
    yield
    O.set_device_semantics(False)


def _setup(case, seed_iv=11):
    name, g, kw = case
    st = S.init_state(g, **kw)
    randomize_interface_vels(st, seed_iv)
    dg = F.DeviceGrid(g)
    ds = F.DeviceState.from_host(dg, st.copy())
    return g, st, dg, ds


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_conversions_exact(case):
    g, st, dg, ds = _setup(case)
    for fn_o, fn_g in ((O.v12rhov1, F.v12rhov1), (O.T2rhoe, F.T2rhoe),
                       (O.rhov12v1, F.rhov12v1), (O.rhoe2T, F.rhoe2T)):
        fn_o(g, st)
        fn_g(ds)
        assert_identical(ds.to_host(st), st, fn_g.__name__)


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_global_boundaries_and_halo_exact(case):
    g, st, dg, ds = _setup(case)
    O.v12rhov1(g, st); O.T2rhoe(g, st)
    F.v12rhov1(ds); F.T2rhoe(ds)
    O.set_global_boundaries(g, st)
    F.set_global_boundaries_allspec(ds)
    assert_identical(ds.to_host(st), st, "set_global_boundaries_allspec")
    O.halo_fluidvars(g, st)
    F.halo_fluidvars(ds)
    assert_identical(ds.to_host(st), st, "halo_fluidvars")
    O.halo_allparams(g, st)
    F.halo_allparams(ds)
    assert_identical(ds.to_host(st), st, "halo_allparams")


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_interface_vels_exact(case):
    g, st, dg, ds = _setup(case)
    O.interface_vels(g, st)
    F.interface_vels_allspec(ds)
    for w, ref in ((1, st.vs1i), (2, st.vs2i), (3, st.vs3i)):
        got = ds.interface_vels(w)
        assert np.array_equal(got, ref), f"vs{w}i differs at {np.argwhere(got != ref)[:3]}"


@pytest.mark.parametrize("case", CASES, ids=IDS)
@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("which", ["mass", "momentum", "energy"])
def test_sweep_exact(case, dim, which):
    g, st, dg, ds = _setup(case)
    O.v12rhov1(g, st); O.T2rhoe(g, st)
    F.v12rhov1(ds); F.T2rhoe(ds)
    dt = 0.37
    O.sweep(g, st, dim, which, dt)
    getattr(F, f"sweep{dim}_allspec_{which}")(ds, dt)
    assert_identical(ds.to_host(st), st, f"sweep{dim}_allspec_{which}")


@pytest.mark.parametrize("case", CASES, ids=IDS)
@pytest.mark.parametrize("iparm", [1, 2, 3])
def test_clean_param_exact(case, iparm):
    g, st, dg, ds = _setup(case)
    O.clean_param(g, st, iparm)
    F.clean_param(ds, iparm)
    assert_identical(ds.to_host(st), st, f"clean_param({iparm})")


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_dt_calc_and_maxcfl_exact(case):
    g, st, dg, ds = _setup(case)
    dt_ref, _ = O.dt_calc(g, st, 0.5)
    dt = F.dt_calc(ds, 0.5)
    assert float(dt.item()) == dt_ref
    # cflcalc at that dt: the CFL number the reference would report
    got = F.maxcfl(ds, dt_ref)
    assert got == pytest.approx(0.5, rel=1e-12)


@pytest.mark.parametrize("case", CASES, ids=IDS)
@pytest.mark.parametrize("solver", [2, 1])
@pytest.mark.parametrize("dtscale", [1.0, 30.0])
def test_energy_diffusion_exact(case, solver, dtscale):
    """energy_diffusion bit for bit, at the CFL step and at a 30x stiffer one (pivots on
    the Dirichlet rows and inside the columns)."""
    g, st, dg, ds = _setup(case)
    dt, _ = O.dt_calc(g, st, 0.5)
    dt *= dtscale
    O.energy_diffusion(g, st, dt, solver)
    F.energy_diffusion(F.FluidCfg(st.Teinf, solver), ds, dt)
    assert_identical(ds.to_host(st), st, f"energy_diffusion solver {solver}")


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_fused_step_equals_reference_order(case):
    """The fused kernels compute exactly what the routine-by-routine sequence computes."""
    name, g, kw = case
    st = S.init_state(g, **kw)
    dg = F.DeviceGrid(g)
    a = F.DeviceState.from_host(dg, st.copy())
    b = F.DeviceState.from_host(dg, st.copy())
    cfg = F.FluidCfg(st.Teinf)
    for _ in range(2):
        dt = F.dt_calc(a, 0.5)
        F.fluid_adv(cfg, a, dt)
        dtb = F.dt_calc(b, 0.5)
        F.fluid_adv_reference_order(cfg, b, dtb)
    ha, hb = a.to_host(st), b.to_host(st)
    assert_identical(ha, hb, "fused vs reference order")
    for w in (1,):
        va, vb = a.interface_vels(w), b.interface_vels(w)
        assert np.array_equal(va[0], vb[0]) and np.array_equal(va[-1], vb[-1])


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_fused_steps_vs_oracle(case):
    """dt_calc + the fused step, five times: every dt and the whole state bit for bit."""
    name, g, kw = case
    st = S.init_state(g, **kw)
    dg = F.DeviceGrid(g)
    ds = F.DeviceState.from_host(dg, st.copy())
    cfg = F.FluidCfg(st.Teinf)
    ref = st.copy()
    nsteps = 5
    dts_ref = O.run_steps(g, ref, nsteps)
    for k in range(nsteps):
        dt = F.dt_calc(ds, 0.5)
        assert float(dt.item()) == dts_ref[k]
        F.fluid_adv(cfg, ds, dt)
    assert_identical(ds.to_host(st), ref, f"{name}: {nsteps} fused steps")
    assert F.check_finite(ds) == 0


@pytest.mark.parametrize("solver", [2, 1])
def test_single_step_bits_match(solver):
    """One fused step from identical inputs, both diffusion solvers: the whole state."""
    name, g, kw = CASES[4]
    st = S.init_state(g, **kw)
    dg = F.DeviceGrid(g)
    ds = F.DeviceState.from_host(dg, st.copy())
    ref = st.copy()
    dt, _ = O.dt_calc(g, ref, 0.5)
    O.fluid_adv(g, ref, dt, solver)
    F.fluid_adv(F.FluidCfg(st.Teinf, solver), ds, dt)
    assert_identical(ds.to_host(st), ref, "one fused step")


@pytest.mark.parametrize("ci", [4, 2, 3], ids=["dipole", "cart_periodic", "cart_2d"])
def test_host_entry_point_matches_device(ci):
    """gem_fluid_adv_host leaves the host blocks exactly as the device step leaves its own:
    every block, the ghost shell of vs2 and vs3 included (the only part of them copied back),
    on a dipole, an x3-periodic and a single-x3-plane grid."""
    name, g, kw = CASES[ci]
    st = S.init_state(g, **kw)
    dg = F.DeviceGrid(g)
    a = F.DeviceState.from_host(dg, st.copy())
    cfg = F.FluidCfg(st.Teinf)
    dt = F.dt_calc(a, 0.5)
    F.fluid_adv(cfg, a, dt)
    b = F.DeviceState.from_host(dg, st.copy())
    h = st.copy()
    # the step recomputes rhovs1|rhoes, ignores all electrovars but J1 and leaves the MHD
    # scalars alone: garbage there must not matter, and the MHD scalars must survive
    rng = np.random.default_rng(0)
    h.fluidauxvars[...] = rng.uniform(-1e3, 1e3, h.fluidauxvars.shape)
    mhd = h.fluidauxvars[..., 2 * 7:].copy()
    keep_J1 = h.electrovars[..., 3].copy()
    h.electrovars[...] = rng.uniform(-1, 1, h.electrovars.shape)
    h.electrovars[..., 3] = keep_J1
    dth = F.fluid_adv_host(cfg, dg, b, h.fluidvars, h.fluidauxvars, h.electrovars, -1.0)
    assert dth == float(dt.item())
    ga = a.to_host(st)
    assert np.array_equal(ga.fluidvars, h.fluidvars)
    assert np.array_equal(ga.fluidauxvars[..., :2 * 7], h.fluidauxvars[..., :2 * 7])
    assert np.array_equal(h.fluidauxvars[..., 2 * 7:], mhd)


@pytest.mark.parametrize("field,where", [("dx2", (0,)), ("dx3", (-1,)), ("dx1", (3,)), ("h1x1i", (5, 2, 1)),
                                         ("h3", (4, 3, 3))])
def test_grid_with_reciprocal_out_of_exact_range_is_rejected(field, where):
    """The sweeps' and the diffusion's exact quotients take every grid reciprocal from tables
    checked at grid creation to lie in [2^-400, 2^400] (ghost spacings included); a grid
    with one entry outside is refused with GEM_EINVAL instead of dividing inexactly."""
    import copy

    from gemini_b200 import _lib
    from gemini_b200 import grid as G

    g = G.dipole_grid(12, 6, 5)
    bad = copy.deepcopy(g)
    a = np.array(getattr(bad, field), dtype=np.float64, copy=True)
    a[where] = 1e-200  # its reciprocal (or that of a product with it) exceeds 2^400 ~ 2.6e120
    setattr(bad, field, a)
    F.DeviceGrid(g).close()
    with pytest.raises(_lib.GemError) as e:
        F.DeviceGrid(bad)
    assert e.value.code == 1  # GEM_EINVAL
