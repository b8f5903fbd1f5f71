"""Host-side logic without a GPU: grid/state generators and the C ABI library surface."""
import ctypes
import os

import numpy as np
import pytest

from gemini_b200 import _lib, build
from gemini_b200 import grid as G
from gemini_b200 import state as S


def test_coord_diffs_definition():
    x = np.cumsum(np.random.default_rng(0).uniform(1, 2, 14))
    dx, xi, dxi = G.coord_diffs(x)
    lx = x.size - 4
    assert dx.size == lx + 3 and xi.size == lx + 1 and dxi.size == lx
    assert np.array_equal(dx, x[1:] - x[:-1])
    assert np.array_equal(xi, 0.5 * (x[1:lx + 2] + x[2:lx + 3]))


def test_cartesian_grid():
    g = G.cartesian_grid(12, 5, 4)
    assert g.gridflag == 2 and g.unit_metrics and g.lnull == 0
    assert g.h1.shape == (16, 9, 8) and g.h1.flags.f_contiguous
    assert g.h2x1i.shape == (13, 5, 4) and g.h3x2i.shape == (12, 6, 4) and g.h1x3i.shape == (12, 5, 5)
    gi = G.cartesian_grid(12, 5, 4, inverted=True)
    assert gi.gridflag == 1


def test_dipole_grid():
    g = G.dipole_grid(48, 6, 4)
    assert g.gridflag == 0 and g.lnull == 0
    assert (g.h1 > 0).all() and (g.h2 > 0).all() and (g.h3 > 0).all()
    alt = g.alt[2:-2, 2:-2, 2:-2]
    assert alt.min() >= 80e3 - 1 and abs(alt[0, 0, 0] - 90e3) < 1.0
    # metric factors do not depend on x3
    assert np.array_equal(g.h1[:, :, 0], g.h1[:, :, -1])
    gn = G.dipole_grid(48, 6, 4, q_extent=0.5)
    assert gn.lnull > 0


def test_dipole_rtheta_roundtrip():
    q = np.array([-0.3, 0.0, 0.2])
    p = np.array([1.5, 2.0, 3.0])
    r, th = G.dipole_rtheta(q, p)
    qq = (G.RE / r) ** 2 * np.cos(th)
    pp = r / G.RE / np.sin(th) ** 2
    assert np.allclose(qq, q, atol=1e-14) and np.allclose(pp, p, rtol=1e-14)


def test_state_generator():
    g = G.cartesian_grid(20, 4, 3)
    st = S.init_state(g, seed=1)
    ns = st.ns
    assert (ns[..., :6] >= 1e6).all()
    assert np.array_equal(ns[..., 6], ns[..., :6].sum(axis=-1))
    assert (st.Ts >= 100).all()
    assert st.nn.shape == (20, 4, 3, 3) and st.Tn.shape == (20, 4, 3)
    st2 = S.init_state(g, seed=1)
    assert np.array_equal(st.fluidvars, st2.fluidvars)


def test_library_builds_and_exports_header_symbols():
    """The C-ABI library loads without a GPU and exports every function include/*.h declares."""
    try:
        build.build()
    except RuntimeError as e:  # no nvcc in this environment
        if not os.path.exists(build.LIB):
            pytest.skip(str(e))
    L = ctypes.CDLL(build.LIB)
    names = _lib.header_symbols()
    assert len(names) > 40
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert _lib.lib().gem_version() >= 1


def test_device_abi_rejects_bad_arguments_without_a_gpu():
    """The device C ABI checks its arguments before any CUDA call: null handles, null
    buffers and impossible sizes come back as GEM_EINVAL with a message (no exit, no fault),
    on a machine without a GPU as on one with."""
    try:
        build.build()
    except RuntimeError as e:  # no nvcc in this environment
        if not os.path.exists(build.LIB):
            pytest.skip(str(e))
    L = _lib.lib()
    EINVAL = 1
    out = ctypes.c_void_p()
    desc = _lib.GemGridDesc()
    desc.lx1, desc.lx2, desc.lx3, desc.gridflag = 0, 4, 4, 0
    cfg = _lib.GemCfg()
    cfg.Teinf, cfg.diffsolvetype = 1500.0, 2
    calls = {
        "gem_grid_create (null desc)": lambda: L.gem_grid_create(None, ctypes.byref(out)),
        "gem_grid_create (lx1 = 0)": lambda: L.gem_grid_create(ctypes.byref(desc), ctypes.byref(out)),
        "gem_work_create": lambda: L.gem_work_create(None, ctypes.byref(out)),
        "gem_step_adjoint_create": lambda: L.gem_step_adjoint_create(None, ctypes.byref(out)),
        "gem_fluid_adv_dev": lambda: L.gem_fluid_adv_dev(ctypes.byref(cfg), None, None, None, None, None, None, None),
        "gem_dt_calc_noalloc_dev": lambda: L.gem_dt_calc_noalloc_dev(None, 0.5, None, None, None),
        "gem_step_vjp_replay_dev": lambda: L.gem_step_vjp_replay_dev(ctypes.byref(cfg), *([None] * 12)),
        "gem_step_vjp_finish_dev": lambda: L.gem_step_vjp_finish_dev(ctypes.byref(cfg), *([None] * 10)),
        "gem_batch_create": lambda: L.gem_batch_create(0, None, None, None, None, None, None, ctypes.byref(out)),
        "gem_vnricht_artvisc_dev": lambda: L.gem_vnricht_artvisc_dev(None, None, None, None),
        "gem_rk2_global_boundary_allspec_dev": lambda: L.gem_rk2_global_boundary_allspec_dev(None, None, None),
        "gem_compression_dev": lambda: L.gem_compression_dev(*([None] * 6)),
        "gem_energy_source_loss_solve_dev": lambda: L.gem_energy_source_loss_solve_dev(*([None] * 8)),
        "gem_momentum_source_loss_solve_dev": lambda: L.gem_momentum_source_loss_solve_dev(*([None] * 7)),
        "gem_mass_source_loss_solve_dev": lambda: L.gem_mass_source_loss_solve_dev(*([None] * 7)),
        "gem_srcs_continuity_dev": lambda: L.gem_srcs_continuity_dev(*([None] * 10)),
        "gem_srcs_energy_dev": lambda: L.gem_srcs_energy_dev(*([None] * 10)),
        "gem_srcs_momentum_dev": lambda: L.gem_srcs_momentum_dev(*([None] * 12)),
        "gem_fluid_adv_compression_dev": lambda: L.gem_fluid_adv_compression_dev(ctypes.byref(cfg), *([None] * 7)),
        "gem_source_loss_allparams_dev": lambda: L.gem_source_loss_allparams_dev(*([None] * 11)),
        "gem_fluid_adv_full_dev": lambda: L.gem_fluid_adv_full_dev(ctypes.byref(cfg), *([None] * 9)),
        "gem_dt_select_dev": lambda: L.gem_dt_select_dev(ctypes.byref(cfg), *([None] * 6)),
        "gem_clock_advance_dev": lambda: L.gem_clock_advance_dev(None, None, None),
        "gem_work_set_sources": lambda: L.gem_work_set_sources(None, None),
        "gem_work_prepare": lambda: L.gem_work_prepare(None, None),
        "gem_work_substep_buffers": lambda: L.gem_work_substep_buffers(None, None, None, None, None),
    }
    for name, call in calls.items():
        assert call() == EINVAL, name
        assert L.gem_last_error().decode(), name
    assert out.value is None
    assert L.gem_fluid_adv_full_scratch_doubles(None) == -1


_CAPI_PROBE = r"""
import ctypes, sys
L = ctypes.CDLL(sys.argv[1])
PP = ctypes.POINTER(ctypes.c_void_p)
L.v12rhov1_C.argtypes = [PP, PP]
L.gem_capi_set_error_mode.argtypes = [ctypes.c_int]
L.gem_capi_set_error_mode(int(sys.argv[2]))
fv, fav = ctypes.c_void_p(None), ctypes.c_void_p(None)
L.v12rhov1_C(ctypes.byref(fv), ctypes.byref(fav))   # no grid bound
print("returned", L.gem_capi_last_status())
"""


def test_capi_error_behaviour_without_a_gpu():
    """The reference-named *_C entry points stop the program on error, printing the
    message and exiting 1 as the reference's error stop does; in record-only mode they return
    and leave the status to gem_capi_last_status.  Called with no grid bound, they fail before
    any CUDA call."""
    import subprocess
    import sys

    try:
        build.build()
    except RuntimeError as e:  # no nvcc in this environment
        if not os.path.exists(build.LIB):
            pytest.skip(str(e))
    r = subprocess.run([sys.executable, "-c", _CAPI_PROBE, build.LIB, "0"], capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 1 and "v12rhov1_C" in r.stderr and "returned" not in r.stdout
    r = subprocess.run([sys.executable, "-c", _CAPI_PROBE, build.LIB, "1"], capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0 and "returned 1" in r.stdout


def test_bench_reference_arm_line_without_a_gpu():
    """bench.py --impl reference times the oracle port on the host cores and prints one JSON
    line with the contract's keys: impl, the same metric/unit/config as the product arm, a
    cpu_baseline describing the run with its value equal to the line's, and an e2e block with
    no host<->device bytes."""
    import json
    import subprocess
    import sys

    here = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, os.path.join(here, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0", "--cpu-seconds", "0.5"], capture_output=True, text=True, timeout=600,
                       cwd=here)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["metric"] == "fluid Gcell-species-steps/s"
    assert line["unit"] == "Gcell-species-steps/s" and line["value"] > 0 and line["steps"] == 1
    assert line["higher_is_better"] is True and line["n_gpus"] == 1
    assert line["config"]["lx1"] == 384 and line["config"]["lx2"] == 192 and line["config"]["lx3"] == 192
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["sample"] and cb["value"] == line["value"]
    e2e = line["e2e"]
    assert e2e["value"] == line["value"] and e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
