"""The drop-in boundary exercised with data: a C++ driver (tests/capi_driver.cpp, built with g++
and linked against libgemini_b200.so) replays the reference driver's fluid_adv
(libgemini.cpp:143-234) through the reference-named C entry points of gemini3d_fluid.h, on
host blocks, for several steps -- advection, compression, diffusion and the source
sub-step -- and the state must match the oracle's full step (ora_fluid_adv_full) at the
full-step tolerance (1e-9: the source rates use the device's pow/exp/log/erf, within a few
ulp of the C library's)."""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

import oracle as O
from gemini_b200 import _lib
from gemini_b200 import build
from gemini_b200 import fluid as F
from gemini_b200 import state as S

from helpers import LSP, cases, state_err
from test_gpu_fullstep import _source_inputs

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = [c for c in cases() if "J1_amp" not in c[2]]


@pytest.fixture(scope="module", autouse=True)
def _device_semantics():
    O.set_device_semantics(True)
    yield
    O.set_device_semantics(False)


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    cxx = shutil.which("g++")
    if not cxx:
        pytest.skip("no g++")
    _lib.lib()  # load the library first: the driver binds to this copy
    libdir = os.path.dirname(build.LIB)
    out = str(tmp_path_factory.mktemp("drv") / "libcapi_driver.so")
    subprocess.check_call([cxx, "-O2", "-std=c++17", "-fPIC", "-shared", "-I", _lib.INCLUDE_DIR,
                           os.path.join(HERE, "capi_driver.cpp"), "-L", libdir, "-lgemini_b200",
                           f"-Wl,-rpath,{libdir}", "-o", out])
    D = ctypes.CDLL(out)
    D.drive_fluid_adv.argtypes = [ctypes.c_void_p] * 9
    D.drive_fluid_adv.restype = None
    return D


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_reference_driver_sequence_vs_oracle(driver, case):
    name, g, kw = case
    L = _lib.lib()
    L.gem_capi_set_error_mode(1)
    st = S.init_state(g, **kw)
    nn, vn, g1, Pri, Qei, alt = _source_inputs(g, st, 61)
    dg = F.DeviceGrid(g)  # creating the grid binds it as the C API's current grid
    work = ctypes.c_void_p()
    _lib.check(L.gem_work_create(dg.handle, ctypes.byref(work)))
    try:
        host = [np.asfortranarray(a, dtype=np.float64) for a in (nn, vn[0], vn[1], vn[2], st.Tn, alt, g1, Pri, Qei)]
        src = F.SourceInputs(*[a.ctypes.data for a in host])
        _lib.check(L.gem_work_set_sources(work, ctypes.byref(src)))
        cfg = _lib.GemCfg(st.Teinf, 2, 0.5, 0)
        h, ref = st.copy(), st.copy()
        lsp, xtype = ctypes.c_int(LSP), ctypes.c_int(1 if name.startswith("dipole") else 0)
        for _ in range(3):
            dt, _ = O.dt_calc(g, ref, 0.5)
            O.fluid_adv_full(g, ref, dt, nn, *vn, g1, Pri, Qei)
            dtc = ctypes.c_double(dt)
            driver.drive_fluid_adv(ctypes.addressof(dtc), ctypes.addressof(lsp), _p(h.fluidvars),
                                   _p(h.fluidauxvars), _p(h.electrovars), ctypes.addressof(xtype),
                                   ctypes.addressof(cfg), dg.handle, work)
            assert L.gem_capi_last_status() == 0, L.gem_last_error()
        assert np.isfinite(h.fluidvars).all()
        err = state_err(h, ref)
        assert max(err.values()) <= 1e-9, err
        assert not np.array_equal(h.fluidvars, st.fluidvars)
    finally:
        L.gem_work_destroy(work)
        L.gem_capi_set_error_mode(0)
        dg.close()
