"""gem_dt_calc_noalloc_dev (static device scratch, no allocation) against gem_dt_calc_dev.

Collected last (file name) so it also runs after every other GPU test; it builds its own
state and passes alone in a fresh process as well.
"""
import ctypes

import numpy as np
import pytest

from gemini_b200 import _lib
from gemini_b200 import fluid as F
from gemini_b200 import grid as G
from gemini_b200 import state as S

pytestmark = pytest.mark.gpu


def _dt_pair(dg, ds, tcfl, stream):
    import torch

    L = _lib.lib()
    ref = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    got = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    Fp = ctypes.c_void_p(ds.fluidvars.data_ptr())
    _lib.check(L.gem_dt_calc_dev(dg.handle, tcfl, Fp, ds.work, ctypes.c_void_p(ref.data_ptr()), stream))
    _lib.check(L.gem_dt_calc_noalloc_dev(dg.handle, tcfl, Fp, ctypes.c_void_p(got.data_ptr()), stream))
    torch.cuda.synchronize()
    return float(ref.item()), float(got.item())


@pytest.mark.parametrize("kind", ["dipole", "cartesian"])
def test_noalloc_dt_matches_dt_calc(kind):
    import torch

    g = G.dipole_grid(40, 8, 6) if kind == "dipole" else G.cartesian_grid(20, 10, 8)
    st = S.init_state(g, seed=5, perturb=0.2)
    dg = F.DeviceGrid(g)
    ds = F.DeviceState.from_host(dg, st)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    # two calls in a row: the first resolves the scratch address, the second reuses it
    for _ in range(2):
        ref, got = _dt_pair(dg, ds, 0.5, stream)
        assert ref > 0
        # max over cells is exact and the quotients are IEEE: the two paths agree to the bit
        assert got == ref
    # a changed state moves both the same way
    v = ds.fluidvars.view(-1)
    ng = (g.lx1 + 4) * (g.lx2 + 4) * (g.lx3 + 4)
    v[7 * ng: 14 * ng] *= 3.0  # vs1 of every species
    ref, got = _dt_pair(dg, ds, 0.25, stream)
    assert got == ref


@pytest.mark.parametrize("lx3", [40, 2048])
def test_noalloc_dt_many_planes(lx3):
    """More x3 planes than one finalize pass covers (40) and the largest accepted count
    (2048), on thin columns: bit-identical to gem_dt_calc_dev, two calls in a row."""
    import torch

    g = G.cartesian_grid(4, 2, lx3)
    st = S.init_state(g, seed=lx3, perturb=0.2)
    dg = F.DeviceGrid(g)
    ds = F.DeviceState.from_host(dg, st)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for _ in range(2):
        ref, got = _dt_pair(dg, ds, 0.5, stream)
        assert ref > 0
        assert got == ref


def test_noalloc_rejects_too_many_planes():
    L = _lib.lib()
    lx3 = 2049  # one x3 plane more than the static scratch holds
    g = G.cartesian_grid(4, 1, lx3)
    dg = F.DeviceGrid(g)
    rc = L.gem_dt_calc_noalloc_dev(dg.handle, 0.5, ctypes.c_void_p(0), ctypes.c_void_p(0), None)
    assert rc == _lib.GEM_EINVAL  # null pointers are checked first
    import torch

    buf = torch.zeros(35 * (4 + 4) * (1 + 4) * (lx3 + 4), dtype=torch.float64, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = L.gem_dt_calc_noalloc_dev(dg.handle, 0.5, ctypes.c_void_p(buf.data_ptr()),
                                   ctypes.c_void_p(out.data_ptr()), None)
    assert rc == _lib.GEM_EINVAL
    assert b"2048" in L.gem_last_error()
