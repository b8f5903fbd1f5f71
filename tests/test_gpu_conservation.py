"""Mass conservation of the device advection (north-star property): with zero velocity on
the two end faces of every line, a sweep is a pure flux difference, so
sum(f * ha1 * dxi) along each line is conserved to round-off."""
import ctypes

import numpy as np
import pytest

from gemini_b200 import _lib
from gemini_b200 import fluid as F
from gemini_b200 import grid as G
from gemini_b200 import state as S

pytestmark = pytest.mark.gpu

CASES = [("cart", lambda: G.cartesian_grid(40, 12, 10)), ("dipole", lambda: G.dipole_grid(64, 10, 8))]


@pytest.mark.parametrize("name,mk", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("dim,frank", [(1, 0), (2, 0), (2, 1), (3, 0), (3, 1)])
def test_device_sweep_conserves_with_closed_ends(name, mk, dim, frank):
    import torch

    g = mk()
    st = S.init_state(g, seed=9, perturb=0.2)
    dg = F.DeviceGrid(g)
    X1, X2, X3 = g.lx1 + 4, g.lx2 + 4, g.lx3 + 4
    f = torch.from_numpy(np.ascontiguousarray(st.fluidvars[..., 0:7].transpose(3, 2, 1, 0))).cuda()
    vshape = {1: (7, g.lx3, g.lx2, g.lx1 + 1), 2: (7, g.lx3, g.lx2 + 1, g.lx1), 3: (7, g.lx3 + 1, g.lx2, g.lx1)}[dim]
    rng = np.random.default_rng(dim)
    v = rng.uniform(-300, 300, vshape)
    ax = {1: 3, 2: 2, 3: 1}[dim]
    sl = [slice(None)] * 4
    for end in (0, -1):
        sl[ax] = end
        v[tuple(sl)] = 0.0
    v = torch.from_numpy(v).cuda()
    dt = torch.full((1,), 2.0, dtype=torch.float64, device="cuda")
    # weights: ha1 (frank-dependent) * dxi along the swept direction, interior cells
    h1, h2, h3 = (np.ascontiguousarray(h.transpose(2, 1, 0)) for h in (g.h1, g.h2, g.h3))
    ha1 = (h1 * h1 * h2 * h3) if frank else (h1 * h2 * h3)
    I = (slice(2, g.lx3 + 2), slice(2, g.lx2 + 2), slice(2, g.lx1 + 2))
    dxi = {1: g.dx1i[None, None, :], 2: g.dx2i[None, :, None], 3: g.dx3i[:, None, None]}[dim]
    w = ha1[I] * dxi

    def line_sums(t):
        a = t.cpu().numpy()[(slice(0, 7),) + I] * w
        return a.sum(axis=ax)

    before = line_sums(f)
    _lib.check(_lib.lib().gem_sweep_field_dev(dg.handle, dim, frank, 7, ctypes.c_void_p(f.data_ptr()),
                                              ctypes.c_void_p(v.data_ptr()), ctypes.c_void_p(dt.data_ptr()),
                                              ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    torch.cuda.synchronize()
    after = line_sums(f)
    assert not np.array_equal(f.cpu().numpy(), st.fluidvars[..., 0:7].transpose(3, 2, 1, 0))  # it moved
    assert np.max(np.abs(after - before) / np.abs(before)) < 1e-13
