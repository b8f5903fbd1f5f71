"""The pure-tensor step transcription (the adjoint's checker) against the oracle (CPU)."""
import numpy as np
import pytest
import torch

import oracle as O
from gemini_b200 import grid as G
from gemini_b200 import state as S
from gemini_b200 import torchstep as TS

from helpers import LSP


def to_t(a):
    """Fortran (X1, X2, X3, S) block -> tensor (S, X3, X2, X1)."""
    return torch.from_numpy(np.ascontiguousarray(np.asarray(a).transpose(3, 2, 1, 0)))


def from_t(t):
    return np.asfortranarray(t.detach().numpy().transpose(3, 2, 1, 0))


def run_torch(g, st, dts, diffsolvetype=2):
    TG = TS.tgrid(g)
    fv = to_t(st.fluidvars)
    ns, vs1, vs2, vs3, Ts = (fv[i * LSP:(i + 1) * LSP] for i in range(5))
    lo = torch.from_numpy(np.ascontiguousarray(st.vs1i[0].transpose(2, 1, 0)))
    hi = torch.from_numpy(np.ascontiguousarray(st.vs1i[-1].transpose(2, 1, 0)))
    nn = torch.from_numpy(np.ascontiguousarray(st.nn.transpose(3, 2, 1, 0)))
    Tn = torch.from_numpy(np.ascontiguousarray(st.Tn.transpose(2, 1, 0)))
    J1 = torch.from_numpy(np.ascontiguousarray(st.electrovars[..., 3].transpose(2, 1, 0)))
    for dt in dts:
        ns, vs1, Ts, lo, hi = TS.step(TG, ns, vs1, vs2, vs3, Ts, lo, hi, nn, Tn, J1, dt, st.Teinf,
                                      diffsolvetype=diffsolvetype)
    return ns, vs1, Ts


CASES = [
    ("cart", lambda: G.cartesian_grid(20, 6, 5), dict(seed=1)),
    ("cart_inverted", lambda: G.cartesian_grid(18, 5, 4, inverted=True), dict(seed=2)),
    ("cart_periodic", lambda: G.cartesian_grid(16, 4, 6, flagper=1), dict(seed=3)),
    ("dipole", lambda: G.dipole_grid(40, 6, 5), dict(seed=5, perturb=0.2)),
    ("cart_J1", lambda: G.cartesian_grid(20, 5, 4), dict(seed=7, J1_amp=1e-5)),
]


@pytest.mark.parametrize("name,mk,kw", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("solver", [2, 1])
def test_torch_step_matches_oracle(name, mk, kw, solver):
    g = mk()
    st = S.init_state(g, **kw)
    ref = st.copy()
    O.set_exact_dependencies(True)
    dts = []
    for _ in range(2):
        dt, _ = O.dt_calc(g, ref, 0.5)
        O.fluid_adv(g, ref, dt, diffsolvetype=solver)
        dts.append(dt)
    ns, vs1, Ts = run_torch(g, st, dts, diffsolvetype=solver)
    I = (slice(2, g.lx1 + 2), slice(2, g.lx2 + 2), slice(2, g.lx3 + 2))
    for got, exp, signed in ((from_t(ns), ref.fluidvars[..., 0:7], False),
                             (from_t(vs1), ref.fluidvars[..., 7:14], True),
                             (from_t(Ts), ref.fluidvars[..., 28:35], False)):
        a, b = got[I], exp[I]
        if signed:
            err = np.max(np.abs(a - b)) / np.max(np.abs(b))
        else:
            err = np.max(np.abs(a - b) / np.abs(b))
        assert err < 1e-10, (name, err)


def test_branch_record_compares_branch_decisions():
    """The branch record of the transcription: the same inputs give the same digest list, a
    change that flips one minmod decision gives a different one, and recording changes no
    value."""
    import torch

    from gemini_b200 import torchstep as TS

    a = torch.tensor([1.0, -2.0, 3.0, 0.5], dtype=torch.float64)
    b = torch.tensor([2.0, 1.0, -1.0, 0.25], dtype=torch.float64)
    TS.BRANCHES = []
    try:
        r1 = TS.minmod(a, b)
        d1 = list(TS.BRANCHES)
        TS.BRANCHES.clear()
        r2 = TS.minmod(a.clone(), b.clone())
        d2 = list(TS.BRANCHES)
        TS.BRANCHES.clear()
        a2 = a.clone()
        a2[3] = 0.2  # |a| < |b| now at element 3
        TS.minmod(a2, b)
        d3 = list(TS.BRANCHES)
    finally:
        TS.BRANCHES = None
    assert d1 == d2 and d1 != d3 and len(d1) == 2
    assert torch.equal(r1, r2) and torch.equal(r1, TS.minmod(a, b))
