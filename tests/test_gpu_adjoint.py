"""The differentiable fluid advance: CUDA forward with checkpoint recomputation and the step
VJP, against autograd through the pure-tensor transcription and central finite differences
(h = 1e-6 relative) on 32 random directions."""
import numpy as np
import pytest

from gemini_b200 import adjoint as AD
from gemini_b200 import grid as G
from gemini_b200 import state as S

pytestmark = pytest.mark.gpu


def _problem(nsteps=6, k=2, lx=(32, 6, 5), seed=4, solver=2):
    import torch

    g = G.cartesian_grid(*lx)
    st = S.init_state(g, seed=seed, perturb=0.1)
    P = AD.DiffProblem(g, st, nsteps, checkpoint_every=k, diffsolvetype=solver)
    I = (slice(2, g.lx3 + 2), slice(2, g.lx2 + 2), slice(2, g.lx1 + 2))
    n0 = P.base[(slice(0, 6),) + I].clone()
    rng = np.random.default_rng(seed)
    Ttop = torch.from_numpy(st.Teinf * (1 + 0.05 * rng.uniform(-1, 1, (g.lx3, g.lx2)))).cuda()
    tgt_T = torch.from_numpy(rng.uniform(1500, 3000, (g.lx3, g.lx2, g.lx1))).cuda()
    tgt_n = torch.from_numpy(rng.uniform(0.5e10, 5e10, (g.lx3, g.lx2, g.lx1))).cuda()
    return g, P, n0, Ttop, tgt_T, tgt_n


def _loss_cuda(P, g, n0, Ttop, tT, tn):
    (ns, vs1, Ts, _, _), _ = P.run(n0, Ttop)
    return float(AD.misfit(ns, Ts, tT, tn, g))


def test_cuda_forward_matches_transcription_with_top_temperature():
    import torch

    g, P, n0, Ttop, tT, tn = _problem()
    (ns, vs1, Ts, _, _), _ = P.run(n0, Ttop)
    ref_loss = AD.torch_reference_loss(P, n0, Ttop, tT, tn)
    cuda_loss = AD.misfit(ns, Ts, tT, tn, g)
    assert float(cuda_loss) == pytest.approx(float(ref_loss), rel=1e-10)
    # the top temperature reaches the solution
    (ns2, _, Ts2, _, _), _ = P.run(n0, Ttop * 1.01)
    assert not torch.equal(Ts2, Ts)


@pytest.mark.parametrize("solver", [2, 1])
def test_gradient_matches_autograd_of_transcription(solver):
    import torch

    g, P, n0, Ttop, tT, tn = _problem(solver=solver)
    a = n0.clone().requires_grad_(True)
    t = Ttop.clone().requires_grad_(True)
    ns, Ts = AD.FluidAdvance.apply(a, t, P)
    AD.misfit(ns, Ts, tT, tn, g).backward()
    b = n0.clone().requires_grad_(True)
    u = Ttop.clone().requires_grad_(True)
    AD.torch_reference_loss(P, b, u, tT, tn).backward()
    for x, y in ((a.grad, b.grad), (t.grad, u.grad)):
        err = float((x - y).abs().max() / y.abs().max())
        assert err < 1e-8, err
    assert float(t.grad.abs().max()) > 0


def test_gradient_independent_of_checkpoint_interval():
    """Every state kept (one pipelined backward segment), and recomputation every 2 or 4
    steps (the recompute of a segment overlapping the previous segment's backward), give the
    same gradients."""
    import torch

    grads = []
    for k in (1, 2, 4):
        g, P, n0, Ttop, tT, tn = _problem(nsteps=7, k=k)
        a = n0.clone().requires_grad_(True)
        t = Ttop.clone().requires_grad_(True)
        ns, Ts = AD.FluidAdvance.apply(a, t, P)
        AD.misfit(ns, Ts, tT, tn, g).backward()
        grads.append((a.grad, t.grad))
        P.close()
    for other in grads[1:]:
        for x, y in zip(grads[0], other):
            assert float((x - y).abs().max() / x.abs().max()) < 1e-12


def test_gradient_vs_central_differences_32_directions():
    import torch

    g, P, n0, Ttop, tT, tn = _problem(nsteps=5, k=2)
    a = n0.clone().requires_grad_(True)
    t = Ttop.clone().requires_grad_(True)
    ns, Ts = AD.FluidAdvance.apply(a, t, P)
    AD.misfit(ns, Ts, tT, tn, g).backward()
    rng = np.random.default_rng(123)
    h = 1e-6
    errs = []
    for _ in range(32):
        dn = torch.from_numpy(rng.standard_normal(n0.shape)).cuda()
        dT = torch.from_numpy(rng.standard_normal(Ttop.shape)).cuda()
        lp = _loss_cuda(P, g, n0 * (1 + h * dn), Ttop * (1 + h * dT), tT, tn)
        lm = _loss_cuda(P, g, n0 * (1 - h * dn), Ttop * (1 - h * dT), tT, tn)
        fd = (lp - lm) / (2 * h)
        an = float((a.grad * n0 * dn).sum() + (t.grad * Ttop * dT).sum())
        errs.append(abs(fd - an) / max(abs(an), 1e-30))
    errs = np.array(errs)
    # the step is piecewise smooth (limiter branches, floors): a perturbation of 1e-6 may
    # cross a branch in a rare direction; the bulk must agree to FD accuracy
    assert np.median(errs) < 1e-5, errs
    assert np.mean(errs < 1e-3) >= 0.9, errs


DIFF_CASES = [
    ("cart_top", lambda: G.cartesian_grid(24, 4, 3), dict(seed=2, perturb=0.1)),
    ("cart_inverted", lambda: G.cartesian_grid(20, 3, 4, inverted=True), dict(seed=3, perturb=0.1)),
    ("dipole", lambda: G.dipole_grid(36, 4, 3), dict(seed=5, perturb=0.2)),
    ("cart_J1", lambda: G.cartesian_grid(22, 3, 3), dict(seed=7, J1_amp=1e-5)),
    # several rows per lane in the warp solver (lx1 = 150: 5 per lane, the last lane partial)
    ("cart_long", lambda: G.cartesian_grid(150, 5, 4), dict(seed=11, perturb=0.1, J1_amp=1e-5)),
    ("dipole_long", lambda: G.dipole_grid(100, 4, 3), dict(seed=13, perturb=0.2)),
]


@pytest.mark.parametrize("name,mk,kw", DIFF_CASES, ids=[c[0] for c in DIFF_CASES])
@pytest.mark.parametrize("solver", [2, 1])
def test_cuda_diffusion_adjoint_matches_autograd(name, mk, kw, solver):
    """The hand-written CUDA VJP of the energy diffusion against autograd through the
    pure-tensor transcription, on random output cotangents."""
    import torch

    from gemini_b200 import torchstep as TS

    g = mk()
    st = S.init_state(g, **kw)
    P = AD.DiffProblem(g, st, 1, diffsolvetype=solver)
    n = P.base[0:7].clone()
    T = P.base[28:35].clone()
    rng = np.random.default_rng(1)
    Ttop = torch.from_numpy(st.Teinf * (1 + 0.05 * rng.uniform(-1, 1, (g.lx3, g.lx2)))).cuda()
    Yb = torch.from_numpy(rng.standard_normal(T.shape)).cuda()
    nb, Tb, tb = P.diffusion_vjp(n, T, Ttop, P.dt_tensor(0), Yb)
    n_ = n.clone().requires_grad_(True)
    T_ = T.clone().requires_grad_(True)
    t_ = Ttop.clone().requires_grad_(True)
    out = TS.energy_diffusion(P.tg, n_, T_, P.J1, P.nn, P.Tn, P.dts[0], P.Teinf, t_, solver)
    (out * Yb).sum().backward()
    I = (slice(None), slice(2, g.lx3 + 2), slice(2, g.lx2 + 2), slice(2, g.lx1 + 2))
    if t_.grad is None:  # closed dipole: no exospheric boundary
        assert float(tb.abs().max()) == 0.0
        t_.grad = torch.zeros_like(tb)
    for got, exp in ((Tb, T_.grad), (nb[I], n_.grad[I]), (tb, t_.grad)):
        scale = float(exp.abs().max())
        err = float((got - exp).abs().max()) / max(scale, 1e-300) if scale > 0 else float(got.abs().max())
        assert err < 1e-9, (name, err)


SWEEP_CASES = [
    ("cart", lambda: G.cartesian_grid(20, 6, 5), dict(seed=1)),
    ("dipole", lambda: G.dipole_grid(24, 6, 5), dict(seed=5, perturb=0.2)),
    # several line segments and 32-line panels per direction
    ("cart_big", lambda: G.cartesian_grid(70, 40, 35), dict(seed=3)),
    ("dipole_big", lambda: G.dipole_grid(64, 34, 33), dict(seed=6, perturb=0.2)),
]


@pytest.mark.parametrize("name,mk,kw", SWEEP_CASES, ids=[c[0] for c in SWEEP_CASES])
@pytest.mark.parametrize("dim,frank,nsp", [(1, 0, 6), (1, 0, 7), (2, 0, 6), (2, 1, 6), (3, 0, 7), (3, 1, 6)])
def test_cuda_sweep_adjoint_matches_autograd(name, mk, kw, dim, frank, nsp):
    """CUDA field sweep and its hand-written VJP (replayed limiter/upwind branches) against
    autograd through the pure-tensor sweep, with random face velocities of both signs."""
    import torch

    from gemini_b200 import torchstep as TS

    g = mk()
    st = S.init_state(g, **kw)
    P = AD.DiffProblem(g, st, 1)
    rng = np.random.default_rng(dim * 10 + frank)
    f = P.base[0:7].clone() * torch.from_numpy(1 + 0.3 * rng.standard_normal(P.base[0:7].shape)).cuda()
    vshape = {1: (7, g.lx3, g.lx2, g.lx1 + 1), 2: (7, g.lx3, g.lx2 + 1, g.lx1), 3: (7, g.lx3 + 1, g.lx2, g.lx1)}[dim]
    v = torch.from_numpy(rng.uniform(-400, 400, vshape)).cuda()
    ob = torch.from_numpy(rng.standard_normal(f.shape)).cuda()
    SF = AD._sweep_fn()
    f1 = f.clone().requires_grad_(True)
    v1 = v.clone().requires_grad_(True)
    out1 = SF.apply(f1, v1, P, dim, frank, nsp, P.dt_tensor(0))
    (out1 * ob).sum().backward()
    f2 = f.clone().requires_grad_(True)
    v2 = v.clone().requires_grad_(True)
    out2 = TS.sweep_field(P.tg, f2, v2, dim, frank, nsp, P.dts[0])
    (out2 * ob).sum().backward()
    assert float((out1 - out2).detach().abs().max() / out2.detach().abs().max()) < 1e-13
    for got, exp in ((f1.grad, f2.grad), (v1.grad, v2.grad)):
        err = float((got - exp).abs().max() / exp.abs().max())
        assert err < 1e-10, (name, dim, frank, err)


def test_batched_adjoint_matches_per_instance_gradients():
    """Uneven instances, batched forward with prescribed time steps (one graph per step),
    per-instance backward: same final states and gradients as each instance on its own."""
    import torch

    specs = [(24, 5, 4, 1), (32, 4, 6, 2), (20, 6, 3, 3)]
    inst = []
    for lx1, lx2, lx3, seed in specs:
        g = G.cartesian_grid(lx1, lx2, lx3)
        inst.append((g, S.init_state(g, seed=seed, perturb=0.1)))
    BA = AD.BatchedAdjoint(inst, 5, checkpoint_every=2, group=2)
    rng = np.random.default_rng(9)
    controls, targets = [], []
    for (g, st), P in zip(inst, BA.problems):
        I = (slice(2, g.lx3 + 2), slice(2, g.lx2 + 2), slice(2, g.lx1 + 2))
        n0 = P.base[(slice(0, 6),) + I].clone()
        Ttop = torch.from_numpy(st.Teinf * (1 + 0.05 * rng.uniform(-1, 1, (g.lx3, g.lx2)))).cuda()
        controls.append((n0, Ttop))
        targets.append((torch.from_numpy(rng.uniform(1500, 3000, (g.lx3, g.lx2, g.lx1))).cuda(),
                        torch.from_numpy(rng.uniform(0.5e10, 5e10, (g.lx3, g.lx2, g.lx1))).cuda()))

    def loss(i, ns, Ts):
        return AD.misfit(ns, Ts, targets[i][0], targets[i][1], inst[i][0])

    res = BA.gradients(controls, loss)
    for i, ((g, st), P) in enumerate(zip(inst, BA.problems)):
        # the batched forward equals the instance's own CUDA forward, bit for bit
        (ns, _, Ts, _, _), _ = P.run(*controls[i])
        fin, _ = BA.forward_group([i], [controls[i]], keep=False)
        assert torch.equal(fin[0][0], ns) and torch.equal(fin[0][2], Ts)
        a = controls[i][0].clone().requires_grad_(True)
        t = controls[i][1].clone().requires_grad_(True)
        nsa, Tsa = AD.FluidAdvance.apply(a, t, P)
        L = loss(i, nsa, Tsa)
        L.backward()
        Lb, gn, gt = res[i]
        assert Lb == pytest.approx(float(L.detach()), rel=1e-12)
        for x, y in ((gn, a.grad), (gt, t.grad)):
            assert float((x - y).abs().max() / y.abs().max()) < 1e-10


def test_graphed_step_vjp_equals_eager():
    """The step VJP replayed from its captured CUDA graph gives the eager result."""
    import torch

    g, P, n0, Ttop, tT, tn = _problem(nsteps=4, k=2)
    P.cuda_step_adjoint = False  # the autograd step VJP (CUDA sweep and diffusion VJPs inside)
    grads = []
    for graphed in (False, True):
        P.vjp_graph = graphed
        P._graphs = {}
        a = n0.clone().requires_grad_(True)
        t = Ttop.clone().requires_grad_(True)
        ns, Ts = AD.FluidAdvance.apply(a, t, P)
        AD.misfit(ns, Ts, tT, tn, g).backward()
        grads.append((a.grad, t.grad))
    assert P.vjp_graph, f"graph capture fell back to eager: {getattr(P, 'vjp_graph_error', '')}"
    for x, y in zip(grads[0], grads[1]):
        assert float((x - y).abs().max() / x.abs().max()) < 1e-12


# (name, grid, state kwargs, floor-free): the dipole state after one step has temperatures
# floored at 100 K, where the diffusion solution sits on the kink of max(T, 100) to within
# round-off -- there any subgradient is valid and two implementations may pick differently,
# so the dipole is compared with autograd running the same CUDA sweep and diffusion VJP
# kernels (the same branch decisions), not with the pure transcription.
STEP_CASES = [
    ("cart", lambda: G.cartesian_grid(24, 6, 5), dict(seed=1, perturb=0.1), True),
    ("cart_inverted", lambda: G.cartesian_grid(20, 5, 4, inverted=True), dict(seed=2, perturb=0.1), True),
    ("dipole", lambda: G.dipole_grid(28, 6, 5), dict(seed=5, perturb=0.2), False),
    ("cart_periodic", lambda: G.cartesian_grid(22, 5, 6, flagper=1), dict(seed=3, perturb=0.1, J1_amp=1e-5), True),
    ("cart_big", lambda: G.cartesian_grid(40, 36, 34), dict(seed=4, perturb=0.1), True),
]


@pytest.mark.parametrize("name,mk,kw,floor_free", STEP_CASES, ids=[c[0] for c in STEP_CASES])
@pytest.mark.parametrize("solver,top", [(2, True), (1, True), (2, False)])
def test_cuda_step_vjp_matches_autograd(name, mk, kw, floor_free, solver, top):
    """The fused CUDA step VJP (gem_step_vjp_dev) against autograd through the tensor step,
    on random interior output cotangents and random boundary-face cotangents: with the
    CUDA sweep and diffusion VJPs inside autograd (every grid) and through the pure
    transcription (grids whose step stays clear of the temperature floor)."""
    import torch

    g = mk()
    st = S.init_state(g, **kw)
    P = AD.DiffProblem(g, st, 2, checkpoint_every=1, diffsolvetype=solver)
    rng = np.random.default_rng(7)
    I = (slice(2, g.lx3 + 2), slice(2, g.lx2 + 2), slice(2, g.lx1 + 2))
    n0 = P.base[(slice(0, 6),) + I].clone()
    Ttop = torch.from_numpy(st.Teinf * (1 + 0.05 * rng.uniform(-1, 1, (g.lx3, g.lx2)))).cuda() if top else None
    _, ck = P.run(n0, Ttop, keep=True)
    state = ck[1]  # the state after one step
    cot = []
    for t in state[:3]:
        c = torch.zeros_like(t)
        c[(slice(None),) + I] = torch.from_numpy(rng.standard_normal(c[(slice(None),) + I].shape)).cuda()
        cot.append(c)
    cot += [torch.from_numpy(rng.standard_normal(t.shape)).cuda() for t in state[3:]]
    got, gtop = P.step_vjp_cuda(state, Ttop, 1, cot)
    refs = [True] + ([False] if floor_free else [])
    for cuda_pieces in refs:
        P.cuda_sweep_adjoint = cuda_pieces
        inp = [t.detach().clone().requires_grad_(True) for t in state]
        tt = None if Ttop is None else Ttop.clone().requires_grad_(True)
        exp, etop = P._vjp_body(inp, tt, P.dt_tensor(1), cot, use_cuda_diffusion_adjoint=cuda_pieces)
        for nm, x, y in zip(("ns", "vs1", "Ts", "lo", "hi"), got, exp):
            scale = float(y.abs().max())
            err = float((x - y).abs().max()) / scale if scale > 0 else float(x.abs().max())
            assert err < 1e-9, (name, cuda_pieces, nm, err)
        if Ttop is not None:
            if g.gridflag == 0:  # closed dipole: no exospheric boundary
                assert float(gtop.abs().max()) == 0.0
            else:
                err = float((gtop - etop).abs().max() / etop.abs().max())
                assert err < 1e-9, (name, cuda_pieces, "Ttop", err)


def test_combined_step_vjp_entry_equals_its_halves():
    """gem_step_vjp_dev (one call) gives the bits of gem_step_vjp_replay_dev followed by
    gem_step_vjp_backward_dev (what the Python backward calls)."""
    import ctypes

    import torch

    from gemini_b200 import _lib
    from gemini_b200 import fluid as F

    g = G.cartesian_grid(30, 7, 6, flagper=1)
    st = S.init_state(g, seed=8, perturb=0.1)
    P = AD.DiffProblem(g, st, 2, checkpoint_every=1)
    rng = np.random.default_rng(3)
    I = (slice(2, g.lx3 + 2), slice(2, g.lx2 + 2), slice(2, g.lx1 + 2))
    Ttop = torch.from_numpy(st.Teinf * (1 + 0.05 * rng.uniform(-1, 1, (g.lx3, g.lx2)))).cuda()
    _, ck = P.run(P.base[(slice(0, 6),) + I].clone(), Ttop, keep=True)
    state = ck[1]
    cot = [torch.from_numpy(rng.standard_normal(t.shape)).cuda() for t in state]
    halves, top_h = P.step_vjp_cuda(state, Ttop, 1, cot)
    out = [torch.empty_like(t) for t in state]
    tb = torch.empty_like(Ttop)
    c = P.cfg.c()
    p = F._ptr
    ns, vs1, Ts, lo, hi = state
    _lib.check(_lib.lib().gem_step_vjp_dev(
        ctypes.byref(c), P.dg.handle, P.ds.work, P._workspace(1), p(ns), p(vs1), p(P.vs2), p(P.vs3), p(Ts), p(lo),
        p(hi), p(P.ds.electrovars), p(P.dt_tensor(1)), *[p(t) for t in cot], *[p(t) for t in out], p(tb),
        F._stream()))
    torch.cuda.synchronize()
    for x, y in zip(out, halves):
        assert torch.equal(x, y)
    assert torch.equal(tb, top_h)
    P.close()


@pytest.mark.parametrize("name,mk,kw,floor_free", STEP_CASES, ids=[c[0] for c in STEP_CASES])
@pytest.mark.parametrize("solver", [2, 1])
def test_replay_finish_gives_the_forward_step(name, mk, kw, floor_free, solver):
    """gem_step_vjp_replay_dev + gem_step_vjp_finish_dev from the state before a step give
    the forward step's next state (ns, vs1, Ts with their ghost cells, the boundary faces)
    bit for bit, so a backward that recomputes by replay + finish sees the forward's states."""
    import torch

    g = mk()
    st = S.init_state(g, **kw)
    P = AD.DiffProblem(g, st, 3, checkpoint_every=1, diffsolvetype=solver)
    rng = np.random.default_rng(5)
    I = (slice(2, g.lx3 + 2), slice(2, g.lx2 + 2), slice(2, g.lx1 + 2))
    Ttop = torch.from_numpy(st.Teinf * (1 + 0.05 * rng.uniform(-1, 1, (g.lx3, g.lx2)))).cuda()
    fin, ck = P.run(P.base[(slice(0, 6),) + I].clone(), Ttop, keep=True)
    P._set_top(Ttop)
    for j in range(3):
        P._replay(0, ck[j], j)
        got = P._finish(0, j)
        want = ck[j + 1] if j + 1 < 3 else fin
        for name_, x, y in zip(("ns", "vs1", "Ts", "lo", "hi"), got, want):
            assert torch.equal(x, y), (j, name_, float((x - y).abs().max()))
    P.close()


def test_slot_backward_equals_two_workspace_backward():
    """The backward that recomputes by replay + finish into k+1 slots and the one that
    recomputes with the plain forward step into two alternating workspaces give the same
    gradients bit for bit (checkpoints every 3 steps over 8 steps: uneven segments)."""
    import torch

    grads = []
    for slots in (True, False):
        g, P, n0, Ttop, tT, tn = _problem(nsteps=8, k=3)
        P.replay_slots = slots
        a = n0.clone().requires_grad_(True)
        t = Ttop.clone().requires_grad_(True)
        ns, Ts = AD.FluidAdvance.apply(a, t, P)
        AD.misfit(ns, Ts, tT, tn, g).backward()
        grads.append((a.grad, t.grad))
        nws = len(P._sa)
        P.close()
        assert nws == (4 if slots else 2)
    for x, y in zip(*grads):
        assert torch.equal(x, y)
