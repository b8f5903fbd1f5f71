"""Differentiable fluid advance: gradients of a loss of the final state with respect to the
initial ion densities and the per-column top (exospheric) temperature.

``FluidAdvance.apply(n0, Ttop, problem)`` runs ``problem.nsteps`` steps of the CUDA step
(``gem_fluid_adv_dev``) on a frozen time-step schedule (dt_calc is not differentiated; the
schedule comes from one plain run of the unperturbed problem), saving the state every
``problem.checkpoint_every`` steps.  The backward pass recomputes each segment from its
checkpoint with the CUDA step and pulls the cotangent back one step at a time with the
step's vector-Jacobian product; the VJP of a step is ``torchstep.step`` differentiated by
torch.autograd (its energy diffusion optionally replaced by the hand-written CUDA adjoint).

State carried between steps: ns, vs1, Ts (interior; the step rebuilds every ghost cell) and
the two x1 boundary faces of vs1i (read, one step stale, by set_global_boundaries); vs2,
vs3, nn, Tn, J1 are inputs of the problem.  Grids without null cells.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from . import fluid as F
from . import torchstep as TS
from .state import LSP


class _CudaArray:
    """__cuda_array_interface__ view of a raw device pointer (float64)."""

    def __init__(self, ptr: int, shape):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": "<f8", "data": (int(ptr), False),
                                         "version": 3, "strides": None}


class DiffProblem:
    """One differentiable problem: grid, fixed inputs, dt schedule, scratch device state."""

    def __init__(self, grid, st, nsteps: int, checkpoint_every: int = 5, tcfl: float = 0.5,
                 diffsolvetype: int = 2, device="cuda", cuda_diffusion_adjoint: bool = True,
                 cuda_sweep_adjoint: bool = True, cuda_step_adjoint: bool = True):
        import torch

        self.cuda_diffusion_adjoint = bool(cuda_diffusion_adjoint)
        self.cuda_sweep_adjoint = bool(cuda_sweep_adjoint)
        self.cuda_step_adjoint = bool(cuda_step_adjoint)
        self._sa = None  # gem_step_adjoint workspaces (the backward's replay slots), made on first use
        self._side = None  # the replay stream of the pipelined backward
        self.replay_slots = True  # recompute by replay + finish when k+1 workspaces fit
        self._dtt = {}
        self._capturing = False
        self._graphs = {}  # (Ttop given) -> captured step VJP
        self.vjp_graph = True
        self.grid = grid
        self.nsteps = int(nsteps)
        self.k = max(1, int(checkpoint_every))
        self.diffsolvetype = diffsolvetype
        self.tg = TS.tgrid(grid, device)
        self.dg = F.DeviceGrid(grid)
        self.ds = F.DeviceState.from_host(self.dg, st.copy())
        self.cfg = F.FluidCfg(st.Teinf, diffsolvetype=diffsolvetype, tcfl=tcfl)
        X1, X2, X3 = grid.lx1 + 4, grid.lx2 + 4, grid.lx3 + 4
        self.shape = (5 * LSP, X3, X2, X1)
        self.base = self.ds.fluidvars.view(self.shape).clone()
        self.vs2 = self.base[2 * LSP:3 * LSP]
        self.vs3 = self.base[3 * LSP:4 * LSP]
        self.nn = torch.from_numpy(np.ascontiguousarray(st.nn.transpose(3, 2, 1, 0))).to(device)
        self.Tn = torch.from_numpy(np.ascontiguousarray(st.Tn.transpose(2, 1, 0))).to(device)
        self.J1 = torch.from_numpy(np.ascontiguousarray(st.electrovars[..., 3].transpose(2, 1, 0))).to(device)
        self.Teinf = float(st.Teinf)
        self.v1i = torch.as_tensor(_CudaArray(_lib.lib().gem_work_array(self.ds.work, 1),
                                              (LSP, grid.lx3, grid.lx2, grid.lx1 + 1)), device=device)
        self.lo0 = self.v1i[..., 0].clone()
        self.hi0 = self.v1i[..., -1].clone()
        # the frozen schedule: dt_calc of a plain run from the base state
        self.dts = []
        self._load(self.base[0:LSP], self.base[LSP:2 * LSP], self.base[4 * LSP:], self.lo0, self.hi0, None)
        for _ in range(self.nsteps):
            dt = F.dt_calc(self.ds, tcfl)
            self.dts.append(float(dt.item()))
            F.fluid_adv(self.cfg, self.ds, dt)

    # -- CUDA state plumbing -------------------------------------------------------------
    def _load(self, ns, vs1, Ts, lo, hi, Ttop):
        fv = self.ds.fluidvars.view(self.shape)
        fv.copy_(self.base)
        fv[0:LSP] = ns
        fv[LSP:2 * LSP] = vs1
        fv[4 * LSP:] = Ts
        self.v1i[..., 0] = lo
        self.v1i[..., -1] = hi
        if Ttop is None:
            _lib.check(_lib.lib().gem_work_set_top_temperature(self.ds.work, None, 0))
        else:
            t = Ttop.detach().contiguous()
            _lib.check(_lib.lib().gem_work_set_top_temperature(self.ds.work, ctypes.c_void_p(t.data_ptr()), 1))

    def _save(self):
        fv = self.ds.fluidvars.view(self.shape)
        return (fv[0:LSP].clone(), fv[LSP:2 * LSP].clone(), fv[4 * LSP:].clone(),
                self.v1i[..., 0].clone(), self.v1i[..., -1].clone())

    def dt_tensor(self, j: int):
        """The step's dt as a cached 1-element device tensor."""
        import torch

        t = self._dtt.get(j)
        if t is None:
            t = torch.full((1,), self.dts[j], dtype=torch.float64, device=self.base.device)
            self._dtt[j] = t
        return t

    def cuda_step(self, j: int) -> None:
        import torch

        dt = torch.full((1,), self.dts[j], dtype=torch.float64, device=self.ds.fluidvars.device)
        F.fluid_adv(self.cfg, self.ds, dt)

    def initial_state(self, n0, Ttop=None):
        """Full-layout initial state with the ion densities n0 (6, lx3, lx2, lx1) in the
        interior; the electrons are their sum (as in the state generator)."""
        import torch

        g = self.grid
        ns = self.base[0:LSP].clone()
        I = (slice(2, g.lx3 + 2), slice(2, g.lx2 + 2), slice(2, g.lx1 + 2))
        ions = n0
        e = ions[0]
        for s in range(1, LSP - 1):
            e = e + ions[s]
        inner = torch.cat([ions, e.unsqueeze(0)], 0)
        ns = ns.clone()
        ns[(slice(None),) + I] = inner
        return ns

    def run(self, n0, Ttop=None, keep=False):
        """CUDA forward from the controls; returns the final (ns, vs1, Ts) tensors and, with
        keep, the checkpoints {step: state}."""
        ns = self.initial_state(n0.detach())
        st = (ns, self.base[LSP:2 * LSP], self.base[4 * LSP:], self.lo0, self.hi0)
        self._load(*st, Ttop)
        ckpt = {}
        for j in range(self.nsteps):
            if keep and j % self.k == 0:
                ckpt[j] = self._save()
            self.cuda_step(j)
        out = self._save()
        return out, ckpt

    # -- the energy diffusion with its hand-written CUDA adjoint ----------------------
    def diffusion_forward(self, n, T, Ttop, dt):
        """gem_energy_diffusion_dev on (n, T): the diffusion output (max(T,100) applied);
        dt is a 1-element device tensor."""
        import torch

        fv = torch.zeros(self.shape, dtype=torch.float64, device=n.device)
        fv[0:LSP] = n
        fv[4 * LSP:] = T
        self._set_top(Ttop)
        c = self.cfg.c()
        _lib.check(_lib.lib().gem_energy_diffusion_dev(ctypes.byref(c), self.dg.handle, F._ptr(fv),
                                                       F._ptr(self.ds.electrovars), self.ds.work, F._ptr(dt),
                                                       F._stream()))
        return fv[4 * LSP:].clone()

    def diffusion_vjp(self, n, T, Ttop, dt, Ybar):
        import torch

        g = self.grid
        self._set_top(Ttop)
        n = n.contiguous()
        T = T.contiguous()
        Yb = Ybar.contiguous()
        Tb = torch.zeros_like(T)
        nb = torch.zeros_like(n)
        tb = torch.zeros((LSP, g.lx3, g.lx2), dtype=torch.float64, device=n.device)
        c = self.cfg.c()
        _lib.check(_lib.lib().gem_diffusion_vjp_dev(ctypes.byref(c), self.dg.handle, F._ptr(T), F._ptr(n),
                                                    F._ptr(self.ds.electrovars), self.ds.work, F._ptr(dt),
                                                    F._ptr(Yb), F._ptr(Tb), F._ptr(nb), F._ptr(tb),
                                                    F._stream()))
        # ghost cells: out = max(T, 100) except the x1 boundary layers, which hold the
        # Dirichlet values max(tmin, 100) / max(tmax, 100)
        ghost = torch.ones_like(T[0], dtype=torch.bool)
        ghost[2:g.lx3 + 2, 2:g.lx2 + 2, 2:g.lx1 + 2] = False
        bc = torch.zeros_like(ghost)
        bc[2:g.lx3 + 2, 2:g.lx2 + 2, 1] = True
        bc[2:g.lx3 + 2, 2:g.lx2 + 2, g.lx1 + 2] = True
        pas = ghost & ~bc
        Tb = Tb + torch.where(pas & (T >= 100.0), Yb, torch.zeros_like(Yb))
        # the boundary layer on the exospheric side carries max(Ttop, 100)
        side = {1: 1, 2: g.lx1 + 2}.get(g.gridflag)
        if side is not None and Ttop is not None:
            bcv = Ttop.unsqueeze(0).expand(LSP, g.lx3, g.lx2)
            tb = tb + torch.where(bcv >= 100.0, Yb[:, 2:g.lx3 + 2, 2:g.lx2 + 2, side], torch.zeros_like(bcv))
        return nb, Tb, tb.sum(0)

    def _set_top(self, Ttop):
        if self._capturing:  # set before the capture / replay (a synchronous copy)
            return
        if Ttop is None:
            _lib.check(_lib.lib().gem_work_set_top_temperature(self.ds.work, None, 0))
        else:
            t = Ttop.detach().contiguous()
            _lib.check(_lib.lib().gem_work_set_top_temperature(self.ds.work, ctypes.c_void_p(t.data_ptr()), 1))

    def step_vjp(self, state, Ttop, j, cot, use_cuda_diffusion_adjoint=False):
        """Pull the cotangent of the state after step j back to the state before it (and
        to Ttop).  state / cot: (ns, vs1, Ts, lo, hi).  With cuda_step_adjoint the whole
        step's VJP runs in CUDA (gem_step_vjp_dev); otherwise autograd through the tensor
        transcription, its sweeps and diffusion optionally replaced by their CUDA VJPs."""
        import torch

        if self.cuda_step_adjoint:
            return self.step_vjp_cuda(state, Ttop, j, cot)
        inp = [t.detach().requires_grad_(True) for t in state]
        tt = None if Ttop is None else Ttop.detach().requires_grad_(True)
        if (self.vjp_graph and use_cuda_diffusion_adjoint and self.cuda_sweep_adjoint
                and all(c is not None for c in cot)):
            try:
                return self._step_vjp_graphed(state, Ttop, j, cot)
            except RuntimeError as e:  # capture unavailable: stay eager
                self.vjp_graph = False
                self.vjp_graph_error = str(e)
                self._capturing = False
        return self._vjp_body(inp, tt, self.dt_tensor(j), cot, use_cuda_diffusion_adjoint)

    def step_vjp_cuda(self, state, Ttop, j, cot):
        """The step VJP in CUDA (the replay and backward halves of gem_step_vjp_dev): forward
        replay and every adjoint piece on the device.  Cotangents at ghost cells of the step's
        outputs are ignored (the next step never reads them); the state's ghost cells get
        zero."""
        state = tuple(t.detach().contiguous() for t in state)
        self._set_top(Ttop)
        self._replay(0, state, j)
        return self._backward(0, state, Ttop, j, cot)

    def _drop_workspaces(self, keep: int = 0):
        """Destroy the step adjoint workspaces beyond the first `keep`."""
        for i in range(keep, len(self._sa or [])):
            if self._sa[i] is not None:
                _lib.lib().gem_step_adjoint_destroy(self._sa[i])
                self._sa[i] = None

    def _workspace(self, i):
        if self._sa is None:
            self._sa = []
        while len(self._sa) <= i:
            self._sa.append(None)
        if self._sa[i] is None:
            h = ctypes.c_void_p()
            _lib.check(_lib.lib().gem_step_adjoint_create(self.dg.handle, ctypes.byref(h)))
            self._sa[i] = h
        return self._sa[i]

    def _replay(self, i, state, j):
        """gem_step_vjp_replay_dev of step j into workspace i, on the current stream."""
        ns, vs1, Ts, lo, hi = state
        p = F._ptr
        c = self.cfg.c()
        _lib.check(_lib.lib().gem_step_vjp_replay_dev(
            ctypes.byref(c), self.dg.handle, self.ds.work, self._workspace(i), p(ns), p(vs1), p(self.vs2),
            p(self.vs3), p(Ts), p(lo), p(hi), p(self.dt_tensor(j)), F._stream()))

    def _backward(self, i, state, Ttop, j, cot):
        """gem_step_vjp_backward_dev of step j from workspace i (replayed), on the current stream."""
        import torch

        ns, vs1, Ts, lo, hi = state
        z = [torch.zeros_like(t) if c is None else c.detach().contiguous() for c, t in zip(cot, state)]
        out = [torch.empty_like(t) for t in state]
        tb = torch.empty((self.grid.lx3, self.grid.lx2), dtype=torch.float64, device=ns.device) \
            if Ttop is not None else None
        p = F._ptr
        c = self.cfg.c()
        _lib.check(_lib.lib().gem_step_vjp_backward_dev(
            ctypes.byref(c), self.dg.handle, self.ds.work, self._workspace(i), p(ns), p(vs1), p(Ts), p(lo), p(hi),
            p(self.ds.electrovars), p(self.dt_tensor(j)), p(z[0]), p(z[1]), p(z[2]), p(z[3]), p(z[4]),
            p(out[0]), p(out[1]), p(out[2]), p(out[3]), p(out[4]), None if tb is None else p(tb), F._stream()))
        return out, tb

    def _finish(self, i, j):
        """gem_step_vjp_finish_dev of step j from workspace i (replayed), on the current
        stream: the state after step j, as the forward writes it, in new tensors."""
        import torch

        g = self.grid
        lo = torch.empty((LSP, g.lx3, g.lx2), dtype=torch.float64, device=self.base.device)
        hi = torch.empty_like(lo)
        p = F._ptr
        c = self.cfg.c()
        _lib.check(_lib.lib().gem_step_vjp_finish_dev(
            ctypes.byref(c), self.dg.handle, self.ds.work, self._workspace(i), p(self.ds.fluidvars),
            p(self.ds.fluidauxvars), p(self.ds.electrovars), p(self.dt_tensor(j)), p(lo), p(hi), F._stream()))
        fv = self.ds.fluidvars.view(self.shape)
        return (fv[0:LSP].clone(), fv[LSP:2 * LSP].clone(), fv[4 * LSP:].clone(), lo, hi)

    def workspace_bytes(self):
        """Device bytes of one step adjoint workspace (gem_step_adjoint_create)."""
        g = self.grid
        F1 = LSP * (g.lx1 + 4) * (g.lx2 + 4) * (g.lx3 + 4)
        n1 = LSP * (g.lx1 + 1) * g.lx2 * g.lx3
        n2 = LSP * g.lx1 * (g.lx2 + 1) * g.lx3
        n3 = LSP * g.lx1 * g.lx2 * (g.lx3 + 1)
        return 8 * (23 * F1 + 5 * n1 + n2 + n3 + 3 * LSP * g.lx2 * g.lx3)

    def close(self):
        """Release the step adjoint workspaces."""
        if self._sa is not None:
            for h in self._sa:
                if h is not None:
                    _lib.lib().gem_step_adjoint_destroy(h)
            self._sa = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _vjp_body(self, inp, tt, dt, cot, use_cuda_diffusion_adjoint=True):
        """The step VJP on given tensors (inp require grad); dt: 1-element device tensor."""
        import torch

        diff = None
        sweep = None
        P = self
        if use_cuda_diffusion_adjoint:
            def diff(n, T, Ttop_):
                return _diffusion_fn().apply(n, T, Ttop_, P, dt)

        if self.cuda_sweep_adjoint:
            def sweep(f, v, dim, frank, nsp):
                return _sweep_fn().apply(f, v, P, dim, frank, nsp, dt)
        with torch.enable_grad():
            out = TS.step(self.tg, inp[0], inp[1], self.vs2, self.vs3, inp[2], inp[3], inp[4], self.nn,
                          self.Tn, self.J1, dt, self.Teinf, tt, self.diffsolvetype, diffusion=diff,
                          sweep_impl=sweep)
            pairs = [(o, c) for o, c in zip(out, cot) if c is not None]
            wrt = list(inp) + ([tt] if tt is not None else [])
            grads = torch.autograd.grad([o for o, _ in pairs], wrt, [c for _, c in pairs], allow_unused=True)
        g_state = [torch.zeros_like(t) if g is None else g for g, t in zip(grads[:5], inp)]
        g_top = None if tt is None else (torch.zeros_like(tt) if grads[5] is None else grads[5])
        return g_state, g_top

    def _step_vjp_graphed(self, state, Ttop, j, cot):
        """The step VJP replayed from a CUDA graph captured once per problem (static input
        buffers: state, cotangent, dt, top temperature)."""
        import torch

        key = Ttop is not None
        G = self._graphs.get(key)
        if G is None:
            G = {"state": [t.detach().clone() for t in state], "cot": [c.detach().clone() for c in cot],
                 "dt": self.dt_tensor(j).clone(), "top": Ttop.detach().clone() if key else None}
            self._set_top(Ttop)
            side = torch.cuda.Stream()
            side.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(side):
                for _ in range(2):  # warm-up outside the capture
                    inp = [t.detach().requires_grad_(True) for t in G["state"]]
                    tt = G["top"].detach().requires_grad_(True) if key else None
                    self._vjp_body(inp, tt, G["dt"], G["cot"])
            torch.cuda.current_stream().wait_stream(side)
            graph = torch.cuda.CUDAGraph()
            self._capturing = True
            try:
                with torch.cuda.graph(graph, capture_error_mode="relaxed"):
                    inp = [t.detach().requires_grad_(True) for t in G["state"]]
                    tt = G["top"].detach().requires_grad_(True) if key else None
                    G["out"] = self._vjp_body(inp, tt, G["dt"], G["cot"])
            finally:
                self._capturing = False
            G["graph"] = graph
            self._graphs[key] = G
        for buf, t in zip(G["state"], state):
            buf.copy_(t)
        for buf, c in zip(G["cot"], cot):
            buf.copy_(c)
        G["dt"].fill_(self.dts[j])
        if key:
            G["top"].copy_(Ttop)
            self._set_top(Ttop)
        G["graph"].replay()
        g_state, g_top = G["out"]
        return [t.clone() for t in g_state], (g_top.clone() if g_top is not None else None)


_DIFF_FN = None
_SWEEP_FN = None


def _sweep_fn():
    """torch.autograd.Function: CUDA field sweep forward, CUDA sweep VJP backward."""
    global _SWEEP_FN
    if _SWEEP_FN is None:
        import torch

        class SweepFn(torch.autograd.Function):
            @staticmethod
            def forward(ctx, f, v, problem, dim, frank, nsp, dt):
                f = f.contiguous()
                v = v.contiguous()
                out = f.clone()
                _lib.check(_lib.lib().gem_sweep_field_dev(problem.dg.handle, dim, frank, nsp, F._ptr(out), F._ptr(v),
                                                          F._ptr(dt), F._stream()))
                ctx.problem, ctx.dim, ctx.frank, ctx.nsp, ctx.dt = problem, dim, frank, nsp, dt
                ctx.save_for_backward(f, v)
                return out

            @staticmethod
            def backward(ctx, obar):
                f, v = ctx.saved_tensors
                P = ctx.problem
                obar = obar.contiguous()
                fbar = obar.clone()
                vbar = torch.zeros_like(v) if ctx.needs_input_grad[1] else None
                dt = ctx.dt
                _lib.check(_lib.lib().gem_sweep_field_vjp_dev(
                    P.dg.handle, ctx.dim, ctx.frank, ctx.nsp, F._ptr(f), F._ptr(v), F._ptr(dt), F._ptr(obar),
                    F._ptr(fbar), None if vbar is None else F._ptr(vbar), F._stream()))
                return fbar, vbar, None, None, None, None, None

        _SWEEP_FN = SweepFn
    return _SWEEP_FN


def _diffusion_fn():
    """torch.autograd.Function: CUDA energy diffusion forward, CUDA adjoint backward."""
    global _DIFF_FN
    if _DIFF_FN is None:
        import torch

        class DiffusionFn(torch.autograd.Function):
            @staticmethod
            def forward(ctx, n, T, Ttop, problem, dt):
                ctx.problem, ctx.dt = problem, dt
                ctx.save_for_backward(n, T, Ttop)
                return problem.diffusion_forward(n, T, Ttop, dt)

            @staticmethod
            def backward(ctx, Ybar):
                n, T, Ttop = ctx.saved_tensors
                nb, Tb, tb = ctx.problem.diffusion_vjp(n, T, Ttop, ctx.dt, Ybar)
                return nb, Tb, (tb if Ttop is not None else None), None, None

        _DIFF_FN = DiffusionFn
    return _DIFF_FN


class FluidAdvance:
    """torch.autograd.Function factory bound to a DiffProblem."""

    @staticmethod
    def apply(n0, Ttop, problem: DiffProblem):
        return _Fn.apply(n0, Ttop, problem)


def backward_from_checkpoints(P: "DiffProblem", ckpt, Ttop, g_ns, g_Ts):
    """Pull the cotangents of the final (ns, Ts) back to (n0, Ttop): segment by segment from
    the checkpoints {step: state}, recomputing each segment with the CUDA step."""
    import torch

    zeros = lambda t: torch.zeros_like(t)
    ns_f = P.base[0:LSP]
    cot = [g_ns if g_ns is not None else zeros(ns_f), zeros(ns_f),
           g_Ts if g_Ts is not None else zeros(ns_f), zeros(P.lo0), zeros(P.hi0)]
    g_top = torch.zeros_like(Ttop) if Ttop is not None else None
    starts = sorted(ckpt)
    if P.cuda_step_adjoint:
        cot, g_top = _backward_cuda(P, ckpt, starts, Ttop, cot, g_top)
        starts = []
    for seg_i in range(len(starts) - 1, -1, -1):
        j0 = starts[seg_i]
        j1 = starts[seg_i + 1] if seg_i + 1 < len(starts) else P.nsteps
        P._load(*ckpt[j0], Ttop)
        states = [ckpt[j0]]
        for j in range(j0, j1 - 1):
            P.cuda_step(j)
            states.append(P._save())
        for j in range(j1 - 1, j0 - 1, -1):
            cot, gt = P.step_vjp(states[j - j0], Ttop, j, cot, P.cuda_diffusion_adjoint)
            if gt is not None:
                g_top = g_top + gt
    g = P.grid
    I = (slice(2, g.lx3 + 2), slice(2, g.lx2 + 2), slice(2, g.lx1 + 2))
    gns = cot[0][(slice(None),) + I]
    g_n0 = gns[:LSP - 1] + gns[LSP - 1].unsqueeze(0)  # electrons = sum of ions
    return g_n0, g_top


def _backward_cuda(P: "DiffProblem", ckpt, starts, Ttop, cot, g_top):
    """The CUDA backward over all steps, last first.  With room on the device for k+1 step
    adjoint workspaces (k: the longest checkpoint segment), each step is replayed once and
    the replay serves both the recompute of the next state and the step's backward
    (_backward_cuda_slots); otherwise two workspaces alternate and the recompute runs the
    plain forward step (_backward_cuda_pingpong)."""
    import torch

    n = P.nsteps
    kmax = max((starts[i + 1] if i + 1 < len(starts) else n) - starts[i] for i in range(len(starts)))
    have = sum(1 for h in (P._sa or []) if h is not None)
    F1 = 8 * LSP * (P.grid.lx1 + 4) * (P.grid.lx2 + 4) * (P.grid.lx3 + 4)
    need = max(0, kmax + 1 - have) * P.workspace_bytes() + 2 * kmax * 3 * F1
    # the recompute's diffusion scratch first; the workspaces are raw cudaMalloc, which cannot
    # use memory held in torch's cache: release that only when the slots do not fit otherwise
    _lib.check(_lib.lib().gem_work_prepare(P.ds.work, P.dg.handle))
    free, _ = torch.cuda.mem_get_info()
    if P.replay_slots and need > 0.8 * free:
        torch.cuda.empty_cache()
        free, _ = torch.cuda.mem_get_info()
    if P.replay_slots and need <= 0.8 * free:
        try:
            for i in range(kmax + 1):  # made before the pipeline starts
                P._workspace(i)
        except _lib.GemError:
            P._drop_workspaces(keep=2)
        else:
            return _backward_cuda_slots(P, ckpt, starts, Ttop, cot, g_top, kmax + 1)
    return _backward_cuda_pingpong(P, ckpt, starts, Ttop, cot, g_top)


def _backward_cuda_slots(P: "DiffProblem", ckpt, starts, Ttop, cot, g_top, nslot):
    """The backward with nslot (>= k+1) replay slots.  The steps are recomputed in the order
    the backward needs them (segments last first, each from its checkpoint forward) on a
    second stream: gem_step_vjp_replay_dev of step j into a free slot, then, inside the
    segment, gem_step_vjp_finish_dev from that slot gives the state before step j+1.  Step
    j's backward (gem_step_vjp_backward_dev on the main stream) reads its slot and frees it;
    the next recompute step takes the freed slot.  With k+1 slots the recompute of a segment
    runs one step behind the backward of the segment after it, so no replay is exposed."""
    import collections

    import torch

    main = torch.cuda.current_stream()
    if getattr(P, "_rec", None) is None:
        P._rec = torch.cuda.Stream()
    rec = P._rec
    n = P.nsteps
    bounds = [(starts[i], starts[i + 1] if i + 1 < len(starts) else n) for i in range(len(starts))]
    seg_end = {j: j1 for j0, j1 in bounds for j in range(j0, j1)}
    P._set_top(Ttop)
    for j in range(n):  # the cached dt tensors, made on the main stream before the fork
        P.dt_tensor(j)
    states = {j0: tuple(t.detach().contiguous() for t in ckpt[j0]) for j0, _ in bounds}
    for i in range(nslot):  # workspaces are made (cudaMalloc) before the pipeline starts
        P._workspace(i)
    rec.wait_stream(main)
    pending = collections.deque(j for j0, j1 in reversed(bounds) for j in range(j0, j1))
    free = collections.deque(range(nslot))
    free_ev, slot_of, rep_ev = {}, {}, {}

    def issue():
        while pending and free:
            j = pending.popleft()
            sl = free.popleft()
            with torch.cuda.stream(rec):
                if sl in free_ev:  # the slot's last reader: a backward on the main stream
                    rec.wait_event(free_ev.pop(sl))
                P._replay(sl, states[j], j)
                slot_of[j] = sl
                rep_ev[j] = torch.cuda.Event()
                rep_ev[j].record(rec)
                if j + 1 < seg_end[j]:
                    st = P._finish(sl, j)
                    for t in st:  # read on the main stream before they are freed
                        t.record_stream(main)
                    states[j + 1] = st

    issue()
    for j in range(n - 1, -1, -1):
        main.wait_event(rep_ev.pop(j))
        sl = slot_of.pop(j)
        cot, gt = P._backward(sl, states.pop(j), Ttop, j, cot)
        if gt is not None:
            g_top = g_top + gt
        ev = torch.cuda.Event()
        ev.record(main)
        free_ev[sl] = ev
        free.append(sl)
        issue()
    main.wait_stream(rec)
    return cot, g_top


def _backward_cuda_pingpong(P: "DiffProblem", ckpt, starts, Ttop, cot, g_top):
    """The CUDA backward over all steps, last first, as one pipeline: the replay of step j-1
    (gem_step_vjp_replay_dev, on a side stream, into workspace (j-1) % 2) runs while step j's
    backward runs (workspace j % 2); with checkpoints every k > 1 steps, the recompute of a
    segment's states (the CUDA forward from its checkpoint, on a third stream) runs while
    the following segment is pulled back."""
    import torch

    main = torch.cuda.current_stream()
    if P._side is None:
        P._side = torch.cuda.Stream()
    if getattr(P, "_rec", None) is None:
        P._rec = torch.cuda.Stream()
    side, rec = P._side, P._rec
    n = P.nsteps
    bounds = [(starts[i], starts[i + 1] if i + 1 < len(starts) else n) for i in range(len(starts))]
    seg_of = {j: si for si, (j0, j1) in enumerate(bounds) for j in range(j0, j1)}
    P._set_top(Ttop)
    for j in range(n):  # the cached dt tensors, made on the main stream before the fork
        P.dt_tensor(j)
    states, ready = {}, {}

    def recompute(si):
        j0, j1 = bounds[si]
        states[j0] = tuple(t.detach().contiguous() for t in ckpt[j0])  # on the main stream
        rec.wait_stream(main)
        with torch.cuda.stream(rec):
            if j1 - j0 > 1:
                P._load(*ckpt[j0], Ttop)
                for j in range(j0, j1 - 1):
                    P.cuda_step(j)
                    st = P._save()
                    for t in st:  # read on the main and replay streams before they are freed
                        t.record_stream(main)
                        t.record_stream(side)
                    states[j + 1] = st
            ready[si] = torch.cuda.Event()
            ready[si].record(rec)

    ev_rep, ev_back = {}, {}

    def replay(j):
        with torch.cuda.stream(side):
            side.wait_event(ready[seg_of[j]])
            if j + 2 in ev_back:  # workspace j % 2 was last read by the backward of step j+2
                side.wait_event(ev_back[j + 2])
            P._replay(j % 2, states[j], j)
            ev_rep[j] = torch.cuda.Event()
            ev_rep[j].record(side)

    recompute(len(bounds) - 1)
    replay(n - 1)
    for j in range(n - 1, -1, -1):
        si = seg_of[j]
        if j == bounds[si][1] - 1 and si > 0:
            recompute(si - 1)  # overlaps this segment's backward
        if j >= 1:
            replay(j - 1)
        main.wait_event(ev_rep[j])
        cot, gt = P._backward(j % 2, states[j], Ttop, j, cot)
        ev_back[j] = torch.cuda.Event()
        ev_back[j].record(main)
        if gt is not None:
            g_top = g_top + gt
        if j + 2 in states:
            del states[j + 2]  # its replay and backward are queued; record_stream keeps it safe
    main.wait_stream(side)
    main.wait_stream(rec)
    return cot, g_top


class BatchedAdjoint:
    """Per-instance gradients for many independent instances (uneven sizes).

    Instances are processed in groups: a group's forward pass is one batched step per time
    step (gem_batch_step_fixed_dt: every instance on its own frozen schedule, all phases as
    one replayed CUDA graph), with each instance's state saved every k steps; then each
    instance's cotangent is pulled back from its checkpoints (recompute + step VJPs).  The
    group size bounds the checkpoint memory."""

    def __init__(self, instances, nsteps: int, checkpoint_every: int = 10, group: int = 8, **problem_kw):
        self.problems = [DiffProblem(g, st, nsteps, checkpoint_every=checkpoint_every, **problem_kw)
                         for g, st in instances]
        self.nsteps = int(nsteps)
        self.k = max(1, int(checkpoint_every))
        self.group = max(1, int(group))

    def forward_group(self, idx, controls, keep=True):
        """Batched forward of the instances idx from their controls [(n0, Ttop)]; returns the
        final states and the checkpoints of each."""
        from . import batch as BT

        Ps = [self.problems[i] for i in idx]
        for P, (n0, Ttop) in zip(Ps, controls):
            ns = P.initial_state(n0.detach())
            P._load(ns, P.base[LSP:2 * LSP], P.base[4 * LSP:], P.lo0, P.hi0, Ttop)
        b = BT.Batch([(P.dg, P.ds, P.cfg) for P in Ps])
        ckpts = [dict() for _ in Ps]
        for j in range(self.nsteps):
            if keep and j % self.k == 0:
                for c, P in zip(ckpts, Ps):
                    c[j] = P._save()
            b.step_fixed_dt([P.dts[j] for P in Ps])
        finals = [P._save() for P in Ps]
        b.close()
        return finals, ckpts

    def gradients(self, controls, loss_fn):
        """controls: [(n0, Ttop)] per instance; loss_fn(i, ns, Ts) -> scalar tensor.
        Returns [(loss, g_n0, g_Ttop)] per instance."""
        import torch

        out = [None] * len(self.problems)
        for g0 in range(0, len(self.problems), self.group):
            idx = list(range(g0, min(g0 + self.group, len(self.problems))))
            finals, ckpts = self.forward_group(idx, [controls[i] for i in idx])
            for i, fin, ck in zip(idx, finals, ckpts):
                ns = fin[0].detach().requires_grad_(True)
                Ts = fin[2].detach().requires_grad_(True)
                L = loss_fn(i, ns, Ts)
                gns, gTs = torch.autograd.grad(L, [ns, Ts], allow_unused=True)
                P = self.problems[i]
                g_n0, g_top = backward_from_checkpoints(P, ck, controls[i][1], gns, gTs)
                out[i] = (float(L.detach()), g_n0, g_top)
                P._graphs = {}  # release the captured VJP's memory pool
                P.close()
            del finals, ckpts
        return out


def _fn_class():
    import torch

    class Fn(torch.autograd.Function):
        @staticmethod
        def forward(ctx, n0, Ttop, problem):
            (ns, vs1, Ts, lo, hi), ckpt = problem.run(n0, Ttop, keep=True)
            ctx.problem = problem
            ctx.ckpt = ckpt
            ctx.save_for_backward(n0, Ttop)
            return ns, Ts

        @staticmethod
        def backward(ctx, g_ns, g_Ts):
            n0, Ttop = ctx.saved_tensors
            g_n0, g_top = backward_from_checkpoints(ctx.problem, ctx.ckpt, Ttop, g_ns, g_Ts)
            return g_n0, g_top, None

    return Fn


class _Lazy:
    _cls = None

    @classmethod
    def get(cls):
        if cls._cls is None:
            cls._cls = _fn_class()
        return cls._cls


class _FnProxy:
    @staticmethod
    def apply(*args):
        return _Lazy.get().apply(*args)


_Fn = _FnProxy


def misfit(ns, Ts, target_Te, target_nOp, grid, Te_scale=1000.0, n_scale=1e11):
    """L2 misfit of the final electron temperature and O+ density (interior)."""
    I = (slice(2, grid.lx3 + 2), slice(2, grid.lx2 + 2), slice(2, grid.lx1 + 2))
    dT = (Ts[(LSP - 1,) + I] - target_Te) / Te_scale
    dn = (ns[(0,) + I] - target_nOp) / n_scale
    return 0.5 * (dT * dT).mean() + 0.5 * (dn * dn).mean()


def torch_reference_loss(problem: DiffProblem, n0, Ttop, target_Te, target_nOp):
    """The same loss computed by the pure-tensor transcription (autograd end to end)."""
    P = problem
    ns = P.initial_state(n0)
    vs1, Ts, lo, hi = P.base[LSP:2 * LSP], P.base[4 * LSP:], P.lo0, P.hi0
    for j in range(P.nsteps):
        ns, vs1, Ts, lo, hi = TS.step(P.tg, ns, vs1, P.vs2, P.vs3, Ts, lo, hi, P.nn, P.Tn, P.J1, P.dts[j],
                                      P.Teinf, Ttop, P.diffsolvetype)
    return misfit(ns, Ts, target_Te, target_nOp, P.grid)
