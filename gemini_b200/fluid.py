"""Device-resident fluid advance with the reference's routine names.

This module mirrors the ``*_in`` procedures of ``src/libgemini.f90`` (731-1075) and the
species wrappers of ``src/multifluid/multifluid.f90`` (49-126) for the advection sweeps and
the energy diffusion, on state blocks that live in GPU memory (torch tensors holding the
reference's Fortran-layout blocks).  Every call goes through the C ABI of
``libgemini_b200.so``; there is no CPU path.

    dg = DeviceGrid(grid)                       # curvmesh on the device (read_grid)
    ds = DeviceState.from_host(dg, state)       # fluidvars / fluidauxvars / electrovars
    dt = dt_calc(ds, tcfl=0.5)                  # device scalar (dt_select)
    fluid_adv(cfg, ds, dt)                      # the advection + diffusion step
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib
from .grid import Grid
from .state import FluidState, LSP, NAUX, NELECTRO, NFLUID


def _torch():
    import torch  # noqa: PLC0415  (torch is only needed for device memory and streams)
    return torch


def _stream(stream=None):
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def _ptr(t) -> ctypes.c_void_p:
    return ctypes.c_void_p(t.data_ptr())


@dataclass
class FluidCfg:
    """gemini_cfg fields read on this path (diffsolvetype, Teinf, tcfl; config_nml.f90)."""

    Teinf: float
    diffsolvetype: int = 2
    tcfl: float = 0.5
    flagglow: int = 0

    def c(self) -> _lib.GemCfg:
        return _lib.GemCfg(float(self.Teinf), int(self.diffsolvetype), float(self.tcfl), int(self.flagglow))


class DeviceGrid:
    """A curvmesh copied to the device once (meshobj fields the hot path reads)."""

    def __init__(self, grid: Grid, unit_metrics: bool | None = None):
        L = _lib.lib()
        self.grid = grid
        self._keep = []
        kw = {}
        for n in ("dx1", "dx1i", "dx2", "dx2i", "dx3", "dx3i", "h1", "h2", "h3", "h1x1i", "h2x1i",
                  "h3x1i", "h1x2i", "h2x2i", "h3x2i", "h1x3i", "h2x3i", "h3x3i"):
            a = np.asfortranarray(getattr(grid, n), dtype=np.float64)
            self._keep.append(a)
            kw[n] = a.ctypes.data_as(_lib._D)
        nul = np.asfortranarray(grid.nullpts, dtype=np.uint8)
        self._keep.append(nul)
        unit = grid.unit_metrics if unit_metrics is None else unit_metrics
        desc = _lib.GemGridDesc(lx1=grid.lx1, lx2=grid.lx2, lx3=grid.lx3, gridflag=grid.gridflag,
                                flagper=grid.flagper, nullpts=nul.ctypes.data_as(_lib._U8),
                                unit_metrics=1 if unit else 0, **kw)
        h = ctypes.c_void_p()
        _lib.check(L.gem_grid_create(ctypes.byref(desc), ctypes.byref(h)))
        self.handle = h
        self._keep = None  # the arrays were copied to the device

    @property
    def dims(self):
        return self.grid.lx1, self.grid.lx2, self.grid.lx3

    @property
    def ng(self) -> int:
        lx1, lx2, lx3 = self.dims
        return (lx1 + 4) * (lx2 + 4) * (lx3 + 4)

    def bind(self) -> None:
        """Make this the grid the size-less reference entry points use."""
        _lib.lib().gem_capi_bind_grid(self.handle)

    def close(self) -> None:
        if getattr(self, "handle", None) is not None and self.handle.value:
            _lib.lib().gem_grid_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 -- interpreter shutdown
            pass


class DeviceState:
    """State blocks in device memory plus the work object (gemini_work equivalent)."""

    def __init__(self, dgrid: DeviceGrid, fluidvars, fluidauxvars, electrovars, Teinf: float):
        self.dgrid = dgrid
        self.fluidvars = fluidvars
        self.fluidauxvars = fluidauxvars
        self.electrovars = electrovars
        self.Teinf = Teinf
        h = ctypes.c_void_p()
        _lib.check(_lib.lib().gem_work_create(dgrid.handle, ctypes.byref(h)))
        self.work = h
        torch = _torch()
        self.dt = torch.zeros(1, dtype=torch.float64, device=fluidvars.device)

    # -- construction / transfer ---------------------------------------------------------
    @classmethod
    def from_host(cls, dgrid: DeviceGrid, st: FluidState, device="cuda") -> "DeviceState":
        torch = _torch()
        def dev(a):
            return torch.from_numpy(np.asfortranarray(a).ravel(order="K").copy()).to(device)
        ds = cls(dgrid, dev(st.fluidvars), dev(st.fluidauxvars), dev(st.electrovars), st.Teinf)
        ds.set_neutrals(st.nn, st.Tn)
        for which, a in ((1, st.vs1i), (2, st.vs2i), (3, st.vs3i)):
            ds.set_interface_vels(which, a)
        return ds

    def set_neutrals(self, nn: np.ndarray, Tn: np.ndarray) -> None:
        nn = np.asfortranarray(nn, dtype=np.float64)
        Tn = np.asfortranarray(Tn, dtype=np.float64)
        _lib.check(_lib.lib().gem_work_set_neutrals(self.work, nn.ctypes.data, Tn.ctypes.data))

    def set_interface_vels(self, which: int, a: np.ndarray) -> None:
        a = np.asfortranarray(a, dtype=np.float64)
        _lib.check(_lib.lib().gem_work_interface_vels(self.work, which, a.ctypes.data, 0))

    def interface_vels(self, which: int) -> np.ndarray:
        lx1, lx2, lx3 = self.dgrid.dims
        shape = {1: (lx1 + 1, lx2, lx3, LSP), 2: (lx1, lx2 + 1, lx3, LSP), 3: (lx1, lx2, lx3 + 1, LSP)}[which]
        a = np.zeros(shape, dtype=np.float64, order="F")
        _lib.check(_lib.lib().gem_work_interface_vels(self.work, which, a.ctypes.data, 1))
        return a

    def to_host(self, like: FluidState | None = None) -> FluidState:
        _torch().cuda.synchronize()
        g = self.dgrid.grid
        gs = g.shape_ghosted
        def host(t, nvar):
            return t.cpu().numpy().reshape(gs + (nvar,), order="F").copy(order="F")
        nn = like.nn if like is not None else None
        Tn = like.Tn if like is not None else None
        return FluidState(host(self.fluidvars, NFLUID), host(self.fluidauxvars, NAUX),
                          host(self.electrovars, NELECTRO), self.interface_vels(1),
                          self.interface_vels(2), self.interface_vels(3), nn, Tn, self.Teinf)

    def close(self) -> None:
        if getattr(self, "work", None) is not None and self.work.value:
            _lib.lib().gem_work_destroy(self.work)
            self.work = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass

    # -- pointers ---------------------------------------------------------------------------
    @property
    def g(self):
        return self.dgrid.handle

    def _dt(self, dt):
        torch = _torch()
        if isinstance(dt, torch.Tensor):
            return dt
        self.dt.fill_(float(dt))
        return self.dt


# ---- the reference's routines (libgemini.f90 *_in, multifluid.f90 wrappers) ------------------

def v12rhov1(ds: DeviceState, stream=None):
    _lib.check(_lib.lib().gem_v12rhov1_dev(ds.g, _ptr(ds.fluidvars), _ptr(ds.fluidauxvars), _stream(stream)))


def T2rhoe(ds: DeviceState, stream=None):
    _lib.check(_lib.lib().gem_T2rhoe_dev(ds.g, _ptr(ds.fluidvars), _ptr(ds.fluidauxvars), _stream(stream)))


def rhov12v1(ds: DeviceState, stream=None):
    _lib.check(_lib.lib().gem_rhov12v1_dev(ds.g, _ptr(ds.fluidvars), _ptr(ds.fluidauxvars), _stream(stream)))


def rhoe2T(ds: DeviceState, stream=None):
    _lib.check(_lib.lib().gem_rhoe2T_dev(ds.g, _ptr(ds.fluidvars), _ptr(ds.fluidauxvars), _stream(stream)))


def set_global_boundaries_allspec(ds: DeviceState, lsp: int = LSP, stream=None):
    _lib.check(_lib.lib().gem_set_global_boundaries_allspec_dev(
        ds.g, _ptr(ds.fluidvars), _ptr(ds.fluidauxvars), ds.work, lsp, _stream(stream)))


def halo_fluidvars(ds: DeviceState, stream=None):
    _lib.check(_lib.lib().gem_halo_fluidvars_dev(ds.g, _ptr(ds.fluidvars), _ptr(ds.fluidauxvars), _stream(stream)))


def halo_allparams(ds: DeviceState, stream=None):
    _lib.check(_lib.lib().gem_halo_allparams_dev(ds.g, _ptr(ds.fluidvars), _ptr(ds.fluidauxvars), _stream(stream)))


def interface_vels_allspec(ds: DeviceState, lsp: int = LSP, stream=None):
    _lib.check(_lib.lib().gem_interface_vels_allspec_dev(ds.g, _ptr(ds.fluidvars), ds.work, lsp, _stream(stream)))


# ---- the compression sub-step (app/main.f90:320-338) -----------------------------------------

def vnricht_artvisc(ds: DeviceState, Q=None, stream=None):
    """VNRicht_artvisc (multifluid.f90:237-268): Q (lx1, lx2, lx3, lsp), Fortran order, as a
    flat float64 device tensor; Q is allocated when not given."""
    torch = _torch()
    lx1, lx2, lx3 = ds.dgrid.dims
    if Q is None:
        Q = torch.empty(lx1 * lx2 * lx3 * LSP, dtype=torch.float64, device=ds.fluidvars.device)
    _lib.check(_lib.lib().gem_vnricht_artvisc_dev(ds.g, _ptr(ds.fluidvars), _ptr(Q), _stream(stream)))
    return Q


def rk2_global_boundary_allspec(ds: DeviceState, stream=None):
    """RK2_global_boundary (sources_mpi.f90:68-111) of vs1, vs2, vs3 on a single rank."""
    _lib.check(_lib.lib().gem_rk2_global_boundary_allspec_dev(ds.g, _ptr(ds.fluidvars), _stream(stream)))


def compression(ds: DeviceState, Q, dt, stream=None):
    """compression (multifluid.f90:274-302): rhoes updated in place with Q from vnricht_artvisc."""
    d = ds._dt(dt)
    _lib.check(_lib.lib().gem_compression_dev(ds.g, _ptr(ds.fluidvars), _ptr(ds.fluidauxvars), _ptr(Q), _ptr(d),
                                              _stream(stream)))


# ---- the source/loss solves (multifluid.f90:474-549) -----------------------------------------
# Pr, Lo, Prprecip, Qeprecip: flat float64 device tensors holding the interior arrays
# (lx1, lx2, lx3, species) in column-major order; Pr is updated in place where the reference
# updates it.

def energy_source_loss_solve(ds: DeviceState, dt, Pr, Lo, Qeprecip, stream=None):
    d = ds._dt(dt)
    _lib.check(_lib.lib().gem_energy_source_loss_solve_dev(ds.g, _ptr(d), _ptr(Pr), _ptr(Lo), _ptr(Qeprecip),
                                                           _ptr(ds.fluidvars), _ptr(ds.fluidauxvars),
                                                           _stream(stream)))


def momentum_source_loss_solve(ds: DeviceState, dt, Pr, Lo, stream=None):
    d = ds._dt(dt)
    _lib.check(_lib.lib().gem_momentum_source_loss_solve_dev(ds.g, _ptr(d), _ptr(Pr), _ptr(Lo), _ptr(ds.fluidvars),
                                                             _ptr(ds.fluidauxvars), _stream(stream)))


def mass_source_loss_solve(ds: DeviceState, dt, Pr, Lo, Prprecip, stream=None):
    d = ds._dt(dt)
    _lib.check(_lib.lib().gem_mass_source_loss_solve_dev(ds.g, _ptr(d), _ptr(Pr), _ptr(Lo), _ptr(Prprecip),
                                                         _ptr(ds.fluidvars), _stream(stream)))


# ---- the production/loss rates (sources.f90) --------------------------------------------------
# nn, vn1..3, Tn, alt, g1, Q: flat float64 device tensors of the interior arrays in column-major
# order; each returns (Pr, Lo), flat (lx1, lx2, lx3, lsp) device tensors.

def _rate_out(ds: DeviceState):
    torch = _torch()
    lx1, lx2, lx3 = ds.dgrid.dims
    mk = lambda: torch.empty(lx1 * lx2 * lx3 * LSP, dtype=torch.float64, device=ds.fluidvars.device)
    return mk(), mk()


def srcs_continuity(ds: DeviceState, nn, vn1, vn2, vn3, Tn, stream=None):
    Pr, Lo = _rate_out(ds)
    _lib.check(_lib.lib().gem_srcs_continuity_dev(ds.g, _ptr(nn), _ptr(vn1), _ptr(vn2), _ptr(vn3), _ptr(Tn),
                                                  _ptr(ds.fluidvars), _ptr(Pr), _ptr(Lo), _stream(stream)))
    return Pr, Lo


def srcs_energy(ds: DeviceState, nn, vn1, vn2, vn3, Tn, stream=None):
    Pr, Lo = _rate_out(ds)
    _lib.check(_lib.lib().gem_srcs_energy_dev(ds.g, _ptr(nn), _ptr(vn1), _ptr(vn2), _ptr(vn3), _ptr(Tn),
                                              _ptr(ds.fluidvars), _ptr(Pr), _ptr(Lo), _stream(stream)))
    return Pr, Lo


def srcs_momentum(ds: DeviceState, nn, vn1, Tn, Q, alt, g1, stream=None):
    """E1 is read from the state's electrovars (block 1)."""
    Pr, Lo = _rate_out(ds)
    _lib.check(_lib.lib().gem_srcs_momentum_dev(ds.g, _ptr(nn), _ptr(vn1), _ptr(Tn), _ptr(ds.fluidvars),
                                                _ptr(ds.electrovars), _ptr(Q), _ptr(alt), _ptr(g1), _ptr(Pr),
                                                _ptr(Lo), _stream(stream)))
    return Pr, Lo


# ---- fluid_adv in full (app/main.f90:280-381) ---------------------------------------------------

class SourceInputs(ctypes.Structure):
    """gem_source_inputs: device pointers of the interior neutral state (nn: O, N2, O2, H, N,
    NO), altitude, gravity and ionization rates the source sub-step reads."""
    _fields_ = [(n, ctypes.c_void_p) for n in ("nn", "vn1", "vn2", "vn3", "Tn", "alt", "g1", "Prionize", "Qeionize")]

    @classmethod
    def of(cls, **tensors):
        s = cls(**{k: t.data_ptr() for k, t in tensors.items()})
        s._keep = tensors  # the tensors must outlive the launches
        return s


def fluid_adv_compression(cfg: FluidCfg, ds: DeviceState, dt, Q=None, stream=None):
    """The step with the compression sub-step (the advection through the fused kernels where
    the grid allows them, the rest as the reference's sequence of routines); returns Q (flat
    interior (lx1, lx2, lx3, lsp) device tensor) for the source sub-step."""
    torch = _torch()
    lx1, lx2, lx3 = ds.dgrid.dims
    if Q is None:
        Q = torch.empty(lx1 * lx2 * lx3 * LSP, dtype=torch.float64, device=ds.fluidvars.device)
    d = ds._dt(dt)
    c = cfg.c()
    _lib.check(_lib.lib().gem_fluid_adv_compression_dev(ctypes.byref(c), ds.g, _ptr(ds.fluidvars),
                                                         _ptr(ds.fluidauxvars), _ptr(ds.electrovars), ds.work,
                                                         _ptr(Q), _ptr(d), _stream(stream)))
    return Q


def fluid_adv_compression_reference_order(cfg: FluidCfg, ds: DeviceState, dt, Q=None, stream=None):
    """The step with the compression sub-step as the reference's sequence of individual
    routines (app/main.f90:280-355); fluid_adv_compression runs the advection part through
    the fused kernels.  Returns Q as fluid_adv_compression does."""
    d = ds._dt(dt)
    v12rhov1(ds, stream)
    T2rhoe(ds, stream)
    set_global_boundaries_allspec(ds, LSP, stream)
    halo_fluidvars(ds, stream)
    interface_vels_allspec(ds, LSP, stream)
    for dim in (3, 1):
        for which in (0, 1, 2):
            _sweep(ds, dim, which, d, stream)
    halo_allparams(ds, stream)
    for which in (0, 1, 2):
        _sweep(ds, 2, which, d, stream)
    rhov12v1(ds, stream)
    clean_param(ds, 1, stream)
    clean_param(ds, 2, stream)
    Q = vnricht_artvisc(ds, Q, stream)
    halo_fluidvars(ds, stream)
    rk2_global_boundary_allspec(ds, stream)
    compression(ds, Q, d, stream)
    rhoe2T(ds, stream)
    clean_param(ds, 3, stream)
    energy_diffusion(cfg, ds, d, stream)
    clean_param(ds, 3, stream)
    T2rhoe(ds, stream)
    return Q


def source_loss_allparams(ds: DeviceState, dt, inputs: SourceInputs, Q, stream=None):
    """The source/loss sub-step (libgemini.f90:1154-1200) after the step with compression."""
    Pr, Lo = _rate_out(ds)
    d = ds._dt(dt)
    _lib.check(_lib.lib().gem_source_loss_allparams_dev(ds.g, _ptr(ds.fluidvars), _ptr(ds.fluidauxvars),
                                                         _ptr(ds.electrovars), ds.work, ctypes.byref(inputs), _ptr(Q),
                                                         _ptr(Pr), _ptr(Lo), _ptr(d), _stream(stream)))


def fluid_adv_full(cfg: FluidCfg, ds: DeviceState, dt, inputs: SourceInputs, scratch=None, stream=None):
    """fluid_adv in full on a single rank: the step with compression, then the sources."""
    torch = _torch()
    if scratch is None:
        n = _lib.lib().gem_fluid_adv_full_scratch_doubles(ds.g)
        scratch = torch.empty(n, dtype=torch.float64, device=ds.fluidvars.device)
    d = ds._dt(dt)
    c = cfg.c()
    _lib.check(_lib.lib().gem_fluid_adv_full_dev(ctypes.byref(c), ds.g, _ptr(ds.fluidvars), _ptr(ds.fluidauxvars),
                                                  _ptr(ds.electrovars), ds.work, ctypes.byref(inputs), _ptr(scratch),
                                                  _ptr(d), _stream(stream)))
    return scratch


def _sweep(ds: DeviceState, dim: int, which: int, dt, stream=None):
    d = ds._dt(dt)
    _lib.check(_lib.lib().gem_sweep_allspec_dev(ds.g, dim, which, _ptr(ds.fluidvars), _ptr(ds.fluidauxvars),
                                                 ds.work, _ptr(d), _stream(stream)))


def sweep1_allspec_mass(ds, dt, stream=None):
    _sweep(ds, 1, 0, dt, stream)


def sweep1_allspec_momentum(ds, dt, stream=None):
    _sweep(ds, 1, 1, dt, stream)


def sweep1_allspec_energy(ds, dt, stream=None):
    _sweep(ds, 1, 2, dt, stream)


def sweep2_allspec_mass(ds, dt, stream=None):
    _sweep(ds, 2, 0, dt, stream)


def sweep2_allspec_momentum(ds, dt, stream=None):
    _sweep(ds, 2, 1, dt, stream)


def sweep2_allspec_energy(ds, dt, stream=None):
    _sweep(ds, 2, 2, dt, stream)


def sweep3_allspec_mass(ds, dt, stream=None):
    _sweep(ds, 3, 0, dt, stream)


def sweep3_allspec_momentum(ds, dt, stream=None):
    _sweep(ds, 3, 1, dt, stream)


def sweep3_allspec_energy(ds, dt, stream=None):
    _sweep(ds, 3, 2, dt, stream)


def clean_param(ds: DeviceState, iparm: int, stream=None):
    _lib.check(_lib.lib().gem_clean_param_dev(ds.g, iparm, _ptr(ds.fluidvars), _stream(stream)))


def energy_diffusion(cfg: FluidCfg, ds: DeviceState, dt, stream=None):
    d = ds._dt(dt)
    c = cfg.c()
    _lib.check(_lib.lib().gem_energy_diffusion_dev(ctypes.byref(c), ds.g, _ptr(ds.fluidvars),
                                                    _ptr(ds.electrovars), ds.work, _ptr(d), _stream(stream)))


def dt_calc(ds: DeviceState, tcfl: float = 0.5, out=None, stream=None):
    """temporal_mpi.f90:86-167 (+ the 1e-6 floor); returns a 1-element device tensor."""
    torch = _torch()
    out = out if out is not None else torch.empty(1, dtype=torch.float64, device=ds.fluidvars.device)
    _lib.check(_lib.lib().gem_dt_calc_dev(ds.g, float(tcfl), _ptr(ds.fluidvars), ds.work, _ptr(out),
                                          _stream(stream)))
    return out


def maxcfl(ds: DeviceState, dt, stream=None) -> float:
    torch = _torch()
    d = ds._dt(dt)
    out = torch.empty(1, dtype=torch.float64, device=ds.fluidvars.device)
    _lib.check(_lib.lib().gem_maxcfl_dev(ds.g, _ptr(ds.fluidvars), ds.work, _ptr(d), _ptr(out), _stream(stream)))
    return float(out.item())


def fluid_adv(cfg: FluidCfg, ds: DeviceState, dt, stream=None):
    """The advection + diffusion subset of fluid_adv (app/main.f90:280-355), fused."""
    d = ds._dt(dt)
    c = cfg.c()
    _lib.check(_lib.lib().gem_fluid_adv_dev(ctypes.byref(c), ds.g, _ptr(ds.fluidvars), _ptr(ds.fluidauxvars),
                                             _ptr(ds.electrovars), ds.work, _ptr(d), _stream(stream)))


def fluid_adv_reference_order(cfg: FluidCfg, ds: DeviceState, dt, stream=None):
    """The same step as fluid_adv, as the reference's sequence of individual routines."""
    d = ds._dt(dt)
    v12rhov1(ds, stream)
    T2rhoe(ds, stream)
    set_global_boundaries_allspec(ds, LSP, stream)
    halo_fluidvars(ds, stream)
    interface_vels_allspec(ds, LSP, stream)
    for dim in (3, 1):
        for which in (0, 1, 2):
            _sweep(ds, dim, which, d, stream)
    halo_allparams(ds, stream)
    for which in (0, 1, 2):
        _sweep(ds, 2, which, d, stream)
    rhov12v1(ds, stream)
    clean_param(ds, 1, stream)
    clean_param(ds, 2, stream)
    rhoe2T(ds, stream)
    clean_param(ds, 3, stream)
    energy_diffusion(cfg, ds, d, stream)
    clean_param(ds, 3, stream)
    T2rhoe(ds, stream)


def check_finite(ds: DeviceState, stream=None) -> int:
    """Number of non-finite interior values of ns, vs1, Ts (check_finite_output analogue)."""
    n = ctypes.c_longlong(0)
    rc = _lib.lib().gem_check_finite(ds.g, _ptr(ds.fluidvars), ds.work, ctypes.byref(n), _stream(stream))
    if rc not in (_lib.GEM_OK, _lib.GEM_ENONFINITE):
        _lib.check(rc)
    return int(n.value)


def fluid_adv_host(cfg: FluidCfg, dgrid: DeviceGrid, work_owner: DeviceState, fluidvars: np.ndarray,
                   fluidauxvars: np.ndarray, electrovars: np.ndarray, dt: float = -1.0, stream=None) -> float:
    """One step through host buffers (gem_fluid_adv_host); returns the dt used."""
    c = cfg.c()
    dtv = ctypes.c_double(dt)
    _lib.check(_lib.lib().gem_fluid_adv_host(ctypes.byref(c), dgrid.handle, fluidvars.ctypes.data,
                                              fluidauxvars.ctypes.data, electrovars.ctypes.data,
                                              work_owner.work, ctypes.byref(dtv), _stream(stream)))
    return float(dtv.value)
