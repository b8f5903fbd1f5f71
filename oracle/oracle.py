"""TEST INFRASTRUCTURE -- the CPU oracle, never the product.

ctypes wrapper over ``oracle/liboracle.so`` (``gemini_oracle.cpp``), a line-by-line C++
restatement of the reference Fortran for the fluid-advance hot path.  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg import this module, to
check or time the product against the reference's algorithm.

Inputs are duck-typed: any grid object with the ``curvmesh`` fields of
``gemini_b200.grid.Grid`` and any state with the block arrays of
``gemini_b200.state.FluidState`` (Fortran-ordered float64 numpy arrays).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
LSP = 7

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)
_U8 = ctypes.POINTER(ctypes.c_ubyte)


class OraGrid(ctypes.Structure):
    _fields_ = [("lx1", ctypes.c_int), ("lx2", ctypes.c_int), ("lx3", ctypes.c_int),
                ("gridflag", ctypes.c_int), ("flagper", ctypes.c_int)] + \
               [(n, _D) for n in ("dx1", "dx1i", "dx2", "dx2i", "dx3", "dx3i",
                                  "h1", "h2", "h3", "h1x1i", "h2x1i", "h3x1i",
                                  "h1x2i", "h2x2i", "h3x2i", "h1x3i", "h2x3i", "h3x3i")] + \
               [("nullpts", _U8)]


def build(force: bool = False) -> str:
    """Compile liboracle.so with its Makefile (test infrastructure)."""
    if force or not os.path.exists(_LIB_PATH) or \
            os.path.getmtime(_LIB_PATH) < os.path.getmtime(os.path.join(_HERE, "gemini_oracle.cpp")):
        subprocess.check_call(["make", "-s", "-C", _HERE, "liboracle.so"])
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        G = ctypes.POINTER(OraGrid)
        L.ora_sweep_allspec.argtypes = [G, ctypes.c_int, _D, _D, ctypes.c_double, ctypes.c_int, ctypes.c_int]
        L.ora_set_global_boundaries_allspec.argtypes = [G, _D, _D, _D, _D, _D, _D, _D, ctypes.c_int]
        L.ora_halo_allparams.argtypes = [G, _D, _D, _D]
        L.ora_halo_fluidvars.argtypes = [G, _D, _D, _D, _D, _D]
        L.ora_interface_vels_allspec.argtypes = [G, _D, _D, _D, _D, _D, _D, ctypes.c_int]
        L.ora_rhoe2T.argtypes = [G, _D, _D, _D]
        L.ora_T2rhoe.argtypes = [G, _D, _D, _D]
        L.ora_v12rhov1.argtypes = [G, _D, _D, _D]
        L.ora_rhov12v1.argtypes = [G, _D, _D, _D]
        L.ora_clean_param.argtypes = [G, ctypes.c_int, _D]
        L.ora_dgbsv.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _D, ctypes.c_int, _I, _D]
        L.ora_dgbsv.restype = ctypes.c_int
        sig1d = [ctypes.c_int, _D, _D, _D, _D, _D, _D, ctypes.c_double, ctypes.c_double,
                 ctypes.c_double, _D, _D, _D]
        L.ora_TRBDF21D.argtypes = sig1d
        L.ora_backEuler1D.argtypes = sig1d
        L.ora_energy_diffusion.argtypes = [G, _D, _D, _D, _D, _D, ctypes.c_double, ctypes.c_int,
                                           ctypes.c_double]
        L.ora_energy_diffusion.restype = ctypes.c_int
        L.ora_dt_calc.argtypes = [G, ctypes.c_double, _D, _D, _D, _D, _D]
        L.ora_dt_calc.restype = ctypes.c_double
        L.ora_dt_select.argtypes = [G, ctypes.c_double, _D, _D, _D, _D, ctypes.c_double, ctypes.c_double,
                                    ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_double]
        L.ora_dt_select.restype = ctypes.c_double
        L.ora_fluid_adv.argtypes = [G, _D, _D, _D, _D, _D, _D, _D, _D, ctypes.c_double,
                                    ctypes.c_double, ctypes.c_int]
        L.ora_fluid_adv.restype = ctypes.c_int
        L.ora_fluid_adv_compression.argtypes = L.ora_fluid_adv.argtypes
        L.ora_fluid_adv_compression.restype = ctypes.c_int
        L.ora_vnricht_artvisc.argtypes = [G, _D, _D, _D]
        L.ora_rk2_global_boundary_allspec.argtypes = [G, _D, _D, _D]
        L.ora_div3D.argtypes = [G, _D, _D, _D, _D]
        L.ora_compression.argtypes = [G, ctypes.c_double, _D, _D, _D, _D, _D]
        L.ora_etd_uncoupled.argtypes = [ctypes.c_longlong, _D, _D, _D, ctypes.c_double, _D]
        L.ora_srcs_continuity.argtypes = [G, _D, _D, _D, _D, _D, _D, _D, _D, _D, _D, _D, _D]
        L.ora_srcs_energy.argtypes = [G, _D, _D, _D, _D, _D, _D, _D, _D, _D, _D, _D, _D]
        L.ora_srcs_momentum.argtypes = [G] + [_D] * 14
        L.ora_fluid_adv_full.argtypes = [G] + [_D] * 16 + [ctypes.c_double, ctypes.c_double, ctypes.c_int]
        L.ora_fluid_adv_full.restype = ctypes.c_int
        L.ora_mass_source_loss_solve.argtypes = [G, ctypes.c_double, _D, _D, _D, _D]
        L.ora_momentum_source_loss_solve.argtypes = [G, ctypes.c_double, _D, _D, _D, _D, _D]
        L.ora_energy_source_loss_solve.argtypes = [G, ctypes.c_double, _D, _D, _D, _D, _D, _D]
        L.ora_constants.argtypes = [_D, _D, _D, _D]
        L.ora_num_threads.restype = ctypes.c_int
        L.ora_set_diffusion_solver.argtypes = [ctypes.c_int]
        L.ora_set_pow_mode.argtypes = [ctypes.c_int]
        L.ora_pow25.argtypes = [ctypes.c_double]
        L.ora_pow25.restype = ctypes.c_double
        L.ora_set_num_threads.argtypes = [ctypes.c_int]
        L.ora_advec1D_MC_curv.argtypes = [_D, _D, ctypes.c_double, _D, _D, _D, _D, _D, ctypes.c_int, _D]
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and (a.flags.f_contiguous or a.ndim == 1), "need Fortran float64"
    return a.ctypes.data_as(_D)


class _GridHandle:
    """Keeps the numpy arrays alive while the C struct points at them."""

    def __init__(self, grid):
        self._keep = []
        kw = {}
        for n in ("dx1", "dx1i", "dx2", "dx2i", "dx3", "dx3i", "h1", "h2", "h3", "h1x1i", "h2x1i",
                  "h3x1i", "h1x2i", "h2x2i", "h3x2i", "h1x3i", "h2x3i", "h3x3i"):
            a = np.asfortranarray(getattr(grid, n), dtype=np.float64)
            self._keep.append(a)
            kw[n] = a.ctypes.data_as(_D)
        nul = np.asfortranarray(grid.nullpts, dtype=np.uint8)
        self._keep.append(nul)
        self.s = OraGrid(lx1=grid.lx1, lx2=grid.lx2, lx3=grid.lx3, gridflag=grid.gridflag,
                         flagper=grid.flagper, nullpts=nul.ctypes.data_as(_U8), **kw)

    @property
    def ref(self):
        return ctypes.byref(self.s)


def set_diffusion_solver(mode: int) -> None:
    """0: LAPACK dgbsv restated (default); 1: extended-precision solve of the same system."""
    lib().ora_set_diffusion_solver(int(mode))


def set_pow_mode(mode: int) -> None:
    """0: libm pow(T, 2.5) as the Fortran calls it (default); 1: correctly rounded T**2.5."""
    lib().ora_set_pow_mode(int(mode))


def set_exact_dependencies(on: bool) -> None:
    set_diffusion_solver(1 if on else 0)
    set_pow_mode(1 if on else 0)


def set_device_semantics(on: bool) -> None:
    """The reference's arithmetic as the device reproduces it: the restated LAPACK band solve
    (solver 0) with the correctly rounded T**2.5 (pow mode 1).  Off: the defaults (LAPACK,
    C-library pow)."""
    set_diffusion_solver(0)
    set_pow_mode(1 if on else 0)


def pow25(x: float) -> float:
    return float(lib().ora_pow25(float(x)))


def markstein_mismatches(n: int, seed: int = 1) -> tuple[int, int]:
    """(mismatches, guarded cases) of the device's reciprocal-corrected division vs a/b."""
    L = lib()
    f = L.ora_markstein_mismatches
    f.restype = ctypes.c_longlong
    f.argtypes = [ctypes.c_longlong, ctypes.c_ulonglong, ctypes.POINTER(ctypes.c_longlong)]
    cnt = ctypes.c_longlong(0)
    bad = f(int(n), int(seed), ctypes.byref(cnt))
    return int(bad), int(cnt.value)


def set_num_threads(n: int) -> None:
    lib().ora_set_num_threads(int(n))


def num_threads() -> int:
    return int(lib().ora_num_threads())


def dgbsv(ab: np.ndarray, b: np.ndarray, kl: int, ku: int):
    """LAPACK dgbsv restated; ab (2kl+ku+1, n) Fortran band storage.  Returns (lu, ipiv, x, info)."""
    ab = np.array(ab, dtype=np.float64, order="F", copy=True)
    x = np.array(b, dtype=np.float64, copy=True)
    n = ab.shape[1]
    ipiv = np.zeros(n, dtype=np.int32)
    info = lib().ora_dgbsv(n, kl, ku, _p(ab), ab.shape[0], ipiv.ctypes.data_as(_I), _p(x))
    return ab, ipiv, x, info


def trbdf2_1d(Ts, A, B, C, D, E, tmin, tmax, dt, dx1, dx1i):
    """PDEparabolic.f90:19-218 on one column."""
    n = len(Ts)
    arr = [np.ascontiguousarray(v, dtype=np.float64) for v in (Ts, A, B, C, D, E, dx1, dx1i)]
    out = np.zeros(n)
    lib().ora_TRBDF21D(n, *(_p(v) for v in arr[:6]), tmin, tmax, dt, _p(arr[6]), _p(arr[7]), _p(out))
    return out


def backeuler_1d(Ts, A, B, C, D, E, tmin, tmax, dt, dx1, dx1i):
    """PDEparabolic.f90:221-346 on one column."""
    n = len(Ts)
    arr = [np.ascontiguousarray(v, dtype=np.float64) for v in (Ts, A, B, C, D, E, dx1, dx1i)]
    out = np.zeros(n)
    lib().ora_backEuler1D(n, *(_p(v) for v in arr[:6]), tmin, tmax, dt, _p(arr[6]), _p(arr[7]), _p(out))
    return out


def constants():
    ms, qs, g = np.zeros(LSP), np.zeros(LSP), np.zeros(LSP)
    tc = np.zeros(LSP - 1)
    lib().ora_constants(_p(ms), _p(qs), _p(g), _p(tc))
    return ms, qs, g, tc


# ---- state-level operations (in place on FluidState-like objects) --------------------

def _blocks(st):
    fv, av = st.fluidvars, st.fluidauxvars
    assert fv.flags.f_contiguous and av.flags.f_contiguous
    ng = fv.shape[0] * fv.shape[1] * fv.shape[2]
    base_f = fv.ctypes.data
    base_a = av.ctypes.data
    P = lambda base, k: ctypes.cast(base + 8 * k * ng, _D)
    return {
        "ns": P(base_f, 0), "vs1": P(base_f, LSP), "vs2": P(base_f, 2 * LSP),
        "vs3": P(base_f, 3 * LSP), "Ts": P(base_f, 4 * LSP),
        "rhovs1": P(base_a, 0), "rhoes": P(base_a, LSP),
    }


def sweep(grid, st, dim: int, which: str, dt: float):
    """sweep{dim}_allspec_{mass,momentum,energy} (multifluid.f90:49-126)."""
    frank, lsp, key = {"mass": (0, 6, "ns"), "momentum": (1, 6, "rhovs1"),
                       "energy": (0, 7, "rhoes")}[which]
    if dim == 1:
        frank = 0
    vsi = {1: st.vs1i, 2: st.vs2i, 3: st.vs3i}[dim]
    g = _GridHandle(grid)
    b = _blocks(st)
    lib().ora_sweep_allspec(g.ref, dim, b[key], _p(vsi), float(dt), frank, lsp)


def advec1D_MC_curv(f, v1i, dt: float, dx, dxi, ha1, ha2i, h1i):
    """advec.f90:384-435 on one line of lx cells: f, ha1 (lx+4, index -1..lx+2); v1i, ha2i,
    h1i (lx+1 faces); dx (lx+3, 0..lx+2); dxi (lx).  Returns the updated line (lx+4)."""
    f, v1i, dx, dxi, ha1, ha2i, h1i = (np.ascontiguousarray(a, dtype=np.float64)
                                       for a in (f, v1i, dx, dxi, ha1, ha2i, h1i))
    lx = f.size - 4
    assert v1i.size == lx + 1 and dx.size == lx + 3 and dxi.size == lx and ha1.size == lx + 4
    out = np.empty_like(f)
    lib().ora_advec1D_MC_curv(_p(f), _p(v1i), float(dt), _p(dx), _p(dxi), _p(ha1), _p(ha2i), _p(h1i), lx,
                              _p(out))
    return out


def set_global_boundaries(grid, st, lsp: int = LSP):
    g = _GridHandle(grid)
    b = _blocks(st)
    lib().ora_set_global_boundaries_allspec(g.ref, b["ns"], b["rhovs1"], b["vs1"], b["vs2"],
                                            b["vs3"], b["rhoes"], _p(st.vs1i), lsp)


def halo_fluidvars(grid, st):
    g = _GridHandle(grid)
    b = _blocks(st)
    lib().ora_halo_fluidvars(g.ref, b["ns"], b["rhovs1"], b["rhoes"], b["vs2"], b["vs3"])


def halo_allparams(grid, st):
    g = _GridHandle(grid)
    b = _blocks(st)
    lib().ora_halo_allparams(g.ref, b["ns"], b["rhovs1"], b["rhoes"])


def interface_vels(grid, st, lsp: int = LSP):
    g = _GridHandle(grid)
    b = _blocks(st)
    lib().ora_interface_vels_allspec(g.ref, b["vs1"], b["vs2"], b["vs3"], _p(st.vs1i),
                                     _p(st.vs2i), _p(st.vs3i), lsp)


def v12rhov1(grid, st):
    g = _GridHandle(grid); b = _blocks(st)
    lib().ora_v12rhov1(g.ref, b["ns"], b["vs1"], b["rhovs1"])


def T2rhoe(grid, st):
    g = _GridHandle(grid); b = _blocks(st)
    lib().ora_T2rhoe(g.ref, b["ns"], b["Ts"], b["rhoes"])


def rhov12v1(grid, st):
    g = _GridHandle(grid); b = _blocks(st)
    lib().ora_rhov12v1(g.ref, b["ns"], b["rhovs1"], b["vs1"])


def rhoe2T(grid, st):
    g = _GridHandle(grid); b = _blocks(st)
    lib().ora_rhoe2T(g.ref, b["ns"], b["rhoes"], b["Ts"])


def clean_param(grid, st, iparm: int):
    g = _GridHandle(grid); b = _blocks(st)
    key = {1: "ns", 2: "vs1", 3: "Ts"}[iparm]
    lib().ora_clean_param(g.ref, iparm, b[key])


def energy_diffusion(grid, st, dt: float, diffsolvetype: int = 2):
    g = _GridHandle(grid); b = _blocks(st)
    J1 = np.asfortranarray(st.electrovars[..., 3])
    rc = lib().ora_energy_diffusion(g.ref, b["ns"], b["Ts"], _p(J1), _p(st.nn), _p(st.Tn),
                                    float(dt), int(diffsolvetype), float(st.Teinf))
    if rc != 0:
        raise ValueError(f"ora_energy_diffusion failed: {rc}")


def dt_calc(grid, st, tcfl: float = 0.5):
    g = _GridHandle(grid); b = _blocks(st)
    gr = np.zeros(3 * LSP)
    dt = lib().ora_dt_calc(g.ref, float(tcfl), b["Ts"], b["vs1"], b["vs2"], b["vs3"], _p(gr))
    return float(dt), gr.reshape(3, LSP)


def dt_select(grid, st, t: float, tout: float, it: int, dtprev: float, tcfl: float = 0.5,
              tglowout: float = float("inf"), flagglow: int = 0) -> float:
    """The step's dt as dt_select chooses it (libgemini_mpi.f90:449-482, single rank): the CFL
    step clipped to the next GLOW / regular output, floored at 1e-6, throttled to at most
    twice the previous step from iteration 2 on."""
    g = _GridHandle(grid); b = _blocks(st)
    return float(lib().ora_dt_select(g.ref, float(tcfl), b["Ts"], b["vs1"], b["vs2"], b["vs3"], float(t),
                                     float(tout), float(tglowout), int(flagglow), int(it), float(dtprev)))


def fluid_adv(grid, st, dt: float, diffsolvetype: int = 2):
    """The advection + diffusion subset of fluid_adv (app/main.f90:280-355), in place."""
    g = _GridHandle(grid)
    J1 = np.asfortranarray(st.electrovars[..., 3])
    rc = lib().ora_fluid_adv(g.ref, _p(st.fluidvars), _p(st.fluidauxvars), _p(J1), _p(st.vs1i),
                             _p(st.vs2i), _p(st.vs3i), _p(st.nn), _p(st.Tn), float(dt),
                             float(st.Teinf), int(diffsolvetype))
    if rc != 0:
        raise ValueError(f"ora_fluid_adv failed: {rc}")


def fluid_adv_compression(grid, st, dt: float, diffsolvetype: int = 2):
    """fluid_adv with the compression sub-step (app/main.f90:320-338) between the
    post-advection clean_param(2) and rhoe2T, in place."""
    g = _GridHandle(grid)
    J1 = np.asfortranarray(st.electrovars[..., 3])
    rc = lib().ora_fluid_adv_compression(g.ref, _p(st.fluidvars), _p(st.fluidauxvars), _p(J1), _p(st.vs1i),
                                         _p(st.vs2i), _p(st.vs3i), _p(st.nn), _p(st.Tn), float(dt),
                                         float(st.Teinf), int(diffsolvetype))
    if rc != 0:
        raise ValueError(f"ora_fluid_adv_compression failed: {rc}")


def fluid_adv_full(grid, st, dt: float, nn, vn1, vn2, vn3, g1, Prionize, Qeionize, diffsolvetype: int = 2):
    """fluid_adv in full (app/main.f90:280-381, single rank), in place: the step with
    compression, then the source/loss sub-step with the given neutral state (nn: interior
    (lx1, lx2, lx3, >=6) O, N2, O2, H, N, NO; the diffusion reads the first three), gravity g1
    and ionization rates (Prionize (lx1, lx2, lx3, lsp-1), Qeionize (lx1, lx2, lx3)); Tn is st.Tn,
    E1 and J1 the state's electrovars."""
    g = _GridHandle(grid)
    E1 = np.asfortranarray(st.electrovars[..., 0])
    J1 = np.asfortranarray(st.electrovars[..., 3])
    alt = grid.alt[2:-2, 2:-2, 2:-2] if grid.alt.shape[0] == grid.lx1 + 4 else grid.alt
    arrs = [np.asfortranarray(a, dtype=np.float64) for a in (nn, vn1, vn2, vn3, st.Tn, alt, g1, Prionize, Qeionize)]
    rc = lib().ora_fluid_adv_full(g.ref, _p(st.fluidvars), _p(st.fluidauxvars), _p(E1), _p(J1), _p(st.vs1i),
                                  _p(st.vs2i), _p(st.vs3i), *[_p(a) for a in arrs], float(dt), float(st.Teinf),
                                  int(diffsolvetype))
    if rc != 0:
        raise ValueError(f"ora_fluid_adv_full failed: {rc}")


def vnricht_artvisc(grid, st):
    """Artificial viscosity Q (multifluid.f90:237-268): interior (lx1, lx2, lx3, lsp)."""
    g = _GridHandle(grid); b = _blocks(st)
    Q = np.zeros((grid.lx1, grid.lx2, grid.lx3, LSP), order="F")
    lib().ora_vnricht_artvisc(g.ref, b["ns"], b["vs1"], _p(Q))
    return Q


def rk2_global_boundary(grid, st):
    """Zero-order-hold velocity ghosts for the compression sub-step (sources_mpi.f90:68-111)."""
    g = _GridHandle(grid); b = _blocks(st)
    lib().ora_rk2_global_boundary_allspec(g.ref, b["vs1"], b["vs2"], b["vs3"])


def div3D(grid, f1, f2, f3):
    """div3D_curv_23 over the slab of grid indices 0..lx+1 (calculus/div.f90:110-200).
    f1, f2, f3: one species, ghosted (lx1+4, lx2+4, lx3+4); returns (lx1+2, lx2+2, lx3+2)."""
    g = _GridHandle(grid)
    fs = [np.asfortranarray(f, dtype=np.float64) for f in (f1, f2, f3)]
    out = np.zeros((grid.lx1 + 2, grid.lx2 + 2, grid.lx3 + 2), order="F")
    lib().ora_div3D(g.ref, _p(fs[0]), _p(fs[1]), _p(fs[2]), _p(out))
    return out


def compression(grid, st, dt: float, Q):
    """The compression energy update (multifluid.f90:274-302) of st's rhoes, in place."""
    g = _GridHandle(grid); b = _blocks(st)
    Qf = np.asfortranarray(Q, dtype=np.float64)
    lib().ora_compression(g.ref, float(dt), b["vs1"], b["vs2"], b["vs3"], _p(Qf), b["rhoes"])


def etd_uncoupled(f, P, L, dt: float):
    """ETD_uncoupled (calculus.in.f90:174-196) on same-shaped arrays."""
    f, P, L = (np.ascontiguousarray(a, dtype=np.float64).ravel() for a in (f, P, L))
    out = np.empty_like(f)
    lib().ora_etd_uncoupled(f.size, _p(f), _p(P), _p(L), float(dt), _p(out))
    return out


def srcs_continuity(grid, st, nn, vn1, vn2, vn3, Tn):
    """Production and loss rates of the continuity equations (sources.f90:18-276).  nn:
    interior (lx1, lx2, lx3, >=6) neutral densities O, N2, O2, H, N, NO; vn1..3, Tn:
    interior.  Returns (Pr, Lo), interior (lx1, lx2, lx3, lsp)."""
    g = _GridHandle(grid); b = _blocks(st)
    nn, vn1, vn2, vn3, Tn = (np.asfortranarray(a, dtype=np.float64) for a in (nn, vn1, vn2, vn3, Tn))
    Pr = np.zeros((grid.lx1, grid.lx2, grid.lx3, LSP), order="F")
    Lo = np.zeros_like(Pr)
    lib().ora_srcs_continuity(g.ref, _p(nn), _p(vn1), _p(vn2), _p(vn3), _p(Tn), b["ns"], b["vs1"], b["vs2"],
                              b["vs3"], b["Ts"], _p(Pr), _p(Lo))
    return Pr, Lo


def srcs_energy(grid, st, nn, vn1, vn2, vn3, Tn):
    """Production and loss rates of the energy equations (sources.f90:396-485, with
    collisions.f90:58-159).  nn: interior (lx1, lx2, lx3, >=4) neutral densities O, N2, O2,
    H; vn1..3, Tn: interior.  Returns (Pr, Lo), interior (lx1, lx2, lx3, lsp)."""
    g = _GridHandle(grid); b = _blocks(st)
    nn, vn1, vn2, vn3, Tn = (np.asfortranarray(a, dtype=np.float64) for a in (nn, vn1, vn2, vn3, Tn))
    Pr = np.zeros((grid.lx1, grid.lx2, grid.lx3, LSP), order="F")
    Lo = np.zeros_like(Pr)
    lib().ora_srcs_energy(g.ref, _p(nn), _p(vn1), _p(vn2), _p(vn3), _p(Tn), b["ns"], b["vs1"], b["vs2"],
                          b["vs3"], b["Ts"], _p(Pr), _p(Lo))
    return Pr, Lo


def srcs_momentum(grid, st, nn, vn1, Tn, E1, Q, g1):
    """Production and loss rates of the momentum equations (sources.f90:279-393), single
    rank.  nn: interior (lx1, lx2, lx3, >=4); vn1, Tn, g1: interior; E1: ghosted; Q: interior
    (lx1, lx2, lx3, lsp); the altitude filter reads grid.alt.  Returns (Pr, Lo)."""
    g = _GridHandle(grid); b = _blocks(st)
    alt = grid.alt
    if alt.shape[0] == grid.lx1 + 4:
        alt = alt[2:-2, 2:-2, 2:-2]
    nn, vn1, Tn, E1, Q, g1, alt = (np.asfortranarray(a, dtype=np.float64) for a in (nn, vn1, Tn, E1, Q, g1, alt))
    Pr = np.zeros((grid.lx1, grid.lx2, grid.lx3, LSP), order="F")
    Lo = np.zeros_like(Pr)
    lib().ora_srcs_momentum(g.ref, _p(nn), _p(vn1), _p(Tn), b["ns"], b["vs1"], b["vs2"], b["vs3"], b["Ts"], _p(E1),
                            _p(Q), _p(alt), _p(g1), _p(Pr), _p(Lo))
    return Pr, Lo


def mass_source_loss_solve(grid, st, dt: float, Pr, Lo, Prprecip):
    """multifluid.f90:532-549 with given rates (interior, (lx1, lx2, lx3, species)); returns Pr
    as updated by the routine."""
    g = _GridHandle(grid); b = _blocks(st)
    Pr = np.asfortranarray(Pr, dtype=np.float64).copy(order="F")
    Lo, Pp = (np.asfortranarray(a, dtype=np.float64) for a in (Lo, Prprecip))
    lib().ora_mass_source_loss_solve(g.ref, float(dt), _p(Pr), _p(Lo), _p(Pp), b["ns"])
    return Pr


def momentum_source_loss_solve(grid, st, dt: float, Pr, Lo):
    """multifluid.f90:500-528 with given rates (interior, (lx1, lx2, lx3, species))."""
    g = _GridHandle(grid); b = _blocks(st)
    Pr, Lo = (np.asfortranarray(a, dtype=np.float64) for a in (Pr, Lo))
    lib().ora_momentum_source_loss_solve(g.ref, float(dt), _p(Pr), _p(Lo), b["ns"], b["rhovs1"], b["vs1"])


def energy_source_loss_solve(grid, st, dt: float, Pr, Lo, Qeprecip):
    """multifluid.f90:474-495 with given rates; returns Pr as updated by the routine."""
    g = _GridHandle(grid); b = _blocks(st)
    Pr = np.asfortranarray(Pr, dtype=np.float64).copy(order="F")
    Lo, Qe = (np.asfortranarray(a, dtype=np.float64) for a in (Lo, Qeprecip))
    lib().ora_energy_source_loss_solve(g.ref, float(dt), _p(Pr), _p(Lo), _p(Qe), b["rhoes"], b["Ts"], b["ns"])
    return Pr


def run_steps(grid, st, nsteps: int, tcfl: float = 0.5, diffsolvetype: int = 2):
    """nsteps of (dt_calc -> fluid_adv); returns the dt sequence."""
    dts = []
    for _ in range(nsteps):
        dt, _ = dt_calc(grid, st, tcfl)
        fluid_adv(grid, st, dt, diffsolvetype)
        dts.append(dt)
    return dts
