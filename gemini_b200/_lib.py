"""ctypes binding of libgemini_b200.so (include/gem_fluid.h, include/gemini3d_fluid.h).

The library is built in tree (``python -m gemini_b200.build``); loading fails loudly when it
is missing -- there is no CPU fallback for the product path.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libgemini_b200.so")
INCLUDE_DIR = os.path.join(os.path.dirname(HERE), "include")

GEM_OK, GEM_EINVAL, GEM_ENONFINITE, GEM_ETIMEOUT, GEM_ECUDA, GEM_ENOMEM = range(6)

_D = ctypes.POINTER(ctypes.c_double)
_U8 = ctypes.POINTER(ctypes.c_ubyte)
_VP = ctypes.c_void_p


class GemGridDesc(ctypes.Structure):
    _fields_ = ([("lx1", ctypes.c_int), ("lx2", ctypes.c_int), ("lx3", ctypes.c_int),
                 ("gridflag", ctypes.c_int), ("flagper", ctypes.c_int)]
                + [(n, _D) for n in ("dx1", "dx1i", "dx2", "dx2i", "dx3", "dx3i",
                                     "h1", "h2", "h3", "h1x1i", "h2x1i", "h3x1i",
                                     "h1x2i", "h2x2i", "h3x2i", "h1x3i", "h2x3i", "h3x3i")]
                + [("nullpts", _U8), ("unit_metrics", ctypes.c_int)])


class GemCfg(ctypes.Structure):
    _fields_ = [("Teinf", ctypes.c_double), ("diffsolvetype", ctypes.c_int),
                ("tcfl", ctypes.c_double), ("flagglow", ctypes.c_int)]


class GemError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"gemini_b200 status {code}: {msg}")
        self.code = code


_lib = None

# (name, restype, argtypes) for the device-resident API
_SIGS = [
    ("gem_last_error", ctypes.c_char_p, []),
    ("gem_version", ctypes.c_int, []),
    ("gem_grid_create", ctypes.c_int, [ctypes.POINTER(GemGridDesc), ctypes.POINTER(_VP)]),
    ("gem_grid_destroy", ctypes.c_int, [_VP]),
    ("gem_grid_dims", ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int)] + [ctypes.POINTER(ctypes.c_int)] * 2),
    ("gem_work_create", ctypes.c_int, [_VP, ctypes.POINTER(_VP)]),
    ("gem_work_destroy", ctypes.c_int, [_VP]),
    ("gem_work_set_neutrals", ctypes.c_int, [_VP, _VP, _VP]),
    ("gem_work_interface_vels", ctypes.c_int, [_VP, ctypes.c_int, _VP, ctypes.c_int]),
    ("gem_work_array", _VP, [_VP, ctypes.c_int]),
    ("gem_work_dt", _VP, [_VP]),
    ("gem_work_set_top_temperature", ctypes.c_int, [_VP, _VP, ctypes.c_int]),
    ("gem_v12rhov1_dev", ctypes.c_int, [_VP, _VP, _VP, _VP]),
    ("gem_T2rhoe_dev", ctypes.c_int, [_VP, _VP, _VP, _VP]),
    ("gem_rhov12v1_dev", ctypes.c_int, [_VP, _VP, _VP, _VP]),
    ("gem_rhoe2T_dev", ctypes.c_int, [_VP, _VP, _VP, _VP]),
    ("gem_set_global_boundaries_allspec_dev", ctypes.c_int, [_VP, _VP, _VP, _VP, ctypes.c_int, _VP]),
    ("gem_halo_fluidvars_dev", ctypes.c_int, [_VP, _VP, _VP, _VP]),
    ("gem_halo_allparams_dev", ctypes.c_int, [_VP, _VP, _VP, _VP]),
    ("gem_interface_vels_allspec_dev", ctypes.c_int, [_VP, _VP, _VP, ctypes.c_int, _VP]),
    ("gem_sweep_allspec_dev", ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, _VP, _VP, _VP, _VP, _VP]),
    ("gem_clean_param_dev", ctypes.c_int, [_VP, ctypes.c_int, _VP, _VP]),
    ("gem_energy_diffusion_dev", ctypes.c_int, [ctypes.POINTER(GemCfg), _VP, _VP, _VP, _VP, _VP, _VP]),
    ("gem_dt_calc_dev", ctypes.c_int, [_VP, ctypes.c_double, _VP, _VP, _VP, _VP]),
    ("gem_maxcfl_dev", ctypes.c_int, [_VP, _VP, _VP, _VP, _VP, _VP]),
    ("gem_dt_calc_noalloc_dev", ctypes.c_int, [_VP, ctypes.c_double, _VP, _VP, _VP]),
    ("gem_sweep_field_dev", ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, ctypes.c_int, _VP, _VP, _VP, _VP]),
    ("gem_sweep_field_vjp_dev", ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, ctypes.c_int] + [_VP] * 7),
    ("gem_diffusion_vjp_dev", ctypes.c_int, [ctypes.POINTER(GemCfg)] + [_VP] * 11),
    ("gem_step_adjoint_create", ctypes.c_int, [_VP, ctypes.POINTER(_VP)]),
    ("gem_step_adjoint_destroy", ctypes.c_int, [_VP]),
    ("gem_step_vjp_dev", ctypes.c_int, [ctypes.POINTER(GemCfg)] + [_VP] * 24),
    ("gem_step_vjp_replay_dev", ctypes.c_int, [ctypes.POINTER(GemCfg)] + [_VP] * 12),
    ("gem_step_vjp_backward_dev", ctypes.c_int, [ctypes.POINTER(GemCfg)] + [_VP] * 22),
    ("gem_step_vjp_finish_dev", ctypes.c_int, [ctypes.POINTER(GemCfg)] + [_VP] * 10),
    ("gem_vnricht_artvisc_dev", ctypes.c_int, [_VP, _VP, _VP, _VP]),
    ("gem_rk2_global_boundary_allspec_dev", ctypes.c_int, [_VP, _VP, _VP]),
    ("gem_compression_dev", ctypes.c_int, [_VP, _VP, _VP, _VP, _VP, _VP]),
    ("gem_energy_source_loss_solve_dev", ctypes.c_int, [_VP] * 8),
    ("gem_momentum_source_loss_solve_dev", ctypes.c_int, [_VP] * 7),
    ("gem_mass_source_loss_solve_dev", ctypes.c_int, [_VP] * 7),
    ("gem_srcs_continuity_dev", ctypes.c_int, [_VP] * 10),
    ("gem_srcs_energy_dev", ctypes.c_int, [_VP] * 10),
    ("gem_srcs_momentum_dev", ctypes.c_int, [_VP] * 12),
    ("gem_fluid_adv_compression_dev", ctypes.c_int, [ctypes.POINTER(GemCfg)] + [_VP] * 7),
    ("gem_source_loss_allparams_dev", ctypes.c_int, [_VP] * 11),
    ("gem_fluid_adv_full_scratch_doubles", ctypes.c_longlong, [_VP]),
    ("gem_fluid_adv_full_dev", ctypes.c_int, [ctypes.POINTER(GemCfg)] + [_VP] * 9),
    ("gem_work_set_sources", ctypes.c_int, [_VP, _VP]),
    ("gem_work_prepare", ctypes.c_int, [_VP, _VP]),
    ("gem_work_substep_buffers", ctypes.c_int, [_VP] * 5),
    ("gem_dt_select_dev", ctypes.c_int, [ctypes.POINTER(GemCfg)] + [_VP] * 6),
    ("gem_clock_advance_dev", ctypes.c_int, [_VP] * 3),
    ("gem_fluid_adv_dev", ctypes.c_int, [ctypes.POINTER(GemCfg), _VP, _VP, _VP, _VP, _VP, _VP, _VP]),
    ("gem_fluid_adv_host", ctypes.c_int, [ctypes.POINTER(GemCfg), _VP, _VP, _VP, _VP, _VP, _D, _VP]),
    ("gem_check_finite", ctypes.c_int, [_VP, _VP, _VP, ctypes.POINTER(ctypes.c_longlong), _VP]),
    ("gem_work_phase_timing", ctypes.c_int, [_VP, ctypes.c_int]),
    ("gem_work_phase_times", ctypes.c_int, [_VP, _D, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                            ctypes.POINTER(ctypes.c_int)]),
    ("gem_batch_create", ctypes.c_int, [ctypes.c_int, _VP, _VP, _VP, _VP, _VP, _VP, ctypes.POINTER(_VP)]),
    ("gem_batch_destroy", ctypes.c_int, [_VP]),
    ("gem_batch_size", ctypes.c_int, [_VP]),
    ("gem_batch_set_param", ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int]),
    ("gem_batch_step", ctypes.c_int, [_VP, _VP]),
    ("gem_batch_step_fixed_dt", ctypes.c_int, [_VP, _D, _VP]),
    ("gem_batch_dts", ctypes.c_int, [_VP, _D]),
    ("gem_batch_info", ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_longlong)]),
    ("gem_capi_bind_grid", None, [_VP]),
    ("gem_capi_set_error_mode", None, [ctypes.c_int]),
    ("gem_capi_last_status", ctypes.c_int, []),
]


def lib():
    """Load libgemini_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m gemini_b200.build` "
                              "(the fluid advance has no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, res, args in _SIGS:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != GEM_OK:
        raise GemError(rc, lib().gem_last_error().decode(errors="replace"))


def header_symbols() -> list[str]:
    """Every function name declared in include/*.h (for the export check)."""
    import re
    names = []
    for fn in sorted(os.listdir(INCLUDE_DIR)):
        if not fn.endswith(".h"):
            continue
        txt = open(os.path.join(INCLUDE_DIR, fn)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for m in re.finditer(r"^\s*(?:extern\s+)?[A-Za-z_][\w\s\*]*?\b([A-Za-z_]\w*)\s*\(", txt, flags=re.M):
            name = m.group(1)
            if name not in ("if", "return", "sizeof") and not name.isupper():
                names.append(name)
    return sorted(set(names))
