"""Batched instances: many independent fluid-advance simulations stepped together.

The reference runs one simulation per MPI job; here n independent grids of uneven sizes
(Cartesian and dipole mixed) share the GPU.  One ``Batch.step()`` equals, for every
instance, ``dt_calc(tcfl)`` followed by ``fluid_adv`` on that instance, bit for bit: each
phase is one persistent launch over an (instance, block) work list, and the whole step is
replayed from a captured CUDA graph (``gem_batch_*`` in include/gem_fluid.h).

    insts = [(DeviceGrid(g), DeviceState.from_host(dg, st), FluidCfg(st.Teinf)), ...]
    b = Batch(insts)
    for _ in range(nsteps):
        b.step()
"""
from __future__ import annotations

import ctypes

from . import _lib
from .fluid import DeviceGrid, DeviceState, FluidCfg, _stream

USE_GRAPH, DIFF_BLOCKS, GRID_PCT = 0, 1, 2


class Batch:
    def __init__(self, instances, use_graph: bool = True):
        """instances: sequence of (DeviceGrid, DeviceState, FluidCfg)."""
        self.instances = list(instances)
        n = len(self.instances)
        if n < 1:
            raise ValueError("a batch needs at least one instance")
        VP = ctypes.c_void_p
        grids = (VP * n)(*[dg.handle.value for dg, _, _ in self.instances])
        works = (VP * n)(*[ds.work.value for _, ds, _ in self.instances])
        fv = (VP * n)(*[ds.fluidvars.data_ptr() for _, ds, _ in self.instances])
        fa = (VP * n)(*[ds.fluidauxvars.data_ptr() for _, ds, _ in self.instances])
        ev = (VP * n)(*[ds.electrovars.data_ptr() for _, ds, _ in self.instances])
        cfgs = (_lib.GemCfg * n)(*[cfg.c() for _, _, cfg in self.instances])
        h = VP()
        _lib.check(_lib.lib().gem_batch_create(n, grids, works, fv, fa, ev, cfgs, ctypes.byref(h)))
        self.handle = h
        if not use_graph:
            self.set_param(USE_GRAPH, 0)

    def __len__(self):
        return len(self.instances)

    def set_param(self, param: int, value: int) -> None:
        _lib.check(_lib.lib().gem_batch_set_param(self.handle, int(param), int(value)))

    def step(self, stream=None) -> None:
        _lib.check(_lib.lib().gem_batch_step(self.handle, _stream(stream)))

    def step_fixed_dt(self, dts, stream=None) -> None:
        """One step with prescribed per-instance time steps (dt_calc skipped)."""
        import numpy as np

        a = np.ascontiguousarray(np.asarray(dts, dtype=np.float64))
        if a.shape != (len(self),):
            raise ValueError(f"need {len(self)} time steps, got shape {a.shape}")
        self._dt_host = a  # the copy is asynchronous: keep the host array alive
        _lib.check(_lib.lib().gem_batch_step_fixed_dt(self.handle, a.ctypes.data_as(_lib._D), _stream(stream)))

    def dts(self):
        import numpy as np

        out = np.zeros(len(self), dtype=np.float64)
        _lib.check(_lib.lib().gem_batch_dts(self.handle, out.ctypes.data_as(_lib._D)))
        return out

    def info(self):
        launches = ctypes.c_int(0)
        items = ctypes.c_longlong(0)
        _lib.check(_lib.lib().gem_batch_info(self.handle, ctypes.byref(launches), ctypes.byref(items)))
        return launches.value, items.value

    def close(self) -> None:
        if getattr(self, "handle", None) is not None and self.handle.value:
            _lib.lib().gem_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 -- interpreter shutdown
            pass


def plain_step(dg: DeviceGrid, ds: DeviceState, cfg: FluidCfg, stream=None):
    """The sequential reference for one instance: dt_calc + fluid_adv on its own; returns
    the dt (1-element device tensor)."""
    from . import fluid as F

    dt = F.dt_calc(ds, cfg.tcfl, stream=stream)
    F.fluid_adv(cfg, ds, dt, stream=stream)
    return dt
