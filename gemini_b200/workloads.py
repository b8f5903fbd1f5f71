"""Workload definitions: the batched instance mix, device-side state generation and the
sharding of instances across GPUs.

Batched mix (the uneven-instance workload): n instances with lx1 ~ U{64..512} and
lx2, lx3 ~ U{16..128}, Cartesian and dipole alternating (50/50), each with its own seed and
the profiles of ``state.init_state`` (Chapman densities over Dirichlet fractions, linear
temperatures, uniform velocities, optional lognormal perturbation).

``device_state`` draws those profiles with torch's generator directly in GPU memory, so
that tens of GB of instances are created in seconds; ``state.init_state`` (numpy) remains
the generator of the parity tests.  The two follow the same formulas but not the same
random stream.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import grid as G
from .state import LSP, NAUX, NELECTRO, NFLUID


@dataclass(frozen=True)
class InstanceSpec:
    kind: str  # "cartesian" | "dipole"
    lx1: int
    lx2: int
    lx3: int
    seed: int

    @property
    def cells(self) -> int:
        return self.lx1 * self.lx2 * self.lx3


def batched_specs(n: int = 64, seed: int = 2024, lx1=(64, 512), lx23=(16, 128)) -> list[InstanceSpec]:
    """The uneven-instance mix: per-instance sizes and seeds from one master seed."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        kind = "cartesian" if i % 2 == 0 else "dipole"
        out.append(InstanceSpec(kind, int(rng.integers(lx1[0], lx1[1] + 1)), int(rng.integers(lx23[0], lx23[1] + 1)),
                                int(rng.integers(lx23[0], lx23[1] + 1)), int(seed * 1000 + i)))
    return out


def make_grid(spec: InstanceSpec):
    if spec.kind == "cartesian":
        return G.cartesian_grid(spec.lx1, spec.lx2, spec.lx3)
    return G.dipole_grid(spec.lx1, spec.lx2, spec.lx3)


def shard(specs, world: int, rank: int) -> list[int]:
    """Indices of the instances rank `rank` of `world` runs: longest-processing-time-first
    over the cost cells x species (all ranks compute the same partition, no communication)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} of {world}")
    order = sorted(range(len(specs)), key=lambda i: (-specs[i].cells, i))
    load = [0] * world
    owner = [0] * len(specs)
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        owner[i] = r
        load[r] += specs[i].cells * LSP
    return [i for i in range(len(specs)) if owner[i] == rank]


def device_state(dgrid, grid, seed: int, perturb: float = 0.2, device="cuda"):
    """A DeviceState with init_state's profiles drawn on the GPU (torch generator)."""
    import torch

    from .fluid import DeviceState

    gen = torch.Generator(device=device)
    gen.manual_seed(int(seed))
    gs = grid.shape_ghosted
    shp = (gs[2], gs[1], gs[0])  # C-order view of the Fortran (x1 fastest) layout
    f64 = torch.float64
    z = torch.from_numpy(np.ascontiguousarray(grid.alt.transpose(2, 1, 0))).to(device)
    fluid = torch.zeros((NFLUID,) + shp, dtype=f64, device=device)
    aux = torch.zeros((NAUX,) + shp, dtype=f64, device=device)
    electro = torch.zeros((NELECTRO,) + shp, dtype=f64, device=device)
    w = torch.empty(LSP - 1, dtype=f64, device=device).exponential_(1.0, generator=gen)
    frac = w / w.sum()  # Dirichlet(1, ..., 1)
    zeta = (z - 300e3) / 50e3
    prof = torch.exp(1.0 - zeta - torch.exp(-zeta))
    T0 = 1000.0 + 2.0 * (z / 1e3)
    for s in range(LSP - 1):
        n = torch.clamp(frac[s] * 1e11 * prof, min=1e6)
        if perturb > 0:
            n = n * torch.exp(perturb * torch.randn(shp, dtype=f64, device=device, generator=gen))
        fluid[s] = n
    fluid[LSP - 1] = fluid[0:LSP - 1].sum(dim=0)
    for s in range(LSP):
        fluid[LSP + s].uniform_(-100.0, 100.0, generator=gen)
        fluid[2 * LSP + s].uniform_(-500.0, 500.0, generator=gen)
        fluid[3 * LSP + s].uniform_(-500.0, 500.0, generator=gen)
        T = T0
        if perturb > 0:
            T = T0 * torch.exp(perturb * torch.randn(shp, dtype=f64, device=device, generator=gen))
        fluid[4 * LSP + s] = torch.clamp(T, min=100.0)
    zi = grid.alt[2:grid.lx1 + 2, 2:grid.lx2 + 2, 2:grid.lx3 + 2]
    dz = zi - 100e3
    nn = np.zeros((grid.lx1, grid.lx2, grid.lx3, 3), dtype=np.float64, order="F")
    nn[..., 0] = 1e17 * np.exp(-dz / 50e3)
    nn[..., 1] = 1e18 * np.exp(-dz / 30e3)
    nn[..., 2] = 1e17 * np.exp(-dz / 25e3)
    Tn = np.asfortranarray(np.minimum(1000.0 + 2.0 * zi / 1e3, 1500.0))
    Teinf = 1000.0 + 2.0 * float(np.max(zi)) / 1e3
    ds = DeviceState(dgrid, fluid.reshape(-1), aux.reshape(-1), electro.reshape(-1), Teinf)
    ds.set_neutrals(nn, Tn)
    return ds
