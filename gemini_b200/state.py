"""Seeded synthetic fluid states in the reference's memory-block layout.

Block layout (libgemini.f90:401-417, 462-519; Fortran order, x1 fastest):
  fluidvars    (-1:lx1+2,-1:lx2+2,-1:lx3+2, 5*lsp)   ns | vs1 | vs2 | vs3 | Ts
  fluidauxvars (-1:lx1+2,-1:lx2+2,-1:lx3+2, 2*lsp+9) rhovs1 | rhoes | 9 MHD scalars
  electrovars  (-1:lx1+2,-1:lx2+2,-1:lx3+2, 7)       E1 E2 E3 J1 J2 J3 Phi
  vs1i (lx1+1,lx2,lx3,lsp), vs2i (lx1,lx2+1,lx3,lsp), vs3i (lx1,lx2,lx3+1,lsp)
  nn (lx1,lx2,lx3,3) = n(O), n(N2), n(O2);  Tn (lx1,lx2,lx3)

The profiles are the synthetic stand-ins for the reference's input files (the MSIS
neutral atmosphere and the HDF5 initial conditions are outside the hot path):
  n_s = f_s * 1e11 * exp(1 - zeta - exp(-zeta)) m^-3, zeta = (z - 300 km)/50 km,
        f ~ Dirichlet(1,...,1) over the 6 ions, floor 1e6; electrons = sum of ions
  T_s = 1000 + 2 z[km] K; v1 ~ U(-100,100), v2, v3 ~ U(-500,500) m/s
  optional seeded multiplicative lognormal perturbation of n and T
  n(O), n(N2), n(O2): exponential with 50/30/25 km scale heights above 100 km
  Tn = min(1000 + 2 z[km], 1500) (equal to Ti at the bottom); J1 = 0 unless asked.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .grid import Grid

LSP = 7
NFLUID = 5 * LSP
NAUX = 2 * LSP + 9
NELECTRO = 7

# phys_consts.in.f90:24-53 (the same constants as the kernels)
KB = 1.38064852e-23
ELCHRG = 1.60217662e-19
AMU = 1.660539040e-27
MS = np.array([16.0, 30.0, 28.0, 32.0, 14.0, 1.0, 5.485799090e-4]) * AMU
QS = np.array([1, 1, 1, 1, 1, 1, -1], dtype=np.float64) * ELCHRG
GAMMAS = np.array([5.0 / 3, 7.0 / 5, 7.0 / 5, 7.0 / 5, 5.0 / 3, 5.0 / 3, 5.0 / 3])


@dataclass
class FluidState:
    """Host copy of the state blocks and the per-run neutral inputs."""

    fluidvars: np.ndarray
    fluidauxvars: np.ndarray
    electrovars: np.ndarray
    vs1i: np.ndarray
    vs2i: np.ndarray
    vs3i: np.ndarray
    nn: np.ndarray
    Tn: np.ndarray
    Teinf: float

    def copy(self) -> "FluidState":
        return FluidState(self.fluidvars.copy(order="F"), self.fluidauxvars.copy(order="F"),
                          self.electrovars.copy(order="F"), self.vs1i.copy(order="F"),
                          self.vs2i.copy(order="F"), self.vs3i.copy(order="F"),
                          self.nn.copy(order="F"), self.Tn.copy(order="F"), self.Teinf)

    # views into the blocks (fluidvar_pointers / fluidauxvar_pointers / electrovar_pointers)
    @property
    def ns(self):
        return self.fluidvars[..., 0:LSP]

    @property
    def vs1(self):
        return self.fluidvars[..., LSP:2 * LSP]

    @property
    def vs2(self):
        return self.fluidvars[..., 2 * LSP:3 * LSP]

    @property
    def vs3(self):
        return self.fluidvars[..., 3 * LSP:4 * LSP]

    @property
    def Ts(self):
        return self.fluidvars[..., 4 * LSP:5 * LSP]

    @property
    def rhovs1(self):
        return self.fluidauxvars[..., 0:LSP]

    @property
    def rhoes(self):
        return self.fluidauxvars[..., LSP:2 * LSP]

    @property
    def J1(self):
        return self.electrovars[..., 3]


def _chapman(z):
    zeta = (z - 300e3) / 50e3
    return np.exp(1.0 - zeta - np.exp(-zeta))


def init_state(grid: Grid, seed: int = 0, *, perturb: float = 0.0, J1_amp: float = 0.0,
               vscale: float = 1.0) -> FluidState:
    """Seeded synthetic state for ``grid`` (profiles in the module docstring).

    ``perturb`` is the standard deviation of the multiplicative lognormal perturbation of
    the densities and temperatures (0.2 for the +-20 % dipole workload).  ``J1_amp`` > 0
    draws J1 ~ U(-J1_amp, J1_amp) A/m^2, which makes the electron thermoelectric term B
    non-zero.
    """
    rng = np.random.default_rng(seed)
    gs = grid.shape_ghosted
    z = grid.alt
    f = rng.dirichlet(np.ones(LSP - 1))
    fluid = np.zeros(gs + (NFLUID,), dtype=np.float64, order="F")
    aux = np.zeros(gs + (NAUX,), dtype=np.float64, order="F")
    electro = np.zeros(gs + (NELECTRO,), dtype=np.float64, order="F")
    prof = _chapman(z)
    T0 = 1000.0 + 2.0 * (z / 1e3)
    for s in range(LSP - 1):
        n = np.maximum(f[s] * 1e11 * prof, 1e6)
        if perturb > 0:
            n = n * np.exp(perturb * rng.standard_normal(gs))
        fluid[..., s] = n
    fluid[..., LSP - 1] = fluid[..., 0:LSP - 1].sum(axis=-1)
    for s in range(LSP):
        fluid[..., LSP + s] = vscale * rng.uniform(-100.0, 100.0, gs)
        fluid[..., 2 * LSP + s] = vscale * rng.uniform(-500.0, 500.0, gs)
        fluid[..., 3 * LSP + s] = vscale * rng.uniform(-500.0, 500.0, gs)
        T = T0.copy()
        if perturb > 0:
            T = T * np.exp(perturb * rng.standard_normal(gs))
        fluid[..., 4 * LSP + s] = np.maximum(T, 100.0)
    if J1_amp > 0:
        electro[..., 3] = rng.uniform(-J1_amp, J1_amp, gs)
    zi = z[2:grid.lx1 + 2, 2:grid.lx2 + 2, 2:grid.lx3 + 2]
    dz = (zi - 100e3)
    nn = np.zeros((grid.lx1, grid.lx2, grid.lx3, 3), dtype=np.float64, order="F")
    nn[..., 0] = 1e17 * np.exp(-dz / 50e3)
    nn[..., 1] = 1e18 * np.exp(-dz / 30e3)
    nn[..., 2] = 1e17 * np.exp(-dz / 25e3)
    Tn = np.asfortranarray(np.minimum(1000.0 + 2.0 * zi / 1e3, 1500.0))
    vs1i = np.zeros((grid.lx1 + 1, grid.lx2, grid.lx3, LSP), order="F")
    vs2i = np.zeros((grid.lx1, grid.lx2 + 1, grid.lx3, LSP), order="F")
    vs3i = np.zeros((grid.lx1, grid.lx2, grid.lx3 + 1, LSP), order="F")
    ztop = float(np.max(zi))
    Teinf = 1000.0 + 2.0 * ztop / 1e3
    return FluidState(fluid, aux, electro, vs1i, vs2i, vs3i, nn, Tn, Teinf)
