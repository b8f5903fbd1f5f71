"""Grids for the fluid-advance hot path: the curvmesh fields the advection and diffusion
read, in the reference's Fortran layouts (column-major, x1 fastest).

The reference builds these once at set-up (``src/numerical/coord/meshobj.f90``; Cartesian
``meshobj_cart.f90:278-326`` with h=1, dipole ``meshobj_dipole.f90:115-231`` with
``calc_hq/calc_hp/calc_hphi_dip`` at 323-360).  Here they are generated on the host with
numpy from the same formulas and handed to the device once; nothing on the hot path
recomputes them.

Layouts (Fortran index ranges):
  x1, x2, x3             (-1:l+2)            cell centres incl. 2 ghosts per side
  dx1, dx2, dx3          (0:l+2)             backward differences  (meshobj.f90:356-389)
  x1i..x3i               (1:l+1)             interfaces
  dx1i..dx3i             (1:l)               interface differences
  h1, h2, h3             (-1:lx1+2,-1:lx2+2,-1:lx3+2)
  h1x1i, h2x1i, h3x1i    (1:lx1+1,1:lx2,1:lx3)
  h1x2i, h2x2i, h3x2i    (1:lx1,1:lx2+1,1:lx3)
  h1x3i, h2x3i, h3x3i    (1:lx1,1:lx2,1:lx3+1)
  alt                    (-1:lx1+2,-1:lx2+2,-1:lx3+2) altitude [m]
  nullpts                (1:lx1,1:lx2,1:lx3) alt < 80 km  (meshobj.f90:574-621)
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

RE = 6371.0e3  # phys_consts.in.f90:34

METRIC_NAMES = ("h1", "h2", "h3",
                "h1x1i", "h2x1i", "h3x1i",
                "h1x2i", "h2x2i", "h3x2i",
                "h1x3i", "h2x3i", "h3x3i")


@dataclass
class Grid:
    """Host copy of a curvilinear mesh (the fields of ``curvmesh`` the hot path reads)."""

    lx1: int
    lx2: int
    lx3: int
    gridflag: int
    flagper: int
    kind: str  # "cartesian" or "dipole"
    x1: np.ndarray
    x2: np.ndarray
    x3: np.ndarray
    dx1: np.ndarray
    dx1i: np.ndarray
    dx2: np.ndarray
    dx2i: np.ndarray
    dx3: np.ndarray
    dx3i: np.ndarray
    h1: np.ndarray
    h2: np.ndarray
    h3: np.ndarray
    h1x1i: np.ndarray
    h2x1i: np.ndarray
    h3x1i: np.ndarray
    h1x2i: np.ndarray
    h2x2i: np.ndarray
    h3x2i: np.ndarray
    h1x3i: np.ndarray
    h2x3i: np.ndarray
    h3x3i: np.ndarray
    alt: np.ndarray
    nullpts: np.ndarray
    meta: dict = field(default_factory=dict)

    @property
    def shape_ghosted(self):
        return (self.lx1 + 4, self.lx2 + 4, self.lx3 + 4)

    @property
    def ncells(self) -> int:
        return self.lx1 * self.lx2 * self.lx3

    @property
    def lnull(self) -> int:
        return int(self.nullpts.sum())

    @property
    def unit_metrics(self) -> bool:
        return bool(self.meta.get("unit_metrics", False))

    @property
    def x3_invariant_metrics(self) -> bool:
        return bool(self.meta.get("x3_invariant_metrics", False))


def coord_diffs(x: np.ndarray):
    """meshobj.f90:356-389 calc_coord_diffs for one dimension; x is (-1:l+2)."""
    lx = x.size - 4
    dx = x[1:] - x[:-1]                              # dx(0:l+2) = x(0:l+2) - x(-1:l+1)
    xi = 0.5 * (x[1:lx + 2] + x[2:lx + 3])           # xi(1:l+1) = 0.5*(x(0:l) + x(1:l+1))
    dxi = xi[1:] - xi[:-1]                           # dxi(1:l) = xi(2:l+1) - xi(1:l)
    return dx.copy(), xi.copy(), dxi.copy()


def _gridflag(alt: np.ndarray, lx1: int) -> int:
    """meshobj.f90:549-570 calc_gridflag (alt ghosted, Fortran order)."""
    a1 = alt[2, 2, 2]
    al = alt[lx1 + 1, 2, 2]
    a2 = alt[3, 2, 2]
    if abs(a1 - al) < 100e3:
        return 0
    if a1 > a2:
        return 1
    return 2


def _f(shape):
    return np.zeros(shape, dtype=np.float64, order="F")


def cartesian_grid(lx1: int, lx2: int, lx3: int, *, zmin: float = 80e3, zmax: float = 1000e3,
                   x2span: float = 600e3, x3span: float = 600e3, flagper: int = 0,
                   inverted: bool = False) -> Grid:
    """Cartesian mesh, h1=h2=h3=1 (meshobj_cart.f90:278-326).

    x1 is altitude; ``inverted`` puts the top at x1 index 1 (gridflag 1).  x2/x3 are
    uniform.  The ghost coordinates continue the uniform spacing.
    """
    def axis(lx, lo, hi):
        if lx == 1:
            d = (hi - lo) if hi > lo else 1.0
            return lo + d * (np.arange(-2, lx + 2, dtype=np.float64) + 0.5)
        d = (hi - lo) / (lx - 1)
        return lo + d * np.arange(-2, lx + 2, dtype=np.float64)

    z = axis(lx1, zmin, zmax)
    # the x1 coordinate always increases with the index; an inverted grid has the highest
    # altitude at x1 index 1 (GEMINI's gridflag 1)
    x1 = z
    alt1 = z[::-1].copy() if inverted else z
    x2 = axis(lx2, -x2span / 2, x2span / 2)
    x3 = axis(lx3, -x3span / 2, x3span / 2)
    dx1, _, dx1i = coord_diffs(x1)
    dx2, _, dx2i = coord_diffs(x2)
    dx3, _, dx3i = coord_diffs(x3)
    g = (lx1 + 4, lx2 + 4, lx3 + 4)
    ones = lambda s: np.ones(s, dtype=np.float64, order="F")
    alt = np.asfortranarray(np.broadcast_to(alt1[:, None, None], g).copy())
    nullpts = np.asfortranarray(alt[2:lx1 + 2, 2:lx2 + 2, 2:lx3 + 2] < 80e3)
    grid = Grid(lx1, lx2, lx3, _gridflag(alt, lx1), int(flagper), "cartesian",
                x1, x2, x3, dx1, dx1i, dx2, dx2i, dx3, dx3i,
                ones(g), ones(g), ones(g),
                ones((lx1 + 1, lx2, lx3)), ones((lx1 + 1, lx2, lx3)), ones((lx1 + 1, lx2, lx3)),
                ones((lx1, lx2 + 1, lx3)), ones((lx1, lx2 + 1, lx3)), ones((lx1, lx2 + 1, lx3)),
                ones((lx1, lx2, lx3 + 1)), ones((lx1, lx2, lx3 + 1)), ones((lx1, lx2, lx3 + 1)),
                alt, nullpts,
                meta={"unit_metrics": True, "x3_invariant_metrics": True,
                      "zmin": zmin, "zmax": zmax})
    return grid


def dipole_rtheta(q: np.ndarray, p: np.ndarray):
    """(q,p) -> (r,theta) for a centred dipole (dipole_fns.f90: rpoly / qr2theta).

    r solves q^2 (r/Re)^4 + (r/Re)/p - 1 = 0; the polynomial is increasing for r > 0 and
    non-negative at r = p*Re, so Newton from r = p*Re converges monotonically.
    """
    q = np.asarray(q, dtype=np.float64)
    p = np.asarray(p, dtype=np.float64)
    q, p = np.broadcast_arrays(q, p)
    r = p.copy()
    q2 = q * q
    for _ in range(200):
        f = q2 * r ** 4 + r / p - 1.0
        fp = 4.0 * q2 * r ** 3 + 1.0 / p
        step = f / fp
        r = r - step
        if np.max(np.abs(step) / r) < 1e-15:
            break
    theta = np.arccos(np.clip(q * r * r, -1.0, 1.0))
    return r * RE, theta


def _hq(r, th):
    return r ** 3 / RE ** 2 / np.sqrt(1 + 3 * np.cos(th) ** 2)


def _hp(r, th):
    return RE * np.sin(th) ** 3 / np.sqrt(1 + 3 * np.cos(th) ** 2)


def _hphi(r, th):
    return r * np.sin(th)


def dipole_grid(lx1: int, lx2: int, lx3: int, *, Lmin: float = 1.2, Lmax: float = 3.0,
                mlon_span_deg: float = 10.0, alt_end: float = 90e3,
                q_extent: float | None = None) -> Grid:
    """Closed dipole mesh in (q, p, phi) (meshobj_dipole.f90:115-231, 323-360).

    q spans [-qmax, qmax] with qmax chosen so that the lowest L-shell ends at ``alt_end``
    (both ends low: gridflag 0); p spans [Lmin, Lmax]; phi spans ``mlon_span_deg``.  The
    metric factors do not depend on phi.  ``q_extent`` overrides qmax (larger values put
    low-L cells below 80 km, i.e. null points).
    """
    rend = (RE + alt_end) / RE
    if q_extent is None:
        sin2 = rend / Lmin
        qmax = np.sqrt(max(1.0 - sin2, 0.0)) / rend ** 2
    else:
        qmax = float(q_extent)
    dq = 2 * qmax / (lx1 - 1) if lx1 > 1 else qmax
    x1 = -qmax + dq * np.arange(-2, lx1 + 2, dtype=np.float64)
    dp = (Lmax - Lmin) / (lx2 - 1) if lx2 > 1 else (Lmax - Lmin)
    x2 = Lmin + dp * np.arange(-2, lx2 + 2, dtype=np.float64)
    # ghost L-shells below the lowest one keep a positive spacing but stay above L=1.05
    dlo = min(dp, (Lmin - 1.05) / 2)
    x2[0], x2[1] = Lmin - 2 * dlo, Lmin - dlo
    span = np.deg2rad(mlon_span_deg)
    if lx3 > 1:
        dphi = span / (lx3 - 1)
        x3 = dphi * np.arange(-2, lx3 + 2, dtype=np.float64)
    else:
        x3 = span * (np.arange(-2, lx3 + 2, dtype=np.float64) + 0.5)

    dx1, x1i, dx1i = coord_diffs(x1)
    dx2, x2i, dx2i = coord_diffs(x2)
    dx3, _, dx3i = coord_diffs(x3)

    g = (lx1 + 4, lx2 + 4, lx3 + 4)
    Q, P = np.meshgrid(x1, x2, indexing="ij")
    r, th = dipole_rtheta(Q, P)
    def tile(a2):
        return np.asfortranarray(np.broadcast_to(a2[:, :, None], g).copy())
    h1 = tile(_hq(r, th))
    h2 = tile(_hp(r, th))
    h3 = tile(_hphi(r, th))
    alt = tile(r - RE)

    # q-interfaces: qint(1:lx1+1) at p(1:lx2)
    Qi, Pi = np.meshgrid(x1i, x2[2:lx2 + 2], indexing="ij")
    ri, thi = dipole_rtheta(Qi, Pi)
    def tile3(a2, n3):
        return np.asfortranarray(np.broadcast_to(a2[:, :, None], a2.shape + (n3,)).copy())
    h1x1i = tile3(_hq(ri, thi), lx3)
    h2x1i = tile3(_hp(ri, thi), lx3)
    h3x1i = tile3(_hphi(ri, thi), lx3)
    # p-interfaces: q(1:lx1), pint(1:lx2+1)
    Qp, Pp = np.meshgrid(x1[2:lx1 + 2], x2i, indexing="ij")
    rp, thp = dipole_rtheta(Qp, Pp)
    h1x2i = tile3(_hq(rp, thp), lx3)
    h2x2i = tile3(_hp(rp, thp), lx3)
    h3x2i = tile3(_hphi(rp, thp), lx3)
    # phi-interfaces: copies of the cell values, last one repeated (meshobj_dipole.f90:183-189)
    def phii(h):
        a = _f((lx1, lx2, lx3 + 1))
        a[:, :, :lx3] = h[2:lx1 + 2, 2:lx2 + 2, 2:lx3 + 2]
        a[:, :, lx3] = a[:, :, lx3 - 1]
        return a
    h1x3i, h2x3i, h3x3i = phii(h1), phii(h2), phii(h3)

    nullpts = np.asfortranarray(alt[2:lx1 + 2, 2:lx2 + 2, 2:lx3 + 2] < 80e3)
    return Grid(lx1, lx2, lx3, _gridflag(alt, lx1), 0, "dipole",
                x1, x2, x3, dx1, dx1i, dx2, dx2i, dx3, dx3i,
                h1, h2, h3, h1x1i, h2x1i, h3x1i, h1x2i, h2x2i, h3x2i, h1x3i, h2x3i, h3x3i,
                alt, nullpts,
                meta={"unit_metrics": False, "x3_invariant_metrics": True,
                      "Lmin": Lmin, "Lmax": Lmax, "qmax": qmax})
