"""Shared test helpers: standard small grids/states and the parity metrics."""
from __future__ import annotations

import numpy as np

from gemini_b200 import grid as G
from gemini_b200 import state as S

LSP = 7
# signed fields are compared norm-wise per species (they cross zero); positive fields cell-wise
SIGNED_FLUID = set(range(LSP, 4 * LSP))  # vs1, vs2, vs3
SIGNED_AUX = set(range(0, LSP))           # rhovs1


def cases():
    """(name, grid, state kwargs) covering the grid types and boundary branches."""
    return [
        ("cart", G.cartesian_grid(20, 10, 8), dict(seed=1)),
        ("cart_inverted", G.cartesian_grid(18, 6, 5, inverted=True), dict(seed=2)),
        ("cart_periodic", G.cartesian_grid(16, 5, 7, flagper=1), dict(seed=3)),
        ("cart_2d", G.cartesian_grid(24, 9, 1), dict(seed=4)),
        ("dipole", G.dipole_grid(40, 8, 6), dict(seed=5, perturb=0.2)),
        ("dipole_nulls", G.dipole_grid(40, 8, 5, q_extent=0.5), dict(seed=6, perturb=0.2)),
        ("cart_J1", G.cartesian_grid(20, 7, 6), dict(seed=7, J1_amp=1e-5)),
    ]


def randomize_interface_vels(st, seed=0):
    rng = np.random.default_rng(seed)
    for a in (st.vs1i, st.vs2i, st.vs3i):
        a[...] = rng.uniform(-300, 300, a.shape)


def rel_err_block(a: np.ndarray, b: np.ndarray, signed: set) -> float:
    """Max relative difference over a 4-D block: cell-wise for positive variables,
    norm-wise (by the variable's max magnitude) for the signed ones."""
    worst = 0.0
    for v in range(a.shape[-1]):
        x, y = a[..., v], b[..., v]
        d = np.abs(x - y)
        if not np.isfinite(d).all():
            return float("inf")
        if v in signed:
            scale = max(np.max(np.abs(y)), 1e-300)
            worst = max(worst, float(np.max(d) / scale))
        else:
            den = np.maximum(np.abs(y), 1e-300)
            worst = max(worst, float(np.max(d / den)))
    return worst


def state_err(gpu, ref, aux_vars: int = 2 * LSP) -> dict:
    return {
        "fluidvars": rel_err_block(gpu.fluidvars, ref.fluidvars, SIGNED_FLUID),
        "fluidauxvars": rel_err_block(gpu.fluidauxvars[..., :aux_vars], ref.fluidauxvars[..., :aux_vars], SIGNED_AUX),
    }


def assert_identical(gpu, ref, what=""):
    """Bit-for-bit equality of the fluid and auxiliary blocks (NaN-free)."""
    for name in ("fluidvars", "fluidauxvars"):
        a, b = getattr(gpu, name), getattr(ref, name)
        if not np.array_equal(a, b):
            bad = np.argwhere(a != b)
            i = tuple(bad[0])
            raise AssertionError(f"{what}: {name} differs at {len(bad)} cells, first {i}: "
                                 f"gpu {a[i]!r} oracle {b[i]!r}")


def rate_inputs(g, seed):
    """A state and neutral inputs for the production/loss rates: drifts of up to 3 km/s (both
    branches of the Coulomb Phi), interior ion temperatures 150..40000 K (every piece of the
    reaction-rate fits), electrons 150..10000 K, neutral densities 1e10..1e16, E1 ghosted, Q and g1 interior."""
    rng = np.random.default_rng(seed)
    shp = (g.lx1, g.lx2, g.lx3)
    st = S.init_state(g, seed=seed, perturb=0.3)
    fv = st.fluidvars
    I = (slice(2, g.lx1 + 2), slice(2, g.lx2 + 2), slice(2, g.lx3 + 2))
    for k in (1, 2, 3):  # drifts large enough for the W >= 0.1 branch and high Teff fits
        fv[..., k * LSP:(k + 1) * LSP] = rng.uniform(-3000, 3000, fv[..., 0:LSP].shape)
    fv[I + (slice(4 * LSP, 5 * LSP),)] = rng.uniform(150, 40000, fv[I + (slice(0, LSP),)].shape)
    # electrons up to 10000 K: far above that the reference's N2 vibrational-loss fit overflows
    # exp (argument ~700 at 33000 K over a 200 K neutral gas)
    fv[I + (5 * LSP - 1,)] = rng.uniform(150, 10000, fv[I + (0,)].shape)
    nn = np.asfortranarray(np.stack([10 ** rng.uniform(10, 16, shp) for _ in range(7)], axis=-1))
    vn = [np.asfortranarray(rng.uniform(-100, 100, shp)) for _ in range(3)]
    Tn = np.asfortranarray(rng.uniform(200, 1500, shp))
    E1 = np.asfortranarray(rng.uniform(-1e-3, 1e-3, (g.lx1 + 4, g.lx2 + 4, g.lx3 + 4)))
    Q = np.asfortranarray(rng.uniform(0, 1e-12, shp + (LSP,)))
    g1 = np.asfortranarray(rng.uniform(-9.8, -8.0, shp))
    alt = g.alt[2:-2, 2:-2, 2:-2] if g.alt.shape[0] == g.lx1 + 4 else g.alt
    return st, nn, vn, Tn, E1, Q, g1, np.asfortranarray(alt, dtype=np.float64)


def harness_flags():
    """Extra g++ flags for the host builds of the device kernel bodies (the *_harness.cpp
    tests), e.g. "-fsanitize=address" to check their index arithmetic for out-of-bounds
    accesses; taken from GEMINI_HARNESS_CFLAGS."""
    import os
    return os.environ.get("GEMINI_HARNESS_CFLAGS", "").split()
