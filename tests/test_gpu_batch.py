"""Batched instances (gem_batch_*) against the plain per-instance path, bit for bit.

One batched step must equal dt_calc + fluid_adv run on each instance on its own; the
instances are the standard parity cases (Cartesian, inverted, periodic, 2-D, dipole, dipole
with null cells, field-aligned current), whose plain path is itself checked against the
oracle in test_gpu_parity.py.
"""
import numpy as np
import pytest

from gemini_b200 import batch as BT
from gemini_b200 import fluid as F

from helpers import assert_identical, cases

pytestmark = pytest.mark.gpu


def _instances(extra=()):
    out = []
    for name, g, kw in list(cases()) + list(extra):
        from gemini_b200 import state as S

        st = S.init_state(g, **kw)
        out.append((name, g, st))
    return out


def _device(insts):
    dev = []
    for name, g, st in insts:
        dg = F.DeviceGrid(g)
        ds = F.DeviceState.from_host(dg, st.copy())
        dev.append((dg, ds, F.FluidCfg(st.Teinf)))
    return dev


def _run(nsteps, **batch_kw):
    import torch

    insts = _instances()
    plain = _device(insts)
    batched = _device(insts)
    last_dt = [None] * len(plain)
    for _ in range(nsteps):
        for k, (dg, ds, cfg) in enumerate(plain):
            last_dt[k] = BT.plain_step(dg, ds, cfg)
    b = BT.Batch(batched, **batch_kw)
    for _ in range(nsteps):
        b.step()
    torch.cuda.synchronize()
    return insts, plain, batched, b, [float(d.item()) for d in last_dt]


@pytest.mark.parametrize("use_graph", [True, False])
def test_batch_equals_plain_steps(use_graph):
    insts, plain, batched, b, plain_dt = _run(3, use_graph=use_graph)
    dts = b.dts()
    for (name, g, st), (_, dsp, _), (_, dsb, _), dtb, dtp in zip(insts, plain, batched, dts, plain_dt):
        assert_identical(dsb.to_host(st), dsp.to_host(st), what=f"batched {name}")
        assert dtb == dtp, name
    launches, items = b.info()
    # zero + finalize + per phase one launch per metric variant (+ diffusion row buckets)
    assert launches <= 2 + 4 * 2 + 5 + 2 * 5 and items > len(insts)


def test_batch_params_do_not_change_results():
    import torch

    insts = _instances()
    ref = _device(insts)
    b0 = BT.Batch(ref)
    for _ in range(2):
        b0.step()
    other = _device(insts)
    b1 = BT.Batch(other)
    b1.set_param(BT.DIFF_BLOCKS, 2)
    b1.set_param(BT.GRID_PCT, 30)
    for _ in range(2):
        b1.step()
    torch.cuda.synchronize()
    for (name, g, st), (_, d0, _), (_, d1, _) in zip(insts, ref, other):
        assert_identical(d1.to_host(st), d0.to_host(st), what=f"tuned batch {name}")
    np.testing.assert_array_equal(b0.dts(), b1.dts())


def test_batch_rejects_bad_params():
    from gemini_b200 import _lib

    insts = _instances()[:2]
    b = BT.Batch(_device(insts))
    with pytest.raises(_lib.GemError):
        b.set_param(BT.DIFF_BLOCKS, 9)
    with pytest.raises(_lib.GemError):
        b.set_param(99, 1)


def test_device_generated_uneven_batch_matches_plain():
    """Instances generated on the device (the bench's generator) with lx1 spread over
    several diffusion row buckets (rows per lane 2..17): batched == plain, finite."""
    import torch

    from gemini_b200 import workloads as WL

    specs = WL.batched_specs(6, seed=11, lx1=(40, 540), lx23=(3, 6))
    specs = specs + [WL.InstanceSpec("dipole", 530, 4, 3, 99), WL.InstanceSpec("cartesian", 260, 3, 4, 98)]

    def build():
        out = []
        for sp in specs:
            g = WL.make_grid(sp)
            dg = F.DeviceGrid(g)
            ds = WL.device_state(dg, g, sp.seed)
            out.append((dg, ds, F.FluidCfg(ds.Teinf)))
        return out

    batched, plain = build(), build()
    b = BT.Batch(batched)
    for _ in range(2):
        b.step()
        for dg, ds, cfg in plain:
            BT.plain_step(dg, ds, cfg)
    torch.cuda.synchronize()
    for (_, db, _), (_, dp, _) in zip(batched, plain):
        assert torch.equal(db.fluidvars, dp.fluidvars)
        assert torch.equal(db.fluidauxvars, dp.fluidauxvars)
        assert F.check_finite(db) == 0
    assert (b.dts() > 0).all()


def test_autotune_picks_and_caches(tmp_path, monkeypatch):
    from gemini_b200 import autotune as AT

    monkeypatch.setenv("GEMINI_B200_CACHE", str(tmp_path / "tune.json"))
    insts = _instances()[:3]
    b = BT.Batch(_device(insts))
    r = AT.tune(b, steps=1)
    assert not r["cached"] and len(r["trials"]) == len(AT.CANDIDATES)
    b2 = BT.Batch(_device(insts))
    r2 = AT.tune(b2, steps=1)
    assert r2["cached"] and r2["params"] == r["params"]
