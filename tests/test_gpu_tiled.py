"""Parity of the tiled engine (FP64 and FP32 mixed precision) against the
CPU oracle, through the C ABI.

FP64 bar: relative L2 <= 1e-12 (fields E, B, J and particle momenta and
positions after full PIC steps).  FP32 mixed precision bar (stated):
relative L2 <= 2e-5 for fields and 1e-6 for momenta after one step from an
identical state, and charge conservation (Gauss-law residual drift) below
1e-5 relative over 20 steps.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from picsar_b200 import picsar as P
from picsar_b200.tiled import TiledConfig, TiledSim
from tests._cases import plasma, random_fields, rel_l2

pytestmark = pytest.mark.gpu

FIELDS = ("ex", "ey", "ez", "bx", "by", "bz")


def _pair(n, order, pusher, prec, st, cfg, fields=None, g=3):
    o = O.OracleSim(n, g, order=order, pusher=pusher)
    o.add_particles(st["x"], st["y"], st["z"], st["ux"], st["uy"], st["uz"], st["w"])
    t = TiledSim(n, order=order, pusher=pusher, precision=prec, config=cfg, track_ids=True)
    if fields is not None:
        for name, a in zip(FIELDS, fields):
            o.set_field(name, a)
            t.import_field(name, P.to_fortran(a), g)
    t.load_particles(st["x"], st["y"], st["z"], st["ux"], st["uy"], st["uz"], st["w"])
    return o, t


def _compare(o, t, g, ftol, ptol, fields=FIELDS + ("jx", "jy", "jz")):
    torch.cuda.synchronize()
    errs = {}
    for name in fields:
        a = t.export_field(name, g).cpu().numpy()
        errs[name] = rel_l2(a, o.get_field(name))
    ref = o.particles()
    got = {k: v.cpu().numpy() for k, v in t.particles().items()}
    assert np.array_equal(got["id"], ref["id"].astype(np.int64))
    for c in ("ux", "uy", "uz", "gaminv"):
        errs["p_" + c] = rel_l2(got[c], ref[c])
    # positions: compare the periodic displacement-insensitive difference
    for c, L in (("x", o.n[0]), ("y", o.n[1]), ("z", o.n[2])):
        dxp = (got[c] - ref[c] + L / 2) % L - L / 2
        errs["p_" + c] = float(np.linalg.norm(dxp) / np.linalg.norm(ref[c]))
    for k, v in errs.items():
        tol = ftol if not k.startswith("p_") else ptol
        assert v <= tol, (k, v, errs)
    return errs


@pytest.mark.parametrize("order", [1, 2, 3])
@pytest.mark.parametrize("pusher", [0, 1])
def test_tiled_fp64_parity(cuda, order, pusher):
    n, g = (16, 24, 16), 3
    st = plasma(n, 4, 0.05, seed=200 + order)
    fields = random_fields(n, g, seed=300 + order, amp=0.02)
    o, t = _pair(n, order, pusher, "fp64", st, TiledConfig(tile=(8, 8, 8), sort_interval=1),
                 fields)
    o.step(2)
    t.step(2, keep_j=True)
    _compare(o, t, g, 1e-12, 1e-12)
    assert t.error_flag() == 0


@pytest.mark.parametrize("order", [1, 2, 3])
def test_tiled_fp64_slow_path(cuda, order):
    """Window margin 0 and no re-sorting: fast particles leave their tile
    window and go through the global-memory gather/deposit path."""
    n, g = (16, 16, 16), 3
    st = plasma(n, 2, 0.4, seed=500 + order)
    o, t = _pair(n, order, 0, "fp64", st, TiledConfig(tile=(4, 4, 4), drift=0, sort_interval=0),
                 random_fields(n, g, seed=7, amp=0.02))
    o.step(3)
    t.step(3, keep_j=True)
    assert t.slow_path_count() > 0
    _compare(o, t, g, 1e-12, 1e-12)


@pytest.mark.parametrize("order", [1, 2, 3])
@pytest.mark.parametrize("pusher", [0, 1])
def test_tiled_fp32_one_step(cuda, order, pusher):
    n, g = (16, 16, 24), 3
    st = plasma(n, 8, 0.05, seed=600 + order)
    fields = random_fields(n, g, seed=700 + order, amp=0.02)
    o, t = _pair(n, order, pusher, "fp32", st, TiledConfig(tile=(8, 8, 8)), fields)
    o.step(1)
    t.step(1, keep_j=True)
    errs = _compare(o, t, g, 2e-5, 1e-6)
    assert errs["jx"] < 2e-5


@pytest.mark.parametrize("acc,tol", [(0, 2e-5), (1, 2e-4), (2, 2e-5)])
def test_tiled_fp32_accumulators(cuda, acc, tol):
    """The three FP32 current accumulators (FP32 atomics, int32 fixed point,
    64-bit fixed point in two int32 words) against the FP64 oracle."""
    n, g = (16, 16, 24), 3
    st = plasma(n, 8, 0.05, seed=650)
    fields = random_fields(n, g, seed=750, amp=0.02)
    o, t = _pair(n, 2, 0, "fp32", st, TiledConfig(tile=(8, 8, 8), acc=acc), fields)
    o.step(1)
    t.step(1, keep_j=True)
    _compare(o, t, g, tol, 1e-6)


@pytest.mark.parametrize("order,acc", [(1, 1), (2, 2), (3, 1), (3, 2)])
def test_tiled_fp32_drifted_tiles(cuda, order, acc):
    """Hot plasma stepped without re-sorting or re-layout: many particles
    change cells, so the particle kernel defers lanes whose bank class a
    lower lane of the warp holds and processes them in its second,
    class-bucketed pass.  Every particle must still be pushed and deposited
    exactly once: the state after several steps matches the oracle to the
    FP32 bars (a skipped or repeated particle would be off by a whole
    displacement)."""
    n, g = (16, 16, 24), 3
    st = plasma(n, 8, 0.15, seed=810 + order)
    fields = random_fields(n, g, seed=820 + order, amp=0.02)
    cfg = TiledConfig(tile=(8, 8, 8), acc=acc, sort_interval=0, relayout_interval=0)
    o, t = _pair(n, order, 0, "fp32", st, cfg, fields)
    o.step(4)
    t.step(4, keep_j=True)
    assert t.deferred_count() > 0
    _compare(o, t, g, 2e-4 if acc == 1 else 5e-5, 5e-6)
    assert t.error_flag() == 0


@pytest.mark.parametrize("order,acc", [(2, 1), (3, 2)])
def test_tiled_fp32_one_pass_equals_two_passes(cuda, order, acc):
    """The bank-class lane selection only reorders the particles' shared
    fixed-point updates, whose integer sums do not depend on order: the same
    drifted state stepped in one pass (select_lanes off) and in two passes
    agrees, and the one-pass kernel defers nothing.  Bar 1e-7 relative L2:
    the FP64 flush atomics may flip an FP32 rounding of E between the runs;
    one particle skipped or deposited twice would change J by ~1e-3."""
    n, g = (16, 16, 24), 3
    st = plasma(n, 8, 0.15, seed=830 + order)
    fields = random_fields(n, g, seed=840 + order, amp=0.02)
    sims = []
    for sel in (True, False):
        cfg = TiledConfig(tile=(8, 8, 8), acc=acc, sort_interval=0, relayout_interval=0,
                          select_lanes=sel)
        _, t = _pair(n, order, 0, "fp32", st, cfg, fields)
        t.step(4, keep_j=True)
        sims.append(t)
    torch.cuda.synchronize()
    two, one = sims
    assert two.deferred_count() > 0 and one.deferred_count() == 0
    for name in FIELDS + ("jx", "jy", "jz"):
        a, b = (s.export_field(name, g).cpu().numpy() for s in sims)
        assert rel_l2(b, a) <= 1e-7, name
    pa, pb = (s.particles() for s in sims)
    for c in ("x", "y", "z", "ux", "uy", "uz"):
        assert rel_l2(pb[c].cpu().numpy(), pa[c].cpu().numpy()) <= 1e-7, c


def _gauss_residual(t, g):
    n = t.n
    ex, ey, ez = (t.export_field(c, g).cpu().numpy() for c in ("ex", "ey", "ez"))
    sl = lambda a, di, dj, dk: a[g + di:g + di + n[0], g + dj:g + dj + n[1], g + dk:g + dk + n[2]]
    dive = (sl(ex, 0, 0, 0) - sl(ex, -1, 0, 0)) / t.d[0] + (sl(ey, 0, 0, 0) - sl(ey, 0, -1, 0)) / \
        t.d[1] + (sl(ez, 0, 0, 0) - sl(ez, 0, 0, -1)) / t.d[2]
    rho = t.rho.cpu().numpy().reshape(n[2], n[1], n[0]).transpose(2, 1, 0)
    return dive * t.eps0 - rho


@pytest.mark.parametrize("order", [1, 2, 3])
def test_tiled_fp32_charge_conservation(cuda, order):
    n, g = (16, 16, 16), 3
    st = plasma(n, 8, 0.05, seed=800 + order)
    t = TiledSim(n, order=order, precision="fp32", config=TiledConfig(tile=(8, 8, 8),
                                                                      sort_interval=5))
    t.load_particles(st["x"], st["y"], st["z"], st["ux"], st["uy"], st["uz"], st["w"])
    t.diagnostics()
    r0 = _gauss_residual(t, g)
    t.step(20)
    t.diagnostics()
    r1 = _gauss_residual(t, g)
    drift = np.linalg.norm(r1 - r0) / np.linalg.norm(r0)
    assert drift < 1e-5, drift
    assert t.error_flag() == 0


def test_tiled_diagnostics_match_oracle(cuda):
    n, g = (16, 16, 16), 3
    st = plasma(n, 4, 0.05, seed=900)
    fields = random_fields(n, g, seed=901, amp=0.02)
    o, t = _pair(n, 2, 0, "fp64", st, TiledConfig(tile=(8, 8, 8)), fields)
    o.step(1)
    t.step(1)
    do, dt = o.diags(), t.diagnostics()
    for k in ("kinetic", "ex", "ey", "ez", "bx", "by", "bz", "gauss_norm"):
        assert abs(dt[k] - do[k]) <= 1e-10 * max(abs(do[k]), 1e-30), (k, dt[k], do[k])


def test_golden_fixtures_fp64(cuda):
    """FP64 tiled engine against the committed golden fixtures (made by the
    oracle, tests/golden/make_golden.py), at 1e-12 relative L2."""
    from tests.golden import make_golden as MG
    fx = np.load(MG.PATH)
    for case in MG.CASES:
        tag = MG.tag(**case)
        n, g = case["n"], MG.G
        _, fields = MG.initial_state(case["n"], case["ppc"], case["sigma"], case["seed"])
        t = TiledSim(n, order=case["order"], pusher=case["pusher"], precision="fp64",
                     config=TiledConfig(tile=(8, 8, 8), sort_interval=1), track_ids=True)
        for name, a in zip(FIELDS, fields):
            t.import_field(name, P.to_fortran(a), g)
        init = [fx[f"{tag}/init_{c}"] for c in ("x", "y", "z", "ux", "uy", "uz", "w")]
        t.load_particles(*init)
        t.step(case["steps"], keep_j=True)
        torch.cuda.synchronize()
        for name in MG.FIELDS:
            err = rel_l2(t.export_field(name, g).cpu().numpy(), fx[f"{tag}/{name}"])
            assert err <= 1e-12, (tag, name, err)
        got = {k: v.cpu().numpy() for k, v in t.particles().items()}
        for c in ("ux", "uy", "uz", "gaminv"):
            err = rel_l2(got[c], fx[f"{tag}/{c}"])
            assert err <= 1e-12, (tag, c, err)
        for c, L in zip(("x", "y", "z"), n):
            ref = fx[f"{tag}/{c}"]
            dxp = (got[c] - ref + L / 2) % L - L / 2
            assert np.linalg.norm(dxp) / np.linalg.norm(ref) <= 1e-12, (tag, c)


@pytest.mark.parametrize("acc", [1, 2])
def test_carried_tile_bounds_match_prepass(cuda, acc):
    """The fixed-point bounds each tile carries to the next step equal what a
    pre-pass over the tile's particles finds: a job descriptor without
    tile_stats (pre-pass every step) gives the same state after 6 steps.
    The scales can differ only by FMA contraction in max |u|^2, so the states
    differ by the accumulator's quantisation: 1e-5 relative with one int32
    word (mode 1), 1e-6 with two (mode 2)."""
    tol = 1e-5 if acc == 1 else 1e-6
    n = (24, 16, 32)
    st = plasma(n, 4, 0.05, seed=31)
    fields = random_fields(n, 3, seed=7, amp=0.02)
    sims = []
    for carried in (True, False):
        t = TiledSim(n, order=3, precision="fp32",
                     config=TiledConfig(tile=(8, 8, 8), acc=acc, relayout_interval=2),
                     track_ids=True)
        for name, a in zip(FIELDS, fields):
            t.import_field(name, P.to_fortran(a), 3)
        if not carried:
            t.job.tile_stats = None
            t._push_job()
        t.load_particles(st["x"], st["y"], st["z"], st["ux"], st["uy"], st["uz"], st["w"])
        t.step(6, keep_j=True)
        sims.append(t)
    torch.cuda.synchronize()
    assert sims[0].tile_stats.view(-1, 4)[:, 3].min().item() == 1.0   # every tile carries
    for name in FIELDS + ("jx", "jy", "jz"):
        a, b = (s.export_field(name, 3).cpu().numpy() for s in sims)
        assert rel_l2(a, b) <= tol, name
    pa, pb = ({k: v.cpu().numpy() for k, v in s.particles().items()} for s in sims)
    for c in ("ux", "uy", "uz"):
        assert rel_l2(pa[c], pb[c]) <= tol, c
