"""Parity of the cell-grouped particle kernel (accumulator mode 4: FP32,
int32 fixed-point current, shape orders 1 and 3) against the CPU oracle,
through the C ABI.

The kernel sorts each tile's particles by cell every step and computes a
pair of particles of a cell per thread; its bars are those of the int32
fixed-point accumulator (mode 1): relative L2 <= 2e-4 for E, B and J (the
J quantisation of one int32 word) and 1e-6 for momenta after one step, and
a Gauss-law residual drift below 1e-5 over 20 steps.  Cases: thermal
plasma (most cells with one or two groups), hot plasma stepped without
re-sorting (cell changes, particles outside the window), dense cells
(hundreds of groups per cell), partial tiles and an empty job.
"""
import numpy as np
import pytest
import torch

from tests._cases import plasma, random_fields, rel_l2
from tests.test_gpu_tiled import FIELDS, _compare, _gauss_residual, _pair
from picsar_b200.tiled import TiledConfig, TiledSim

pytestmark = pytest.mark.gpu


def _cfg(**kw):
    return TiledConfig(tile=(8, 8, 8), drift=1, acc=4, **kw)


@pytest.mark.parametrize("order", [1, 3])
@pytest.mark.parametrize("pusher", [0, 1])
def test_cell_groups_one_step(cuda, order, pusher):
    n, g = (16, 16, 24), 3
    st = plasma(n, 8, 0.05, seed=1600 + order)
    fields = random_fields(n, g, seed=1700 + order, amp=0.02)
    o, t = _pair(n, order, pusher, "fp32", st, _cfg(), fields)
    o.step(1)
    t.step(1, keep_j=True)
    _compare(o, t, g, 2e-4, 1e-6)
    assert t.error_flag() == 0


@pytest.mark.parametrize("order", [1, 3])
def test_cell_groups_agree_with_one_particle_per_thread(cuda, order):
    """Mode 4 and the one-particle-per-thread kernel with the same int32
    accumulator (mode 1) take the same state to the same place: the gathers
    are the same sums up to FMA contraction, the deposits differ by one
    rounding per term (an FMA onto the fixed-point grid instead of a rounded
    product), so the states agree to a few quanta of the accumulator."""
    n, g = (16, 24, 16), 3
    st = plasma(n, 8, 0.05, seed=1650 + order)
    fields = random_fields(n, g, seed=1750 + order, amp=0.02)
    sims = []
    for acc in (1, 4):
        _, t = _pair(n, order, 0, "fp32", st, TiledConfig(tile=(8, 8, 8), drift=1, acc=acc),
                     fields)
        t.step(3, keep_j=True)
        sims.append(t)
    torch.cuda.synchronize()
    for name in FIELDS + ("jx", "jy", "jz"):
        a, b = (s.export_field(name, g).cpu().numpy() for s in sims)
        assert rel_l2(b, a) <= 1e-4, name
    pa, pb = (s.particles() for s in sims)
    for c in ("ux", "uy", "uz"):
        assert rel_l2(pb[c].cpu().numpy(), pa[c].cpu().numpy()) <= 1e-6, c


@pytest.mark.parametrize("order", [1, 3])
def test_cell_groups_drifted_and_outside_window(cuda, order):
    """Hot plasma stepped without re-sorting: particles change cells every
    step (node-change queue) and some leave the tile window (global path).
    Every particle must be pushed and deposited exactly once."""
    n, g = (16, 16, 24), 3
    st = plasma(n, 8, 0.3, seed=1810 + order)
    fields = random_fields(n, g, seed=1820 + order, amp=0.02)
    o, t = _pair(n, order, 0, "fp32", st, _cfg(sort_interval=0, relayout_interval=0), fields)
    o.step(5)
    t.step(5, keep_j=True)
    assert t.slow_path_count() > 0
    _compare(o, t, g, 3e-4, 5e-6)
    assert t.error_flag() == 0


def _errors(o, t, g):
    torch.cuda.synchronize()
    errs = {name: rel_l2(t.export_field(name, g).cpu().numpy(), o.get_field(name))
            for name in FIELDS + ("jx", "jy", "jz")}
    ref, got = o.particles(), {k: v.cpu().numpy() for k, v in t.particles().items()}
    for c in ("ux", "uy", "uz"):
        errs["p_" + c] = rel_l2(got[c], ref[c])
    return errs


@pytest.mark.parametrize("order", [1, 3])
def test_cell_groups_dense_cells(cuda, order):
    """Thousands of particles in two cells: hundreds of groups per cell,
    beyond the first levels of their bank class.  The fixed-point scale of
    such a tile is set by its 1500 particles per cell, so one int32 word
    resolves J to only ~1e-2 here: mode 4 must do as well as mode 1 (the
    same accumulator with one particle per thread) against the oracle."""
    n, g = (16, 16, 16), 3
    rng = np.random.default_rng(1900 + order)
    m = 3000
    st = {"x": 3.0 + 0.999 * rng.random(m),
          "y": np.where(rng.random(m) < 0.5, 5.0, 12.0) + 0.999 * rng.random(m),
          "z": 9.0 + 0.999 * rng.random(m), "w": 0.01 + 0.01 * rng.random(m)}
    for c in ("ux", "uy", "uz"):
        st[c] = 0.02 * rng.standard_normal(m)
    fields = random_fields(n, g, seed=1950 + order, amp=0.02)
    errs = {}
    for acc in (1, 4):
        o, t = _pair(n, order, 0, "fp32", st, TiledConfig(tile=(8, 8, 8), drift=1, acc=acc),
                     fields)
        o.step(2)
        t.step(2, keep_j=True)
        errs[acc] = _errors(o, t, g)
        assert t.error_flag() == 0
    for k, e4 in errs[4].items():
        e1 = errs[1][k]
        bar = 1e-3 if k.startswith("p_") else 2e-2
        assert e4 <= bar and e1 <= bar, (k, e4, e1)
        assert e4 <= 1.5 * e1 + (1e-7 if k.startswith("p_") else 2e-5), (k, e4, e1)


@pytest.mark.parametrize("order", [1, 3])
def test_cell_groups_crowded_tile(cuda, order):
    """7000 particles in one 8^3 tile (14 per cell): more than the 20 per
    thread whose cell and rank the kernel keeps in registers, so the rest go
    through the global scratch between count and placement.  Two steps
    against the oracle, to the int32 accumulator's resolution: mode 4 as
    close as mode 1."""
    n, g = (16, 16, 16), 3
    rng = np.random.default_rng(2300 + order)
    m = 7000
    st = {c: 8.0 * rng.random(m) for c in ("x", "y", "z")}
    for c in ("ux", "uy", "uz"):
        st[c] = 0.05 * rng.standard_normal(m)
    st["w"] = np.full(m, 1.0 / 14.0)
    fields = random_fields(n, g, seed=2350 + order, amp=0.02)
    errs = {}
    for acc in (1, 4):
        o, t = _pair(n, order, 0, "fp32", st, TiledConfig(tile=(8, 8, 8), drift=1, acc=acc),
                     fields)
        o.step(2)
        t.step(2, keep_j=True)
        errs[acc] = _errors(o, t, g)
        assert t.error_flag() == 0
    for k, e4 in errs[4].items():
        e1 = errs[1][k]
        assert e4 <= (1e-5 if k.startswith("p_") else 1e-3), (k, e4, e1)
        assert e4 <= 1.5 * e1 + (1e-7 if k.startswith("p_") else 2e-5), (k, e4, e1)


@pytest.mark.parametrize("order", [1, 3])
def test_cell_groups_partial_tiles(cuda, order):
    """Grid extents that are not multiples of the tile edge (partial tiles,
    periodic wrap inside a window), particles on cell faces and just below
    the periodic edge, Vay pusher.  The edge particles sit 2^-10 below it,
    a position FP32 offsets hold exactly: at order 1 the staggered gather is
    the order-0 shape, discontinuous at faces, so a particle closer to the
    face than FP32 resolves would read the next cell's E."""
    n, g = (13, 20, 11), 3
    st = plasma(n, 8, 0.05, seed=2000 + order)
    st["x"][:50] = np.floor(st["x"][:50])
    st["z"][50:100] = np.float64(n[2]) - 2.0 ** -10
    fields = random_fields(n, g, seed=2100 + order, amp=0.02)
    o, t = _pair(n, order, 1, "fp32", st, _cfg(), fields)
    o.step(3)
    t.step(3, keep_j=True)
    _compare(o, t, g, 2e-4, 4e-6)


def test_cell_groups_no_particles(cuda):
    t = TiledSim((16, 16, 16), order=3, precision="fp32", config=_cfg())
    z = np.zeros(0)
    t.load_particles(z, z, z, z, z, z, z)
    t.step(2)
    torch.cuda.synchronize()
    assert t.error_flag() == 0


@pytest.mark.parametrize("order", [1, 3])
def test_cell_groups_charge_conservation(cuda, order):
    n, g = (16, 16, 16), 3
    st = plasma(n, 8, 0.05, seed=2200 + order)
    t = TiledSim(n, order=order, precision="fp32", config=_cfg(sort_interval=5))
    t.load_particles(st["x"], st["y"], st["z"], st["ux"], st["uy"], st["uz"], st["w"])
    t.diagnostics()
    r0 = _gauss_residual(t, g)
    t.step(20)
    t.diagnostics()
    r1 = _gauss_residual(t, g)
    drift = np.linalg.norm(r1 - r0) / np.linalg.norm(r0)
    assert drift < 1e-5, drift
    assert t.error_flag() == 0


def test_cell_groups_reject_order_2(cuda):
    with pytest.raises(ValueError):
        TiledSim((16, 16, 16), order=2, precision="fp32", config=_cfg())
