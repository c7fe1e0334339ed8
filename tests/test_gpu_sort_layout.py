"""Layout of the particles inside a tile after the sort.

The particle kernel reads each warp's gather stencils and adds its deposits at
shared-memory addresses whose bank (address mod 32) is fixed by the
particle's cell in the tile window.  The sort therefore numbers the tile's
particles within their bank class (cell-major) and lays them out by
(level, class).  These tests rebuild the class of every sorted particle on
the host and check the exact class sequence and the cell-major order inside
each class, for orders 1-3 (order 2 shifts the class cell to the nearest
node), 4^3 and 8^3 tiles, and a tile whose class outgrows the level table;
and the same class sequence after particles moved and pxrb_tiled_relayout
put each tile back in bank order (a permutation inside the tile).
"""
import numpy as np
import pytest
import torch

from picsar_b200.tiled import TiledConfig, TiledSim

# window pitch (row SY, plane SZ) per (tile edge, window edge), as compiled
PITCH = {(8, 9): (9, 84), (8, 11): (11, 124), (8, 13): (13, 172), (8, 15): (15, 228),
         (4, 5): (6, 40), (4, 7): (8, 58), (4, 9): (10, 104)}


def _window(tile, drift, order):
    return tile + 2 * drift + (1 if order == 1 else 3)


def test_pitch_table_gives_equal_bank_classes():
    for (T, W), (sy, sz) in PITCH.items():
        assert sy >= W and sz >= sy * W
        a, b, c = np.meshgrid(np.arange(T), np.arange(T), np.arange(T), indexing="ij")
        h = np.bincount(((a + sy * b + sz * c) % 32).ravel(), minlength=32)
        assert h.min() == h.max() == T ** 3 // 32


def _check(sim, after_sort=True):
    """after_sort: particles inside their tile, cell-major inside each class;
    otherwise (after a re-layout of moved particles) within the tile window,
    any order inside a class."""
    T = sim.tile[0]
    D = sim.cfg.drift
    sy, sz = PITCH[(T, _window(T, sim.cfg.drift, sim.order))]
    arr = sim.arrays()
    cell = arr["cell"].cpu().numpy().astype(np.int64)
    off = sim.tile_off.cpu().numpy()
    o = [arr[c].cpu().numpy() for c in ("ox", "oy", "oz")]
    ntx, nty, _ = sim.nt
    x, y, z = cell & 2047, (cell >> 11) & 2047, cell >> 22
    checked = 0
    for t in range(sim.ntiles):
        b0, b1 = off[t], off[t + 1]
        if b0 == b1:
            continue
        sl = slice(b0, b1)
        loc = []
        for v, t0, nn in ((x[sl], (t % ntx) * T, sim.n[0]), (y[sl], ((t // ntx) % nty) * T, sim.n[1]),
                          (z[sl], (t // (ntx * nty)) * T, sim.n[2])):
            lv = v - t0
            lv = np.where(lv > T - 1 + D, lv - nn, np.where(lv < -D, lv + nn, lv))
            lo, hi = (0, T - 1) if after_sort else (-D, T - 1 + D)
            assert lv.min() >= lo and lv.max() <= hi, "particle outside its tile window"
            loc.append(lv)
        lx, ly, lz = loc
        hx, hy, hz = lx.copy(), ly.copy(), lz.copy()
        if sim.order == 2:
            hx += o[0][sl] >= 0.5
            hy += o[1][sl] >= 0.5
            hz += o[2][sl] >= 0.5
        k = (hx + sy * hy + sz * hz) & 31
        n = np.bincount(k, minlength=32)
        want = np.array([c for lev in range(n.max()) for c in range(32) if n[c] > lev])
        assert np.array_equal(k, want), f"tile {t}: class sequence"
        if after_sort:
            lc = lx + T * ly + T * T * lz
            for c in range(32):
                assert np.all(np.diff(lc[k == c]) >= 0), f"tile {t} class {c}: not cell-major"
        checked += 1
    return checked


def _sim(n, order, tile, drift, ppc, seed, prec="fp32", crowd=0):
    rng = np.random.default_rng(seed)
    m = int(np.prod(n)) * ppc
    pos = [rng.uniform(0, L, m) for L in n]
    if crowd:
        for a in range(3):
            pos[a][:crowd] = 3.0 + rng.uniform(0, 1, crowd)
    u = [0.01 * rng.standard_normal(m) for _ in range(3)]
    cfg = TiledConfig(tile=(tile,) * 3, drift=drift, acc=1 if prec == "fp32" else 2)
    s = TiledSim(n, order=order, precision=prec, config=cfg)
    s.load_particles(*pos, *u, np.full(m, 0.1))
    torch.cuda.synchronize()
    return s


@pytest.mark.gpu
@pytest.mark.parametrize("order,tile,drift,prec", [(1, 8, 1, "fp32"), (2, 8, 1, "fp32"),
                                                   (3, 8, 1, "fp32"), (3, 4, 1, "fp32"),
                                                   (2, 8, 2, "fp32"), (3, 8, 1, "fp64")])
def test_layout_by_level_and_bank_class(cuda, order, tile, drift, prec):
    s = _sim((24, 16, 32), order, tile, drift, 8, 10 + order, prec)
    assert _check(s) == s.ntiles
    host = lambda d: {c: v.cpu().numpy() for c, v in d.items()}
    s.step(3)                    # positions move; the re-layout restores the bank order
    mid = host(s.particles())
    s.relayout()
    torch.cuda.synchronize()
    assert _check(s, after_sort=False) == s.ntiles
    after = host(s.particles())  # the same particles, permuted inside their tiles
    key = lambda d: np.lexsort([d[c] for c in ("uz", "uy", "ux", "z", "y", "x")])
    for c in mid:
        assert np.array_equal(mid[c][key(mid)], after[c][key(after)]), c
    s.sort()
    torch.cuda.synchronize()
    assert _check(s) == s.ntiles


@pytest.mark.gpu
def test_layout_of_a_crowded_tile(cuda):
    # 70,000 particles in one cell: one class of 70,000 levels (beyond the
    # level table, summed directly)
    s = _sim((16, 16, 16), 3, 8, 1, 20, 5, crowd=70000)
    assert _check(s) == s.ntiles
    s.step(1)
    s.relayout()                 # a class beyond the level table: summed directly
    torch.cuda.synchronize()
    assert _check(s, after_sort=False) == s.ntiles
    assert s.error_flag() == 0
