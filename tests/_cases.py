"""Shared seeded inputs and comparison helpers for the parity tests."""
from __future__ import annotations

import numpy as np

from picsar_b200.init import thermal_plasma, cfl_dt


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))


def random_fields(n, g, seed, amp=0.05):
    """Six smooth-ish random guarded fields with valid periodic guards."""
    from oracle import oracle as O
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(6):
        a = O.zeros_grid(*n, g)
        a[...] = amp * rng.standard_normal(a.shape)
        O.field_bc(a, n, g)
        out.append(a)
    return out


def plasma(n, ppc, sigma, seed, drift=(0.0, 0.0, 0.0)):
    st = thermal_plasma(n, ppc, sigma, seed, drift=drift, shuffle=True).numpy()
    return st


def fresh_particles(st, clight=1.0):
    """Particle dict with gaminv and zeroed particle fields."""
    d = {c: st[c].copy() for c in ("x", "y", "z", "ux", "uy", "uz", "w")}
    u2 = d["ux"] ** 2 + d["uy"] ** 2 + d["uz"] ** 2
    d["gaminv"] = 1.0 / np.sqrt(1.0 + u2 / clight ** 2)
    for c in ("ex", "ey", "ez", "bx", "by", "bz"):
        d[c] = np.zeros_like(d["x"])
    return d


__all__ = ["rel_l2", "random_fields", "plasma", "fresh_particles", "cfl_dt"]
