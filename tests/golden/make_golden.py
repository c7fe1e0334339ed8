"""Golden fixtures of the PIC step, made by the oracle.

The reference ships no golden vectors for this path; these fixtures are made
by the oracle (pinned bit for bit to the reference's own routines by
tests/test_oracle_vs_reference.py) from seeded inputs, so that parity tests
on machines without the reference sources compare against fixed numbers.

Each case: a periodic thermal electron plasma on a small grid with random
initial fields, ``steps`` full PIC steps (gather+push, periodic particle
boundaries, Esirkepov deposit, Yee B/E/B with guard exchange).  Stored per
case: the initial particles, the final particles (sorted by id) and the
final E, B and J grids (Fortran order, lower bound -g).

Regenerate with ``python -m tests.golden.make_golden`` from the repository
root.
"""
from __future__ import annotations

import os

import numpy as np

PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "oracle_steps.npz")
G = 3
FIELDS = ("ex", "ey", "ez", "bx", "by", "bz", "jx", "jy", "jz")
PCOLS = ("x", "y", "z", "ux", "uy", "uz", "gaminv")
CASES = [
    dict(n=(8, 8, 12), ppc=2, sigma=0.01, order=1, pusher=0, steps=4, seed=1001),
    dict(n=(8, 12, 8), ppc=2, sigma=0.05, order=2, pusher=1, steps=3, seed=1002),
    dict(n=(12, 8, 8), ppc=2, sigma=0.05, order=3, pusher=0, steps=3, seed=1003),
]


def tag(n, ppc, sigma, order, pusher, steps, seed):
    return f"o{order}_p{pusher}_s{seed}"


def initial_state(n, ppc, sigma, seed):
    from picsar_b200.init import thermal_plasma
    from tests._cases import random_fields
    st = thermal_plasma(n, ppc, sigma, seed, shuffle=True).numpy()
    fields = random_fields(n, G, seed=seed + 1, amp=0.02)
    return st, fields


def run_case(n, ppc, sigma, order, pusher, steps, seed, st=None):
    from oracle import oracle as O
    st0, fields = initial_state(n, ppc, sigma, seed)
    if st is None:
        st = st0
    s = O.OracleSim(n, G, order=order, pusher=pusher)
    for name, a in zip(FIELDS[:6], fields):
        s.set_field(name, a)
    s.add_particles(st["x"], st["y"], st["z"], st["ux"], st["uy"], st["uz"], st["w"])
    s.step(steps)
    out = {f"init_{c}": st[c] for c in ("x", "y", "z", "ux", "uy", "uz", "w")}
    p = s.particles()
    for c in PCOLS:
        out[c] = p[c]
    for f in FIELDS:
        out[f] = s.get_field(f)
    return out


def main():
    arrays = {}
    for case in CASES:
        for k, v in run_case(**case).items():
            arrays[f"{tag(**case)}/{k}"] = v
    np.savez_compressed(PATH, **arrays)
    print(PATH, os.path.getsize(PATH))


if __name__ == "__main__":
    main()
