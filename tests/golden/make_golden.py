"""Writes the golden fixtures of tests/golden/ from the CPU restatement (the oracle).

The reference ships no golden vectors and cannot be compiled here (Fortran, MPI), so these
fixtures pin the restatement itself: a 32x32 box with a Boris-magnetised particle set, a
smooth potential, and the oracle's outputs of calc_Efield, part_mover, charge_deposition,
calc_rhs, iterative_solver and part_sorting.  Positions are placed on the GPU's fixed-point
grid (2^-S of a cell) so the device receives them exactly.

    python tests/golden/make_golden.py
"""
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from jd_lepic_b200 import configs, deck as dk  # noqa: E402
from jd_lepic_b200.simulation import species_params  # noqa: E402
from oracle import oracle as O  # noqa: E402


def fixed_shift(nx, ny):
    k = 0
    while (1 << k) < max(nx, ny):
        k += 1
    return min(24, 32 - k)


def golden_case():
    case = configs.case0(ppc=4, nx=32, ny=32)
    case.flag_B, case.Bc = 1, (0.001, -0.002, 0.03)
    return case


def make():
    case = golden_case()
    d = dk.read_reactions(case.deck_text, case.ngas)
    sp = species_params(case, d)
    cfg = O.make_cfg(case, sp)
    S = fixed_shift(case.nx, case.ny)
    rng = np.random.default_rng(20241203)
    n = 1000
    out = {}
    for s in range(2):
        p = np.zeros((n, 6))
        X = rng.integers(0, case.nx << S, n)
        Y = rng.integers(0, case.ny << S, n)
        p[:, 0] = X * (case.dx * 2.0 ** -S)
        p[:, 1] = Y * (case.dy * 2.0 ** -S)
        p[:, 3:] = rng.normal(0, sp.vt0[s] / math.sqrt(2), (n, 3)).astype(np.float32)
        out[f"p{s}"] = p
    i = np.arange(case.nx + 3) - 1
    Xg, Yg = np.meshgrid(i / case.nx, i / case.ny)
    phi = np.where(case.bcnd >= 1, 0.0, 25.0 * np.sin(math.pi * Xg) * np.sin(2 * math.pi * Yg) + 5.0 * Xg)
    out["phi"] = phi
    E = O.efield(cfg, phi, case.bcnd)
    out["E"] = E
    kq = O.kq_of(case.bcnd)
    npg = np.zeros((2, case.ny + 3, case.nx + 3))
    for s in range(2):
        q = out[f"p{s}"].copy()
        m, _t = O.mover(cfg, s, E, None, case.bcnd, q)
        out[f"pushed{s}"] = q[:m]
        O.deposit(cfg, s, q, m, kq, npg[s])
    out["np"] = npg
    rhs = O.calc_rhs(cfg, npg)
    out["rhs"] = rhs
    u = np.where(case.bcnd >= 1, case.phi0, 0.0)
    rc, st = O.solve(cfg, u, rhs, case.bcnd, case.levels(), 1e-10)
    assert rc == 0
    out["phi_solved"] = u
    out["solve_k"] = np.array([st.k, st.sweeps_fine])
    q = out["pushed0"].copy()
    out["plist0"] = O.sort(cfg, q, q.shape[0])
    out["sorted0"] = q
    np.savez_compressed(os.path.join(HERE, "golden_32x32.npz"), **out)
    return out


if __name__ == "__main__":
    o = make()
    print({k: v.shape for k, v in o.items()})
