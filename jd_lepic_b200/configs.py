"""The five synthetic workloads of the benchmark, built as the reference's host would
build them: a node mask ``bcnd`` with wall potentials (generate_boundary.f90 semantics:
>0 Dirichlet wall label, -1 interior, ghosts copied from the edge), optional B fields,
species/reaction decks in the reference's text format, and the device load.

    cfg 0  128x128,  e + Ar+, 100 ppc, uniform 1e16, Te 2 eV, Ti 0.03 eV, Ar 1 Pa/300 K,
           dt 5e-12, MG to 1e-10 (the reference's L1 metric), 100 steps
    cfg 1  512x512,  200 ppc, Gaussian 5e16 peak / 1e15 floor, sigma 0.25 L, 500 steps
    cfg 2  1024x512, 100 ppc, line-dipole B (|B|max 0.05 T) + Bz 0.01 T, bottom wall -300 V,
           dt 2e-12, mixed-precision Poisson to 1e-8, 1000 steps
    cfg 3  1024x1024, He+ + e, 150 ppc, synthetic He cross sections, 20k training pairs
    cfg 4  2048x2048, 50 ppc, 3-aperture plate at x = 0.8 L (+1 kV, 40-cell apertures),
           -50 V source wall, Bz 0.005 T, dt 1e-12, 2000 steps
Every case can be shrunk (``ppc``, grid) for tests; the mask and field shapes scale with it.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import deck as dk

KB = 1.380649e-23


@dataclass
class Case:
    name: str
    nx: int
    ny: int
    dx: float
    dy: float
    dt: float
    bcnd: np.ndarray              # int32 (ny+3, nx+3): [j, i] = bcnd(i, j)
    phi0: np.ndarray              # float64 (ny+3, nx+3) wall potentials
    deck_text: str
    ngas: float
    te: float                     # electron temperature, eV
    n0: float                     # reference density for Nm (main.f90:471)
    ppc: int                      # macroparticles per cell per species
    profile: int = 0              # 0 uniform, 1 Gaussian
    n_peak: float = 0.0
    n_floor: float = 0.0
    sigma: float = 0.0
    flag_B: int = 0
    Bc: tuple = (0.0, 0.0, 0.0)
    Bi: Optional[np.ndarray] = None   # float64 (ny+3, nx+3, 4)
    eps: float = 1e-8
    poisson_mode: int = 1
    steps: int = 100
    ng: int = 0
    zmax: float = 1.0
    seed: int = 1
    # boundary options (read_input.f90): periodic y, specular y walls with it, Neumann at x = 0
    flag_pbc: int = 0
    flag_spec: int = 0
    flag_nmn: int = 0
    # particle decomposition over MPI ranks (load_part.f90:96): ppc is the deck's np_cell, the
    # particles per cell of all ranks together, which sets Nm = n0 Vc / np_cell (main.f90:471);
    # each rank loads NINT(np_cell n_cell / nproc_mpi) of them, and rho is summed over ranks
    nproc_mpi: int = 1
    extra: dict = field(default_factory=dict)

    @property
    def n_particles(self) -> int:
        return self.ppc * self.nx * self.ny

    @property
    def n_load(self) -> int:
        """Particles per species that one rank loads (load_part.f90:96, nproc = 1 per rank)."""
        return int(math.floor(self.n_particles / self.nproc_mpi + 0.5))

    def levels(self) -> int:
        if self.ng:
            return self.ng
        return int(round(min(math.log2(self.nx), math.log2(self.ny))))  # main.f90:264-267


def box_mask(nx: int, ny: int, label_left=1, label_right=1, label_bottom=1, label_top=1):
    """Closed box: edge nodes carry wall labels, ghosts copy the edge (generate_boundary.f90
    draws polylines out to the ghost index 0 and n+2, :189-190, :203-207)."""
    b = np.full((ny + 3, nx + 3), -1, dtype=np.int32)
    b[:, 0:2] = label_left
    b[:, nx + 1:] = label_right
    b[0:2, :] = label_bottom
    b[ny + 1:, :] = label_top
    return b


def potentials(bcnd: np.ndarray, volts: dict) -> np.ndarray:
    phi = np.zeros(bcnd.shape)
    for lab, v in volts.items():
        phi[bcnd == lab] = v
    return phi


def gas_density(p_pa: float = 1.0, t_k: float = 300.0) -> float:
    return p_pa / (KB * t_k)


def case0(ppc: int = 100, nx: int = 128, ny: int = 128, steps: int = 100) -> Case:
    b = box_mask(nx, ny)
    return Case("cfg0-128x128-uniform", nx, ny, 1e-4, 1e-4, 5e-12, b, potentials(b, {1: 0.0}),
                dk.argon_deck(0.03), gas_density(), 2.0, 1e16, ppc, eps=1e-10, poisson_mode=0,
                steps=steps)


def case1(ppc: int = 200, nx: int = 512, ny: int = 512, steps: int = 500) -> Case:
    b = box_mask(nx, ny)
    L = nx * 1e-4
    return Case("cfg1-512x512-gaussian", nx, ny, 1e-4, 1e-4, 5e-12, b, potentials(b, {1: 0.0}),
                dk.argon_deck(0.03), gas_density(), 2.0, 1e16, ppc, profile=1, n_peak=5e16,
                n_floor=1e15, sigma=0.25 * L, eps=1e-8, poisson_mode=1, steps=steps)


def dipole_field(nx: int, ny: int, dx: float, dy: float, bmax: float = 0.05, bz: float = 0.01):
    """2-D line-dipole array: 4 dipoles of alternating sign a distance 0.1*Ly below the bottom
    wall; B = m (2 (d.r) r - d |r|^2) / |r|^4, scaled so that max |B_in-plane| = bmax over the
    nodes; a uniform Bz is added.  Returns Bi(4, 0:nx+2, 0:ny+2) as (ny+3, nx+3, 4)."""
    Lx, Ly = nx * dx, ny * dy
    i = np.arange(nx + 3) - 1
    j = np.arange(ny + 3) - 1
    X, Y = np.meshgrid(i * dx, j * dy)
    Bx = np.zeros_like(X)
    By = np.zeros_like(X)
    for k in range(4):
        x0, y0 = (k + 0.5) * Lx / 4, -0.1 * Ly
        s = 1.0 if k % 2 == 0 else -1.0
        rx, ry = X - x0, Y - y0
        r2 = rx * rx + ry * ry
        dot = s * ry
        Bx += (2 * dot * rx) / (r2 * r2)
        By += (2 * dot * ry - s * r2) / (r2 * r2)
    mag = np.sqrt(Bx[1:ny + 2, 1:nx + 2] ** 2 + By[1:ny + 2, 1:nx + 2] ** 2).max()
    Bx *= bmax / mag
    By *= bmax / mag
    Bz = np.full_like(X, bz)
    Bi = np.stack([Bx, By, Bz, np.sqrt(Bx * Bx + By * By + Bz * Bz)], axis=-1)  # main.f90:415
    return Bi


def case2(ppc: int = 100, nx: int = 1024, ny: int = 512, steps: int = 1000) -> Case:
    b = box_mask(nx, ny, label_bottom=2)
    b[0:2, :] = 2
    return Case("cfg2-1024x512-magnetron", nx, ny, 1e-4, 1e-4, 2e-12, b,
                potentials(b, {1: 0.0, 2: -300.0}), dk.argon_deck(0.03), gas_density(), 2.0, 1e16,
                ppc, flag_B=2, Bi=dipole_field(nx, ny, 1e-4, 1e-4), eps=1e-8, poisson_mode=1,
                steps=steps)


def case3(ppc: int = 150, nx: int = 1024, ny: int = 1024, steps: int = 100) -> Case:
    b = box_mask(nx, ny)
    return Case("cfg3-1024x1024-helium", nx, ny, 1e-4, 1e-4, 5e-12, b, potentials(b, {1: 0.0}),
                dk.helium_deck(0.03), gas_density(), 2.0, 1e16, ppc, eps=1e-8, poisson_mode=1,
                steps=steps, extra={"training_pairs": 20000})


def aperture_plate(nx: int, ny: int, x_frac: float = 0.8, thickness: int = 32, aperture: int = 40,
                   n_ap: int = 3):
    """Box with the source (left) wall at label 3, the other walls at label 1, and an embedded
    conductor plate (label 2) of `thickness` cells at x = x_frac*L with `n_ap` apertures of
    `aperture` cells centred at (k+1)/(n_ap+1) of the height."""
    b = box_mask(nx, ny, label_left=3)
    i0 = int(round(x_frac * nx)) + 1
    i1 = min(i0 + thickness, nx)
    plate = np.ones(ny + 3, dtype=bool)
    plate[0:2] = False
    plate[ny + 1:] = False
    for k in range(n_ap):
        c = int(round((k + 1) * ny / (n_ap + 1))) + 1
        plate[c - aperture // 2 + 1: c + aperture // 2] = False
    for i in range(i0, i1 + 1):
        b[plate, i] = np.where(b[plate, i] == -1, 2, b[plate, i])
    return b


def case4(ppc: int = 50, nx: int = 2048, ny: int = 2048, steps: int = 2000) -> Case:
    # 40-cell apertures; the plate is 32 cells thick: with thinner plates the injection-
    # coarsened masks of the reference's 11-level V-cycle lose the conductor and the
    # multigrid diverges (8 cells: divergence after 3 cycles; 32 cells: 12 cycles to 1e-8)
    ap = max(5, int(round(40 * nx / 2048)))
    th = max(4, int(round(32 * nx / 2048)))
    b = aperture_plate(nx, ny, thickness=th, aperture=ap)
    return Case("cfg4-2048x2048-aperture-plate", nx, ny, 1e-4, 1e-4, 1e-12, b,
                potentials(b, {1: 0.0, 2: 1000.0, 3: -50.0}), dk.argon_deck(0.03), gas_density(),
                2.0, 1e16, ppc, flag_B=1, Bc=(0.0, 0.0, 0.005), eps=1e-8, poisson_mode=1,
                steps=steps)


CASES = {0: case0, 1: case1, 2: case2, 3: case3, 4: case4}


def make_case(idx: int, **kw) -> Case:
    return CASES[idx](**kw)
