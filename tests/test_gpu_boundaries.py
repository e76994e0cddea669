"""The boundary options of the reference on the B200 path, against the CPU restatement:
periodic y (bcnd label 0 on the y edges, flag_pbc), specular y walls (label -3, flag_spec)
and the Neumann column at x = 0 (label -2, flag_nmn), as generate_boundary.f90:137-145 sets
them.  They reach the mover (part_expmover.f90:222-241, 454-459), the density fold
(calc_rho.f90:1-35), the smoother and the restriction (sors.f90:66-109, 185-200; mg.f90:298-311,
512-547) and the field (Efield.f90:43-82).

Tolerances are those of the Dirichlet parity tests: positions 1e-6 dx and velocities 1e-6
relative after one push; the density (folded) to 1e-12 of its maximum; E and the right-hand
side bit-identical; the FP64 V-cycle with the same cycle and sweep counts and phi to 1e-13."""
import math

import numpy as np
import pytest

from jd_lepic_b200 import _capi as capi, configs
from oracle import oracle as O

pytestmark = pytest.mark.gpu

N = 64


def boundary_case(kind):
    """A 64 x 64 box: walls at 0 V (label 1) on the left and 10 V (label 2) on the right;
    'pbc' / 'spec' make the y edges periodic, 'nmn' makes the x = 0 column Neumann."""
    case = configs.case0(ppc=20, nx=N, ny=N)
    b = configs.box_mask(N, N, label_left=1, label_right=2, label_bottom=1, label_top=1)
    if kind in ("pbc", "spec", "pbc_nmn"):
        b[0:2, 2:N + 1] = 0
        b[N + 1:, 2:N + 1] = 0
        case.flag_pbc = 1
        case.flag_spec = 1 if kind == "spec" else 0
    if kind in ("nmn", "pbc_nmn"):
        rows = slice(0, N + 3) if kind == "pbc_nmn" else slice(2, N + 1)
        b[rows, 0:2] = -2
        case.flag_nmn = 1
    case.bcnd = b
    case.phi0 = configs.potentials(b, {1: 0.0, 2: 10.0})
    return case


def smooth_phi(case, amp=30.0):
    i = np.arange(case.nx + 3) - 1
    j = np.arange(case.ny + 3) - 1
    X, Y = np.meshgrid(i / case.nx, j / case.ny)
    phi = 10.0 * X + amp * np.sin(2 * math.pi * Y) * np.sin(math.pi * X) * (1 + 0.3 * np.cos(3 * X + 5 * Y))
    return np.where(case.bcnd >= 1, case.phi0, phi)


def sim_for(case):
    from jd_lepic_b200.simulation import GpuSimulation
    return GpuSimulation(case, tile=(8, 8))


KINDS = ["pbc", "spec", "nmn", "pbc_nmn"]


@pytest.mark.parametrize("kind", KINDS)
def test_efield_bit_exact(gpu_lib, kind):
    case = boundary_case(kind)
    s = sim_for(case)
    try:
        phi = smooth_phi(case)
        s.set_phi(phi)
        E = s.efield()
        Eref = O.efield(O.make_cfg(case, s.sp), phi, case.bcnd)
        assert np.array_equal(E, Eref)
    finally:
        s.close()


@pytest.mark.parametrize("kind", KINDS)
def test_push_and_folded_density_match_oracle(gpu_lib, kind):
    case = boundary_case(kind)
    s = sim_for(case)
    try:
        s.set_phi(smooth_phi(case))
        E = s.efield()
        cfg = O.make_cfg(case, s.sp)
        p0 = [s.get_particles(k) for k in range(2)]
        # electrons fast enough that many cross the y edges (and reach x = 0) in one step
        for k in range(2):
            v = p0[k].copy()
            rng = np.random.default_rng(10 + k)
            near = rng.random(len(v)) < 0.3
            v[near, 1] = np.where(rng.random(near.sum()) < 0.5, 0.2, N - 0.2) * case.dy
            v[near, 0] = np.where(rng.random(near.sum()) < 0.5, rng.random(near.sum()) * case.dx,
                                  v[near, 0])
            vmax = 0.8 * case.dy / case.dt
            v[near, 4] = np.float32(np.clip(rng.normal(0, vmax / 2, near.sum()), -vmax, vmax))
            v[near, 3] = np.float32(np.clip(rng.normal(0, vmax / 2, near.sum()), -vmax, vmax))
            s.put_particles(k, v)
            s.sort(k)
            p0[k] = s.get_particles(k)
        s.push(1)
        got_all = [s.get_particles(k) for k in range(2)]
        for sp in range(2):
            ref = p0[sp].copy()
            n_ref, _ = O.mover(cfg, sp, E, case.Bi, case.bcnd, ref)
            ref = ref[:n_ref]
            got = got_all[sp]
            assert abs(got.shape[0] - n_ref) <= 2
            if got.shape[0] == n_ref:
                vth = s.sp.vt0[sp]
                dy = np.abs(got[:, 1] - ref[:, 1])
                if case.flag_pbc:   # y = ymax after a wrap is stored as y = 0
                    dy = np.minimum(dy, np.abs(dy - case.ny * case.dy))
                assert np.abs(got[:, 0] - ref[:, 0]).max() <= 1e-6 * case.dx
                assert dy.max() <= 1e-6 * case.dy
                vmag = np.linalg.norm(ref[:, 3:], axis=1)
                dvel = (np.linalg.norm(got[:, 3:] - ref[:, 3:], axis=1) / (vmag + vth)).max()
                assert dvel <= 1e-6, dvel
        # the density after the periodic fold (calc_rho.f90:1-35)
        kq = O.kq_of(case.bcnd)
        npg = np.zeros((2, case.ny + 3, case.nx + 3))
        for sp in range(2):
            O.deposit(cfg, sp, got_all[sp], got_all[sp].shape[0], kq, npg[sp])
        O.np_periodic(cfg, npg, case.bcnd)
        dev = np.stack([s.grid(capi.GRID_NP + sp) for sp in range(2)])
        inner = (slice(None), slice(1, case.ny + 2), slice(1, case.nx + 2))
        assert np.abs(dev[inner] - npg[inner]).max() <= 1e-12 * np.abs(npg).max()
        # the right-hand side from the device's folded densities
        assert np.array_equal(s.calc_rhs(), O.calc_rhs(cfg, dev))
    finally:
        s.close()


def _rhs(case, s):
    rhs = s.calc_rhs()
    i = np.arange(case.nx + 1)
    j = np.arange(case.ny + 1)
    X, Y = np.meshgrid(i / case.nx, j / case.ny)
    return rhs + 1.6e-3 * np.sin(3 * math.pi * X) * np.cos(2 * math.pi * Y)


@pytest.mark.parametrize("kind", ["pbc", "nmn", "pbc_nmn"])
def test_mg_fp64_matches_oracle(gpu_lib, kind):
    case = boundary_case(kind)
    s = sim_for(case)
    try:
        rhs = _rhs(case, s)
        a = np.ascontiguousarray(rhs)
        import ctypes as C
        s.check(s.lib.lepic_gpu_set_grid(s.ctx, capi.GRID_RHS, a.ctypes.data_as(C.POINTER(C.c_double))), "set_grid")
        st = s.solve(eps=1e-10, mode=capi.POISSON_FP64_MG, phi=case.phi0.copy())
        cfg = O.make_cfg(case, s.sp)
        ref = case.phi0.copy()
        rc, ost = O.solve(cfg, ref, rhs, case.bcnd, case.levels(), 1e-10)
        assert rc == 0
        assert st["cycles"] == ost.k
        assert st["sweeps_fine"] == ost.sweeps_fine
        assert np.abs(st["phi"] - ref).max() <= 1e-13 * np.abs(ref).max()
        # the mixed-precision mode hands these masks to the FP64 V-cycle with the relative L2
        # criterion; 1e-8 in the residual is about 1e-5 in phi with a Neumann column
        st2 = s.solve(eps=1e-8, mode=capi.POISSON_MIXED_IR, phi=case.phi0.copy())
        assert st2["res_l2_rel"] <= 1e-8
        assert O.l2_residual(cfg, st2["phi"], rhs, case.bcnd) <= 1e-8
        assert np.abs(st2["phi"] - ref).max() <= 2e-4 * np.abs(ref).max()
    finally:
        s.close()
