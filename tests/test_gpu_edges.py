"""Edge cases of the step on the B200: a context without particles, and particle counts that
are not multiples of the 8-slot groups the push and the sort read with 16-byte vectors.

Tolerances are those of the parity tests: positions 1e-6 dx and velocities 1e-6 relative
after one push against the FP64 mover; the sort order exact (integer work)."""
import numpy as np
import pytest

from jd_lepic_b200 import _capi as capi, configs
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def sim_for(case, **kw):
    from jd_lepic_b200.simulation import GpuSimulation
    return GpuSimulation(case, tile=(8, 8), **kw)


def test_empty_context_runs_full_steps(gpu_lib):
    """No particles: twelve steps (the sorts of steps 1 and 11, the collision step 11, the
    Poisson solves) succeed and leave an empty plasma with zero density."""
    case = configs.case0(ppc=1, nx=32, ny=32)
    s = sim_for(case, load=False, capacity=64)
    try:
        for it in range(1, 13):
            s.step(it)
        s.sync()
        assert s.push_stats()["np_tot"] == [0, 0]
        for k in range(2):
            assert np.all(s.grid(capi.GRID_NP + k) == 0.0)
            assert s.get_particles(k).shape == (0, 6)
    finally:
        s.close()


@pytest.mark.parametrize("n", [1, 7, 13, 1029])
def test_ragged_counts_sort_and_push(gpu_lib, n):
    case = configs.case0(ppc=1, nx=32, ny=32)
    from jd_lepic_b200.simulation import GpuSimulation
    s = GpuSimulation(case, tile=(case.nx, 1), load=False, capacity=4096)   # the reference's cell order
    try:
        rng = np.random.default_rng(n)
        cfg = O.make_cfg(case, s.sp)
        for k, vs in ((0, 2.0e5), (1, 5.0e2)):
            v = np.zeros((n, 6))
            v[:, 0] = (1.0 + rng.random(n) * (case.nx - 2)) * case.dx
            v[:, 1] = (1.0 + rng.random(n) * (case.ny - 2)) * case.dy
            v[:, 3:] = rng.normal(0.0, vs, (n, 3)).astype(np.float32)
            s.put_particles(k, v)
        # the sort: the reference order (stable by cell) of the device's own positions
        for k in range(2):
            before = s.get_particles(k)
            s.sort(k)
            after = s.get_particles(k)
            cell = ((before[:, 0] / case.dx + 1e-9).astype(int) + case.nx * (before[:, 1] / case.dy + 1e-9).astype(int))
            order = np.argsort(cell, kind="stable")
            assert np.array_equal(after, before[order])
        s.set_phi(np.zeros((case.ny + 3, case.nx + 3)))
        E = s.efield()
        p0 = [s.get_particles(k) for k in range(2)]
        s.push(1)
        for k in range(2):
            ref = p0[k].copy()
            n_ref, _ = O.mover(cfg, k, E, case.Bi, case.bcnd, ref)
            got = s.get_particles(k)
            assert got.shape[0] == n_ref == n
            assert np.abs(got[:, :2] - ref[:n_ref, :2]).max() <= 1e-6 * case.dx
            vmag = np.linalg.norm(ref[:n_ref, 3:], axis=1) + s.sp.vt0[k]
            assert (np.linalg.norm(got[:, 3:] - ref[:n_ref, 3:], axis=1) / vmag).max() <= 1e-6
            npg = np.zeros((case.ny + 3, case.nx + 3))
            O.deposit(cfg, k, got, got.shape[0], O.kq_of(case.bcnd), npg)
            assert np.abs(s.grid(capi.GRID_NP + k) - npg).max() <= 1e-12 * np.abs(npg).max()
    finally:
        s.close()
