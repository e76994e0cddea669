"""The particle backup (particlesNNN.bak) written from and read into the device, against the
record-format checker (oracle/fortran_records.py)."""
import os

import numpy as np
import pytest

from oracle import fortran_records as FR
from jd_lepic_b200 import _capi as capi, configs
from jd_lepic_b200.simulation import GpuSimulation

pytestmark = pytest.mark.gpu


def test_write_then_read_round_trip(gpu_lib, tmp_path):
    case = configs.case0(ppc=4, nx=64, ny=64)
    a = GpuSimulation(case)
    b = GpuSimulation(case, load=False)
    try:
        a.set_options(fortran_max_subrecord=1000)   # every particle record is split
        a.push(1)                                   # some particles are lost: holes are skipped
        a.deposit()
        path = str(tmp_path / "particles000.bak")
        a.write_backup(path, 3.5e-7, 2, 0.875)
        t, g, pc, np_tot, parts = FR.read_backup(path, 2)
        assert (t, g, pc) == (3.5e-7, 2, 0.875) and np_tot.shape == (1, 2)
        live = [a.get_particles(s) for s in (0, 1)]
        assert np_tot[0].tolist() == [len(live[0]), len(live[1])] == a.push_stats()["np_tot"]
        assert os.path.getsize(path) > 48 * len(live[0])
        for s in (0, 1):
            assert np.array_equal(parts[s][0], live[s])          # z is written as 0
        t2 = b.read_backup(path)
        assert t2 == (3.5e-7, 2, 0.875)
        for s in (0, 1):
            assert np.array_equal(b.get_particles(s), live[s])
            assert np.array_equal(b.grid(capi.GRID_NP + s), a.grid(capi.GRID_NP + s))
    finally:
        a.close()
        b.close()


def test_read_file_of_two_threads(gpu_lib, tmp_path):
    case = configs.case0(ppc=4, nx=64, ny=64)
    sim = GpuSimulation(case, load=False)
    try:
        rng = np.random.default_rng(2)

        def block(n):
            v = np.zeros((n, 6))
            v[:, 0] = rng.random(n) * case.nx * case.dx * 0.999
            v[:, 1] = rng.random(n) * case.ny * case.dy * 0.999
            v[:, 2] = rng.random(n)
            v[:, 3:] = rng.normal(0, 1e5, (n, 3)).astype(np.float32)
            return v
        blocks = [[block(300), block(50)], [block(200), block(0)]]
        path = str(tmp_path / "p.bak")
        FR.write_backup(path, 1.0, 7, 1.0, blocks, max_sub=1000)
        sim.read_backup(path)
        unit = case.dx * 2.0 ** -21
        for s in (0, 1):
            got = sim.get_particles(s)
            ref = np.concatenate([blocks[0][s], blocks[1][s]])
            assert len(got) == len(ref)
            assert np.abs(got[:, :2] - ref[:, :2]).max() <= unit
            assert np.array_equal(got[:, 3:], ref[:, 3:])
    finally:
        sim.close()


def test_read_beyond_capacity(gpu_lib, tmp_path):
    case = configs.case0(ppc=4, nx=64, ny=64)
    sim = GpuSimulation(case, load=False, capacity=100)
    try:
        v = np.zeros((150, 6))
        v[:, 0] = 1e-4
        v[:, 1] = 1e-4
        path = str(tmp_path / "big.bak")
        FR.write_backup(path, 0.0, 0, 1.0, [[v, v[:10]]])
        assert sim.lib.lepic_gpu_read_backup(sim.ctx, path.encode(), None, None, None) == capi.ECAPACITY
        assert sim.push_stats()["np_tot"] == [0, 0]
    finally:
        sim.close()


def test_slab_layout_put_get(gpu_lib):
    """vxp(6, nmax, ntype, nproc) with np_tot(ntype, nproc), the reference's own arrays."""
    import ctypes as C
    case = configs.case0(ppc=4, nx=64, ny=64)
    sim = GpuSimulation(case, load=False)
    try:
        rng = np.random.default_rng(3)
        nmax, ntype, nproc = 500, 2, 3
        vxp = np.zeros((nproc, ntype, nmax, 6))          # Fortran vxp(6, nmax, ntype, nproc)
        np_tot = np.zeros((nproc, ntype), dtype=np.int32)  # Fortran np_tot(ntype, nproc)
        for p in range(nproc):
            for s in range(ntype):
                k = int(rng.integers(0, nmax))
                np_tot[p, s] = k
                u = np.zeros((k, 6))
                # positions on the fixed-point grid, FP32 velocities: the round trip is exact
                u[:, 0] = np.floor(rng.random(k) * case.nx * 2 ** 21) * case.dx * 2.0 ** -21
                u[:, 1] = np.floor(rng.random(k) * case.ny * 2 ** 21) * case.dy * 2.0 ** -21
                u[:, 3:] = rng.normal(0, 1e5, (k, 3)).astype(np.float32)
                vxp[p, s, :k] = u
        dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
        ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int32))
        sim.check(sim.lib.lepic_gpu_put_particles_slabs(sim.ctx, dp(vxp), ip(np_tot), nmax, ntype, nproc), "put_slabs")
        for s in range(ntype):
            ref = np.concatenate([vxp[p, s, :np_tot[p, s]] for p in range(nproc)])
            assert np.array_equal(sim.get_particles(s), ref)
        out = np.zeros_like(vxp)
        nt = np.zeros_like(np_tot)
        sim.check(sim.lib.lepic_gpu_get_particles_slabs(sim.ctx, dp(out), ip(nt), nmax, ntype, nproc), "get_slabs")
        for s in range(ntype):
            total = np_tot[:, s].sum()
            assert nt[:, s].sum() == total and nt[:, s].max() - nt[:, s].min() <= 1
            got = np.concatenate([out[p, s, :nt[p, s]] for p in range(nproc)])
            assert np.array_equal(got, np.concatenate([vxp[p, s, :np_tot[p, s]] for p in range(nproc)]))
    finally:
        sim.close()


def test_truncated_backup_is_rejected(gpu_lib, tmp_path):
    """A backup cut short (in the header, inside a particle record, before the last length
    marker) is refused with LEPIC_EINVAL; the context keeps its particles and stays usable."""
    case = configs.case0(ppc=2, nx=32, ny=32)
    a = GpuSimulation(case)
    b = GpuSimulation(case, load=False)
    try:
        full = str(tmp_path / "full.bak")
        a.write_backup(full, 1.0, 0, 1.0)
        data = open(full, "rb").read()
        for cut in (10, 40, len(data) // 2, len(data) - 4, len(data) - 1):
            p = str(tmp_path / f"cut{cut}.bak")
            open(p, "wb").write(data[:cut])
            rc = b.lib.lepic_gpu_read_backup(b.ctx, p.encode(), None, None, None)
            assert rc == capi.EINVAL, cut
            assert b.push_stats()["np_tot"] == [0, 0], cut
        b.read_backup(full)
        for s in (0, 1):
            assert np.array_equal(b.get_particles(s), a.get_particles(s))
    finally:
        a.close()
        b.close()


def test_external_restart_from_two_files_then_duplication(gpu_lib, tmp_path):
    """The reference's external restart (restart.f90:66-108): one rank reads several backup
    files, appending each; then np_dup (:115-129) follows every species' particles with
    |np_dup| - 1 copies of themselves, and the density is deposited from all of them."""
    from oracle import oracle as O
    case = configs.case0(ppc=2, nx=32, ny=32)
    a = GpuSimulation(case)
    b = GpuSimulation(case, load=False, capacity=6 * case.n_particles)
    try:
        p1 = str(tmp_path / "particles000.bak")
        p2 = str(tmp_path / "particles001.bak")
        a.write_backup(p1)
        a.push(1)
        a.deposit()
        a.write_backup(p2)
        live = [np.concatenate([FR.read_backup(p, 2)[4][s][0] for p in (p1, p2)]) for s in (0, 1)]
        b.read_backup(p1)
        b.read_backup(p2)
        for s in (0, 1):
            assert np.array_equal(b.get_particles(s), live[s])
        with pytest.raises(capi.LepicError) as e:
            b.check(b.lib.lepic_gpu_duplicate_particles(b.ctx, 7), "duplicate")
        assert e.value.code == capi.ECAPACITY
        b.check(b.lib.lepic_gpu_duplicate_particles(b.ctx, -3), "duplicate")
        cfg = O.make_cfg(case, b.sp)
        kq = O.kq_of(case.bcnd)
        for s in (0, 1):
            got = b.get_particles(s)
            assert np.array_equal(got, np.concatenate([live[s]] * 3))
            assert b.push_stats()["np_tot"][s] == 3 * len(live[s])
            npg = np.zeros((case.ny + 3, case.nx + 3))
            O.deposit(cfg, s, got, got.shape[0], kq, npg)
            assert np.abs(b.grid(capi.GRID_NP + s) - npg).max() <= 1e-12 * np.abs(npg).max()
        b.step(1)                                   # the context runs on
        b.sync()
    finally:
        a.close()
        b.close()
