"""Particle decomposition over ranks (load_part.f90:96, calc_rho.f90:71-74) through the library,
on one GPU: two contexts each holding half of the particles, at the same Nm as one context
holding all of them.  Their charge accumulators (lepic_gpu_deposit_grid, int64 CIC weights in
units of 2^-44) summed on the device must equal the single context's accumulator bit for bit,
and so must the right-hand side formed from the sum (calc_rhs); the accumulator itself must
equal the integer CIC restated in numpy (oracle.int_deposit), which the gloo rank test uses.
Also dens_red (calc_rho.f90:134-199) against the oracle's restatement."""
import ctypes as C

import numpy as np
import pytest

from jd_lepic_b200 import _capi as capi, configs
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _acc_view(sim, sp):
    import torch
    ptr = C.c_void_p()
    sim.check(sim.lib.lepic_gpu_deposit_grid(sim.ctx, sp, C.byref(ptr)), "deposit_grid")
    nn = (sim.case.nx + 3) * (sim.case.ny + 3)

    class _A:
        __cuda_array_interface__ = {"shape": (nn,), "typestr": "<i8", "data": (ptr.value, False), "version": 3,
                                    "stream": sim.stream_ptr() or 1}
    return torch.as_tensor(_A(), device=f"cuda:{torch.cuda.current_device()}")


def _fixed_point(sim, sp):
    import torch
    X, Y, VX = C.c_void_p(), C.c_void_p(), C.c_void_p()
    n, shift = C.c_int64(), C.c_int32()
    sim.check(sim.lib.lepic_gpu_particle_arrays(sim.ctx, sp, C.byref(X), C.byref(Y), C.byref(VX), None, None,
                                                C.byref(n), C.byref(shift)), "particle_arrays")
    out = []
    for p in (X, Y):
        class _A:
            __cuda_array_interface__ = {"shape": (n.value,), "typestr": "<u4", "data": (p.value, False),
                                        "version": 3, "stream": sim.stream_ptr() or 1}
        out.append(torch.as_tensor(_A(), device=f"cuda:{torch.cuda.current_device()}").cpu().numpy()
                   .astype(np.int64))
    return out[0], out[1], shift.value


@pytest.mark.parametrize("nx", [64, 1024])
def test_two_ranks_sum_to_one(gpu_lib, nx):
    import torch
    from jd_lepic_b200.simulation import GpuSimulation
    case = configs.case0(ppc=20 if nx == 64 else 2, nx=nx, ny=nx)
    src = GpuSimulation(case, tile=(16, 16))                # the synthetic load, read back once
    parts = [src.get_particles(k) for k in range(2)]
    src.close()
    full = GpuSimulation(case, tile=(16, 16), load=False)
    halves = [GpuSimulation(case, tile=(16, 16), load=False) for _ in range(2)]
    try:
        assert all(h.sp.Nm[k] == full.sp.Nm[k] for h in halves for k in range(2))
        for k in range(2):
            n = parts[k].shape[0]
            full.put_particles(k, parts[k])
            halves[0].put_particles(k, parts[k][: n // 2])
            halves[1].put_particles(k, parts[k][n // 2:])
        for s in [full] + halves:
            s.deposit()
            s.sync()
        for k in range(2):
            a, b, f = _acc_view(halves[0], k), _acc_view(halves[1], k), _acc_view(full, k)
            total = a + b                                   # the all-reduce's sum, on the device
            torch.cuda.synchronize()
            assert torch.equal(total, f), k
            X, Y, S = _fixed_point(full, k)
            ref = O.int_deposit(X, Y, case.nx, case.ny, S).view(np.int64)
            assert np.array_equal(f.cpu().numpy(), ref), k
            a.copy_(total)                                  # rank 0 after the all-reduce
            torch.cuda.synchronize()
        rhs0 = halves[0].calc_rhs()
        rhsf = full.calc_rhs()
        assert np.array_equal(rhs0, rhsf)
        # and the oracle's calc_rhs of the densities scaled from the integer grids
        cfg = O.make_cfg(case, full.sp)
        kq = O.kq_of(case.bcnd)
        npg = np.stack([O.np_from_acc(cfg, k, _acc_view(full, k).cpu().numpy().view(np.uint64), kq)
                        for k in range(2)])
        assert np.array_equal(O.calc_rhs(cfg, npg), rhsf)
    finally:
        for s in [full] + halves:
            s.close()


def test_dens_red_matches_oracle(gpu_lib):
    from jd_lepic_b200.simulation import GpuSimulation
    case = configs.case4(ppc=4, nx=128, ny=128)              # walls inside the box: np_mx over -1 nodes
    s = GpuSimulation(case, tile=(16, 16))
    try:
        for it in range(1, 4):
            s.step(it)
        s.sync()
        ntype = s.sp.ntype
        nn = (case.nx + 3) * (case.ny + 3)
        red = np.zeros(ntype * nn)
        mx = np.zeros(ntype)
        s.check(s.lib.lepic_gpu_dens_red(s.ctx, red.ctypes.data_as(C.POINTER(C.c_double)),
                                         mx.ctypes.data_as(C.POINTER(C.c_double))), "dens_red")
        npg = np.stack([s.grid(capi.GRID_NP + k) for k in range(ntype)])
        cfg = O.make_cfg(case, s.sp)
        ref, ref_mx = O.dens_red(cfg, npg, case.bcnd)
        assert np.array_equal(red.reshape(ref.shape), ref)
        assert np.array_equal(mx, ref_mx)
        assert (mx > 0).all()
    finally:
        s.close()
