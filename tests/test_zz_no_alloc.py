"""lepic_gpu_deposit_noalloc: the charge deposition for callers that cannot call cudaMalloc
(their device memory is reserved up front and handed out by their own allocator, or an
allocation's implicit synchronisation is not allowed where they deposit).  The caller passes
only buffers it owns; the accumulator is the library's fixed static device array.

Checked through the C ABI against the context path (lepic_gpu_charge_deposition, read back with
lepic_gpu_get_grid) on two calls in a row: the second call must not see the first call's sums.
This file is collected last so that a run stopping at the first failure has run the rest."""
import ctypes as C

import numpy as np
import pytest

from jd_lepic_b200 import _capi as capi, configs

pytestmark = pytest.mark.gpu


def test_deposit_noalloc_matches_context_path(gpu_lib):
    import torch
    from jd_lepic_b200.simulation import GpuSimulation
    from oracle import oracle as O

    case = configs.case0(ppc=8, nx=64, ny=64)
    s = GpuSimulation(case, tile=(8, 8))          # loads and deposits through the context
    lib = s.lib
    dev = torch.device("cuda", torch.cuda.current_device())
    kq = torch.from_numpy(O.kq_of(case.bcnd).ravel()).to(dev)
    nn = (case.nx + 3) * (case.ny + 3)
    k1 = [s.sp.Nm[k] / (case.dx * case.dy * case.zmax) for k in range(2)]
    stream = s.stream_ptr()
    for sp in range(2):
        ref = s.grid(capi.GRID_NP + sp).ravel()        # the context path's np grid
        X, Y, VX = C.c_void_p(), C.c_void_p(), C.c_void_p()
        n, shift = C.c_int64(), C.c_int32()
        s.check(lib.lepic_gpu_particle_arrays(s.ctx, sp, C.byref(X), C.byref(Y), C.byref(VX), None, None,
                                              C.byref(n), C.byref(shift)), "particle_arrays")
        for call in range(2):                          # two calls in a row share the scratch
            out = torch.full((nn,), float("nan"), dtype=torch.float64, device=dev)
            rc = lib.lepic_gpu_deposit_noalloc(X, Y, VX, n.value, case.nx, case.ny, shift.value, k1[sp],
                                               C.c_void_p(kq.data_ptr()), C.c_void_p(out.data_ptr()),
                                               C.c_void_p(stream))
            assert rc == capi.OK
            s.sync()
            got = out.cpu().numpy()
            assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max(), (sp, call)
            assert np.array_equal(got, ref)
    s.close()


def test_deposit_noalloc_rejects_oversized_grid(gpu_lib):
    lib = gpu_lib
    # (nx+3)*(ny+3) above the 2^20-node static scratch: refused before any launch
    rc = lib.lepic_gpu_deposit_noalloc(None, None, None, 0, 2048, 2048, 20, 1.0, C.c_void_p(1), C.c_void_p(1),
                                       None)
    assert rc == capi.ECAPACITY
