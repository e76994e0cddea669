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


def _noalloc(lib, X, Y, VX, n, case, shift, k1, kq, stream):
    import torch
    nn = (case.nx + 3) * (case.ny + 3)
    out = torch.full((nn,), float("nan"), dtype=torch.float64, device=kq.device)
    ptr = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None
    rc = lib.lepic_gpu_deposit_noalloc(X if isinstance(X, C.c_void_p) else ptr(X),
                                       Y if isinstance(Y, C.c_void_p) else ptr(Y),
                                       VX if isinstance(VX, C.c_void_p) or VX is None else ptr(VX),
                                       n, case.nx, case.ny, shift, k1, ptr(kq), ptr(out), C.c_void_p(stream))
    assert rc == capi.OK
    return out


def test_deposit_noalloc_skips_holes_after_push(gpu_lib):
    """After a few steps without a sort the slot arrays hold holes (a lost particle's slot keeps
    its loss record in X and Y): with VX passed they are skipped and the grid still equals the
    context's deposit of the moved particles, bit for bit."""
    import torch
    from jd_lepic_b200.simulation import GpuSimulation
    from oracle import oracle as O

    case = configs.case0(ppc=8, nx=64, ny=64)
    s = GpuSimulation(case, tile=(8, 8))
    try:
        for it in range(1, 5):                     # step 1 sorts, steps 2-4 leave holes behind
            s.step(it)
        s.sync()
        st = s.push_stats()
        assert st["n_slots"][0] > st["np_tot"][0], st   # electrons were lost: holes exist
        dev = torch.device("cuda", torch.cuda.current_device())
        kq = torch.from_numpy(O.kq_of(case.bcnd).ravel()).to(dev)
        for sp in range(2):
            ref = s.grid(capi.GRID_NP + sp).ravel()
            X, Y, VX = C.c_void_p(), C.c_void_p(), C.c_void_p()
            n, shift = C.c_int64(), C.c_int32()
            s.check(s.lib.lepic_gpu_particle_arrays(s.ctx, sp, C.byref(X), C.byref(Y), C.byref(VX), None, None,
                                                    C.byref(n), C.byref(shift)), "particle_arrays")
            k1 = s.sp.Nm[sp] / (case.dx * case.dy * case.zmax)
            got = _noalloc(s.lib, X, Y, VX, n.value, case, shift.value, k1, kq, s.stream_ptr())
            s.sync()
            assert np.array_equal(got.cpu().numpy(), ref), sp
    finally:
        s.close()


def test_deposit_noalloc_skips_out_of_box_positions(gpu_lib):
    """VX = NULL on hole-free arrays built by the caller, with positions outside the box mixed
    in (at the far edges, past them, and at the largest uint32): those are skipped, so the grid
    equals the deposit of the in-box particles alone (bit for bit) and the oracle's FP64 CIC of
    them (to 1e-12 of the maximum)."""
    import torch
    from jd_lepic_b200.simulation import GpuSimulation
    from oracle import oracle as O

    case = configs.case0(ppc=2, nx=64, ny=64)
    s = GpuSimulation(case, tile=(8, 8), load=False)
    try:
        S = 24
        rng = np.random.default_rng(7)
        n_in = 20000
        xi = rng.integers(0, case.nx << S, n_in, dtype=np.int64)
        yi = rng.integers(0, case.ny << S, n_in, dtype=np.int64)
        bad = np.array([[case.nx << S, 5], [5, case.ny << S], [(case.nx << S) + 12345, 77],
                        [0xFFFFFFFF, 0xFFFFFFFF], [3, 0xFFFFFFFF], [(case.nx + 1) << S, (case.ny + 1) << S]],
                       dtype=np.int64)
        X_all = np.concatenate([xi, bad[:, 0]])
        Y_all = np.concatenate([yi, bad[:, 1]])
        perm = rng.permutation(X_all.size)
        X_all, Y_all = X_all[perm], Y_all[perm]
        dev = torch.device("cuda", torch.cuda.current_device())
        as_u32 = lambda a: torch.from_numpy(a.astype(np.uint32).view(np.int32)).to(dev)
        kq_np = O.kq_of(case.bcnd)
        kq = torch.from_numpy(kq_np.ravel()).to(dev)
        k1 = s.sp.Nm[0] / (case.dx * case.dy * case.zmax)
        stream = s.stream_ptr()
        got = _noalloc(s.lib, as_u32(X_all), as_u32(Y_all), None, X_all.size, case, S, k1, kq, stream)
        ref = _noalloc(s.lib, as_u32(xi), as_u32(yi), None, n_in, case, S, k1, kq, stream)
        s.sync()
        got, ref = got.cpu().numpy(), ref.cpu().numpy()
        assert np.array_equal(got, ref)
        p = np.zeros((n_in, 6))
        p[:, 0] = xi / float(1 << S) * case.dx
        p[:, 1] = yi / float(1 << S) * case.dy
        npg = np.zeros((case.ny + 3, case.nx + 3))
        O.deposit(O.make_cfg(case, s.sp), 0, p, n_in, kq_np, npg)
        assert np.abs(got.reshape(npg.shape) - npg).max() <= 1e-12 * np.abs(npg).max()
    finally:
        s.close()
