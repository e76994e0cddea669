"""The learned Poisson warm start on the GPU, through the C ABI.

* The tensor-core network (forward output, loss and every parameter gradient) against the
  CPU oracle in BF16-emulation mode on the same weights and inputs.  The tolerance covers
  FP32 accumulation in a different order than the oracle's exact sums, which can move a
  BF16-stored activation by one unit in the last place (2^-8 relative).
* Adam steps on a fixed batch lower the loss.
* A/B on PIC steps: after online training, the learned mode keeps its prediction, lowers the
  starting residual and needs no more CG iterations than the plain mixed-precision solve
  from the previous potential, reaching the same residual."""
import ctypes as C

import numpy as np
import pytest

from jd_lepic_b200 import _capi as capi, configs
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FP = C.POINTER(C.c_float)


def fp(a):
    return a.ctypes.data_as(FP) if a is not None else None


@pytest.fixture(scope="module")
def net(gpu_lib):
    import torch
    torch.cuda.init()
    h = C.c_void_p()
    assert gpu_lib.lepic_cnn_create(C.byref(h), 5) == capi.OK
    yield gpu_lib, h
    gpu_lib.lepic_cnn_destroy(h)


def _set(lib, h, p):
    p32 = np.ascontiguousarray(p, dtype=np.float32)
    assert lib.lepic_cnn_params(h, fp(p32), p32.size, 1) == capi.OK
    return p32.astype(np.float64)


def _gpu_loss_grad(lib, h, x, t, m):
    N, H, W = t.shape
    x32 = np.ascontiguousarray(x, dtype=np.float32)
    t32 = np.ascontiguousarray(t, dtype=np.float32)
    m32 = np.ascontiguousarray(m, dtype=np.float32)
    out = np.zeros((N, H, W), np.float32)
    g = np.zeros(O.cnn_nparams(), np.float32)
    L = C.c_double()
    rc = lib.lepic_cnn_loss_grad(h, fp(x32), fp(t32), fp(m32), N, H, W, fp(out), fp(g), C.byref(L))
    assert rc == capi.OK, lib.lepic_cnn_last_error(h)
    return L.value, out.astype(np.float64), g.astype(np.float64)


def _layers():
    k = 0
    for ci, co in zip(O.CNN_CIN, O.CNN_COUT):
        yield k, k + co * ci * 9, k + co * ci * 9 + co
        k += co * ci * 9 + co


@pytest.mark.parametrize("N,H,W", [(2, 16, 24), (1, 40, 136)])
def test_network_matches_oracle(net, N, H, W):
    lib, h = net
    rng = np.random.default_rng(N * 100 + H)
    p = O.cnn_init_params(N + H)
    p[np.arange(p.size) % 11 == 0] += 0.05          # biases away from zero
    p = _set(lib, h, p)
    x = rng.standard_normal((N, H, W, 2))
    t = rng.standard_normal((N, H, W))
    m = (rng.random((N, H, W)) > 0.1).astype(np.float64)
    Lg, outg, gg = _gpu_loss_grad(lib, h, x, t, m)
    Lo, outo, go = O.cnn_loss_grad(p, x, t, m, emulate_bf16=True)
    assert np.linalg.norm(outg - outo) <= 1e-2 * np.linalg.norm(outo)
    assert np.abs(outg - outo).max() <= 5e-2 * np.abs(outo).max()
    assert abs(Lg - Lo) <= 1e-2 * Lo
    for l, (a, b, c) in enumerate(_layers()):
        dw = np.linalg.norm(gg[a:b] - go[a:b]) / max(np.linalg.norm(go[a:b]), 1e-30)
        db = np.linalg.norm(gg[b:c] - go[b:c]) / max(np.linalg.norm(go[b:c]), 1e-30)
        assert dw <= 3e-2, (l, dw)
        assert db <= 3e-2 or np.linalg.norm(go[b:c]) < 1e-6 * np.linalg.norm(go), (l, db)


def test_forward_only_matches_training_forward(net):
    lib, h = net
    rng = np.random.default_rng(2)
    _set(lib, h, O.cnn_init_params(4))
    x = rng.standard_normal((1, 32, 48, 2)).astype(np.float32)
    out = np.zeros((1, 32, 48), np.float32)
    assert lib.lepic_cnn_loss_grad(h, fp(x), None, None, 1, 32, 48, fp(out), None, None) == capi.OK
    t = np.zeros((1, 32, 48)); m = np.ones((1, 32, 48))
    _, out2, _ = _gpu_loss_grad(lib, h, x, t, m)
    assert np.array_equal(out, out2.astype(np.float32))


def test_adam_lowers_the_loss(net):
    lib, h = net
    rng = np.random.default_rng(3)
    _set(lib, h, O.cnn_init_params(9))
    N, H, W = 2, 32, 32
    r = rng.standard_normal((N, H, W))
    x = np.stack([r, np.zeros_like(r)], -1)
    t = np.cumsum(np.cumsum(r, 1), 2) * 0.05        # a smooth response of the input
    m = np.ones((N, H, W))
    L0 = _gpu_loss_grad(lib, h, x, t, m)[0]
    for _ in range(30):
        _gpu_loss_grad(lib, h, x, t, m)
        assert lib.lepic_cnn_adam_step(h, C.c_float(2e-3)) == capi.OK
    L1 = _gpu_loss_grad(lib, h, x, t, m)[0]
    assert L1 < 0.5 * L0, (L0, L1)


def test_learned_warm_start_saves_iterations(gpu_lib):
    from jd_lepic_b200.simulation import GpuSimulation
    case = configs.case4(ppc=20, nx=256, ny=256)
    s = GpuSimulation(case, tile=(16, 16))
    cfg = capi.LepicCnnConfig(enable_training=1, warmup_solves=1000, steps_warmup=3, train_every=1, steps_after=1,
                              crop=128, batch=4, lr=C.c_float(2e-3), seed=11)
    s.check(s.lib.lepic_gpu_cnn_configure(s.ctx, C.byref(cfg)), "cnn_configure")
    eps = 1e-8
    it = 1
    for _ in range(80):                       # PIC steps with online training
        it += 1
        s.check(s.lib.lepic_gpu_step(s.ctx, it, eps, capi.POISSON_LEARNED), "step")
    # A/B on the next steps: same right-hand side, same starting potential
    plain, learned, ratios = [], [], []
    for _ in range(6):
        it += 1
        s.check(s.lib.lepic_gpu_calc_rhs(s.ctx, None), "calc_rhs")
        phi_prev = s.grid(capi.GRID_PHI).copy()
        st_p = s.solve(eps=eps, mode=capi.POISSON_MIXED_IR)
        s.set_phi(phi_prev)
        st_l = s.solve(eps=eps, mode=capi.POISSON_LEARNED)
        cs = capi.LepicCnnStats()
        s.check(s.lib.lepic_gpu_cnn_stats(s.ctx, C.byref(cs)), "cnn_stats")
        assert st_p["res_l2_rel"] <= eps and st_l["res_l2_rel"] <= eps
        plain.append(st_p["cycles"]); learned.append(st_l["cycles"]); ratios.append(cs.last_res_ratio)
        s.check(s.lib.lepic_gpu_calc_efield(s.ctx, None), "efield")
        s.push(it)
    print("plain", plain, "learned", learned, "residual ratios", np.round(ratios, 3))
    assert max(ratios) < 0.5, ratios
    assert sum(learned) <= sum(plain) and min(learned) < max(plain), (plain, learned)
    s.close()
