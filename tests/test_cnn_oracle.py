"""The CPU restatement of the warm-start network (oracle/cnn_oracle.c): its backward pass
against central finite differences of its own loss (double precision, no BF16 rounding), and
its BF16-emulation mode against the exact mode."""
import numpy as np
import pytest

from oracle import oracle as O


@pytest.fixture(scope="module")
def problem():
    rng = np.random.default_rng(7)
    p = O.cnn_init_params(3)
    p += 0.02 * rng.standard_normal(p.size)       # non-zero biases too
    N, H, W = 2, 16, 24
    x = rng.standard_normal((N, H, W, 2))
    t = rng.standard_normal((N, H, W))
    m = (rng.random((N, H, W)) > 0.15).astype(float)
    return p, x, t, m


def test_parameter_count():
    assert O.cnn_nparams() == sum(co * ci * 9 + co for ci, co in zip(O.CNN_CIN, O.CNN_COUT)) == 205953


def test_backward_matches_finite_differences(problem):
    p, x, t, m = problem
    L, out, g = O.cnn_loss_grad(p, x, t, m, emulate_bf16=False)
    assert np.isfinite(L) and L > 0
    rng = np.random.default_rng(11)
    # coordinates in every layer (first, middle and last weight, first bias), plus random ones
    offs, k = [], 0
    for ci, co in zip(O.CNN_CIN, O.CNN_COUT):
        offs += [k, k + co * ci * 9 // 2, k + co * ci * 9]
        k += co * ci * 9 + co
    idx = np.unique(np.concatenate([offs, rng.choice(p.size, 24, replace=False)]))
    worst = 0.0
    scale = np.abs(g).max()
    for i in idx:
        h = 1e-6
        pp = p.copy(); pp[i] += h
        pm = p.copy(); pm[i] -= h
        fd = (O.cnn_loss_grad(pp, x, t, m, False, False)[0] - O.cnn_loss_grad(pm, x, t, m, False, False)[0]) / (2 * h)
        worst = max(worst, abs(fd - g[i]) / scale)
    assert worst < 1e-6, worst


def test_bf16_emulation_close_to_exact(problem):
    p, x, t, m = problem
    Le, oute, ge = O.cnn_loss_grad(p, x, t, m, emulate_bf16=True)
    Lx, outx, gx = O.cnn_loss_grad(p, x, t, m, emulate_bf16=False)
    assert abs(Le - Lx) <= 0.05 * Lx
    assert np.linalg.norm(oute - outx) <= 0.05 * np.linalg.norm(outx)
    assert np.linalg.norm(ge - gx) <= 0.1 * np.linalg.norm(gx)
