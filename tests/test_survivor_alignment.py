"""The survivor alignment the push parity tests rely on (oracle.align_survivors): two
order-preserving compactions of one particle array that differ in a few losses are paired
particle by particle, and every other particle is compared."""
import numpy as np
import pytest

from jd_lepic_b200 import configs, deck as dk
from jd_lepic_b200.simulation import species_params
from oracle import oracle as O


def _moved(seed=3, n=4000):
    case = configs.case0(ppc=1, nx=32, ny=32)
    sp = species_params(case, dk.read_reactions(case.deck_text, case.ngas))
    cfg = O.make_cfg(case, sp)
    rng = np.random.default_rng(seed)
    p = np.zeros((n, 6))
    p[:, 0] = rng.uniform(0, case.nx * case.dx, n)
    p[:, 1] = rng.uniform(0, case.ny * case.dy, n)
    p[:, 3:] = rng.normal(0, 3 * sp.vt0[0], (n, 3))
    E = np.zeros((case.ny + 3, case.nx + 3, 2))
    ref, ids, t = O.mover_tagged(cfg, 0, E, None, case.bcnd, p)
    return case, p, ref, ids, t


def test_mover_tagged_ids_are_the_survivors():
    case, p, ref, ids, t = _moved()
    assert t.n_lost > 0 and ids.size == p.shape[0] - t.n_lost
    assert np.all(np.diff(ids) > 0)                       # order preserved
    assert np.all(ref[:, 2] == 0.0)
    assert np.allclose(ref[:, 3:], p[ids, 3:])            # no field: velocities unchanged


@pytest.mark.parametrize("drop_ref,drop_got", [((), ()), ((5, 900), ()), ((), (17,)), ((40,), (41, 2000))])
def test_align_survivors_pairs_all_common_particles(drop_ref, drop_got):
    case, p, ref, ids, _ = _moved()
    got = ref.copy()
    # a "device" that lost ref rows drop_ref and kept extra particles after rows drop_got
    keep = np.ones(ref.shape[0], dtype=bool)
    keep[list(drop_ref)] = False
    rows = []
    for k in range(ref.shape[0]):
        if keep[k]:
            rows.append(got[k])
        if k in drop_got:
            extra = got[k].copy()
            extra[0] += 0.37 * case.dx
            rows.append(extra)
    dev = np.array(rows) + 1e-9 * case.dx                 # a rounding-sized difference
    gi, rj, g_only, r_only = O.align_survivors(dev, ref, case.dx, case.dy)
    assert r_only == len(drop_ref) and g_only == len(drop_got)
    assert gi.size == rj.size == ref.shape[0] - len(drop_ref)
    assert np.abs(dev[gi, :2] - ref[rj, :2]).max() <= 1e-6 * case.dx
    assert not np.isin(np.array(drop_ref, dtype=np.int64), rj).any()
