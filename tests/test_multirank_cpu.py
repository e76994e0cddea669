"""The multi-GPU exchange of the path, on CPU ranks (gloo, world size 2).

With particle decomposition (each rank owns a share of the particles at the deck's Nm, the grid
is replicated, calc_rho.f90:71-74 all-reduces rho), the device keeps rho as int64 fixed-point
CIC weights (2^-44, the layout of lepic_gpu_deposit_grid).  Integer addition is associative, so
the all-reduced grid must equal the grid of a single rank holding every particle, bit for bit,
whatever the reduction order, and so must the right-hand side formed from it.  The
accumulators here are oracle.int_deposit, the numpy restatement that
tests/test_gpu_decomposition.py pins to the library's own accumulator bit for bit."""
import os

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from jd_lepic_b200 import configs, deck as dk
from jd_lepic_b200.simulation import species_params
from oracle import oracle as O

NX = NY = 32
S = 24


def particles(n=20000, seed=3):
    rng = np.random.default_rng(seed)
    return (rng.integers(0, NX << S, n, dtype=np.int64), rng.integers(0, NY << S, n, dtype=np.int64))


def _rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    X, Y = particles()
    part = slice(rank, None, world)  # an arbitrary particle decomposition
    acc = O.int_deposit(X[part], Y[part], NX, NY, S).view(np.int64)
    t = torch.from_numpy(acc.copy())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    if rank == 0:
        np.save(out, t.numpy())
    dist.barrier()
    dist.destroy_process_group()


def test_int64_rho_allreduce_is_exact(tmp_path):
    out = str(tmp_path / "acc.npy")
    port = 29500 + (os.getpid() % 1000)
    mp.spawn(_rank, args=(2, port, out), nprocs=2, join=True)
    X, Y = particles()
    ref = O.int_deposit(X, Y, NX, NY, S).view(np.int64)
    got = np.load(out)
    assert np.array_equal(got, ref)
    # and the weights of each particle sum to 2^44 up to the rounding of four terms
    assert abs(int(ref.sum()) - len(X) * (1 << O.DEP_SHIFT)) <= 2 * len(X)
    # the right-hand side formed from the reduced grid is the single rank's
    case = configs.case0(ppc=2, nx=NX, ny=NY)
    cfg = O.make_cfg(case, species_params(case, dk.read_reactions(case.deck_text, case.ngas)))
    kq = O.kq_of(case.bcnd)
    rhs_red = O.calc_rhs(cfg, np.stack([O.np_from_acc(cfg, 0, got.view(np.uint64), kq)] * 2))
    rhs_one = O.calc_rhs(cfg, np.stack([O.np_from_acc(cfg, 0, ref.view(np.uint64), kq)] * 2))
    assert np.array_equal(rhs_red, rhs_one)


def test_rank_load_counts_follow_the_reference():
    """load_part.f90:96: each of nproc_mpi ranks loads NINT(np_cell n_cell / nproc_mpi), at the
    Nm of the deck's np_cell (main.f90:471)."""
    case = configs.case0(ppc=25, nx=32, ny=32)
    d = dk.read_reactions(case.deck_text, case.ngas)
    nm1 = species_params(case, d).Nm[0]
    case.nproc_mpi = 3
    assert case.n_load == int(np.floor(25 * 32 * 32 / 3 + 0.5))
    assert species_params(case, d).Nm[0] == nm1
