"""The multi-GPU exchange of the path, on CPU ranks (gloo, world size 2).

With particle decomposition (each rank owns a share of the particles, the grid is replicated,
calc_rho.f90:71-74 all-reduces rho), the device keeps rho as int64 fixed-point CIC weights
(2^-44).  Integer addition is associative, so the all-reduced grid must equal the grid of a
single rank holding every particle, bit for bit, whatever the reduction order.  The weights
below follow the device's integer formula (products of the fixed-point offsets)."""
import os

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

NX = NY = 32
S = 24
SHIFT = 44


def int_deposit(X, Y):
    """uint64 CIC accumulation of the device (push.cu: deposit_warp) in numpy."""
    W = NX + 3
    acc = np.zeros((NY + 3) * W, dtype=np.uint64)
    mask = (1 << S) - 1
    A = 1 << S
    fx = (X & mask).astype(np.uint64)
    fy = (Y & mask).astype(np.uint64)
    ax, ay = np.uint64(A) - fx, np.uint64(A) - fy
    sh = 2 * S - SHIFT
    ix = (X >> S).astype(np.int64) + 1
    iy = (Y >> S).astype(np.int64) + 1
    for w, dx, dy in ((ax * ay, 0, 0), (fx * ay, 1, 0), (fx * fy, 1, 1), (ax * fy, 0, 1)):
        w = (w + np.uint64(1 << (sh - 1))) >> np.uint64(sh)
        np.add.at(acc, (ix + dx) + (iy + dy) * W, w)
    return acc


def particles(n=20000, seed=3):
    rng = np.random.default_rng(seed)
    return (rng.integers(0, NX << S, n, dtype=np.int64), rng.integers(0, NY << S, n, dtype=np.int64))


def _rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    X, Y = particles()
    part = slice(rank, None, world)  # an arbitrary particle decomposition
    acc = int_deposit(X[part], Y[part]).view(np.int64)
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
    ref = int_deposit(X, Y).view(np.int64)
    got = np.load(out)
    assert np.array_equal(got, ref)
    # and the weights of each particle sum to 2^44 up to the rounding of four terms
    assert abs(int(ref.sum()) - len(X) * (1 << SHIFT)) <= 2 * len(X)
