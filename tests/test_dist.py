"""Multi-rank logic of spsim_b200.dist on CPU with the gloo backend (world size 2):
unit assignment, sharded forward with no collective, gather to one rank,
gradient all-reduce (against the FP64 oracle's VJP over all orientations),
and a rank that dies before a collective."""
import os
import socket
import tempfile

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from spsim_b200 import dist as D


def test_slab_range_matches_reference_split():
    # src/mpi.c:30-48: floor splits, the last rank takes the remainder
    assert [D.slab_range(10, r, 3) for r in range(3)] == [(0, 3), (3, 6), (6, 10)]
    assert [D.slab_range(2, r, 4) for r in range(4)] == [(0, 0), (0, 1), (1, 1), (1, 2)]


def test_balanced_assignment_covers_and_balances():
    rng = np.random.default_rng(0)
    costs = list(np.exp(rng.uniform(np.log(500), np.log(1e5), 64)) * rng.choice([128 ** 2, 1024 ** 2], 64))
    parts = D.balanced_assignment(costs, 8)
    assert sorted(i for p in parts for i in p) == list(range(64))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) <= (sum(costs) / 8) + max(costs)  # LPT bound


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, fn, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=20))
    try:
        fn(rank, world, out_dir)
    finally:
        if dist.is_initialized():
            dist.destroy_process_group()


def _run(fn, world=2):
    with tempfile.TemporaryDirectory() as td:
        mp.start_processes(_worker, args=(world, _free_port(), fn, td), nprocs=world, join=True,
                           start_method="spawn")
        return {f: np.load(os.path.join(td, f), allow_pickle=True) for f in os.listdir(td)}


def _case():
    from oracle import oracle as O
    from spsim_b200 import synth

    Z, pos = synth.random_molecule(30, 1.0e-9, 4)
    R = synth.haar_rotations(5, 9)
    q0 = O.hkl_detector(8, 8, 8 * 600e-6, 8 * 600e-6, 0.1, 0.2e-9)
    return Z, pos, R, q0


def _sharded_forward_and_gather(rank, world, out):
    from oracle import oracle as O

    Z, pos, R, q0 = _case()
    local = D.forward_sharded(len(R), lambda i: torch.from_numpy(
        O.structure_factor(Z, pos.astype(np.float64), q0 @ R[i].T, nthreads=1)[1]))
    full = D.gather_to(local, len(R), (q0.shape[0],), torch.float64, dst=0)
    np.save(os.path.join(out, "mine_%d.npy" % rank), np.array(sorted(local)))
    if rank == 0:
        np.save(os.path.join(out, "full.npy"), full.numpy())


def test_sharded_forward_gather_equals_single_process():
    from oracle import oracle as O

    res = _run(_sharded_forward_and_gather)
    Z, pos, R, q0 = _case()
    assert list(res["mine_0.npy"]) == [0, 1] and list(res["mine_1.npy"]) == [2, 3, 4]
    ref = np.stack([O.structure_factor(Z, pos.astype(np.float64), q0 @ r.T)[1] for r in R])
    np.testing.assert_allclose(res["full.npy"], ref, rtol=1e-12)


def _sharded_orientation_batch(rank, world, out):
    from oracle import oracle as O

    Z, pos, R, q0 = _case()

    def batch(rots):  # stands in for a batched GPU call (forward_nufft_batch / forward_batch)
        return torch.from_numpy(np.stack([O.structure_factor(Z, pos.astype(np.float64), q0 @ r.T, nthreads=1)[1]
                                          for r in rots]))

    local, (s, e) = D.sharded_orientations(R, batch)
    np.save(os.path.join(out, "range_%d.npy" % rank), np.array([s, e]))
    full = D.gather_to(local, len(R), (q0.shape[0],), torch.float64)
    if rank == 0:
        np.save(os.path.join(out, "full.npy"), full.numpy())


def test_sharded_orientation_batch_gather_equals_single_process():
    from oracle import oracle as O

    res = _run(_sharded_orientation_batch)
    Z, pos, R, q0 = _case()
    assert list(res["range_0.npy"]) == [0, 2] and list(res["range_1.npy"]) == [2, 5]
    ref = np.stack([O.structure_factor(Z, pos.astype(np.float64), q0 @ r.T)[1] for r in R])
    np.testing.assert_allclose(res["full.npy"], ref, rtol=1e-12)


def _sharded_pixel_slabs(rank, world, out):
    from oracle import oracle as O

    Z, pos, R, q0 = _case()
    q = (q0 @ R[0].T)[:61]  # 61 pixels: uneven slabs, the last rank takes the remainder

    def slab(s, e):  # stands in for a GPU forward over the pixel slab
        F, I = O.structure_factor(Z, pos.astype(np.float64), q[s:e], nthreads=1)
        return torch.from_numpy(np.stack([F.real, F.imag, I], axis=1))

    full, local, (s, e) = D.sharded_pixels(q.shape[0], slab)
    np.save(os.path.join(out, "range_%d.npy" % rank), np.array([s, e, local.shape[0]]))
    if rank == 0:
        np.save(os.path.join(out, "full.npy"), full.numpy())
    else:
        assert full is None


def test_one_pattern_split_in_pixel_slabs_equals_single_process():
    # spsim's MPI split of one HKL list (src/mpi.c:30-48) and the gather to the
    # master (src/mpi.c:96-117), on three gloo ranks
    from oracle import oracle as O

    res = _run(_sharded_pixel_slabs, world=3)
    Z, pos, R, q0 = _case()
    q = (q0 @ R[0].T)[:61]
    assert [list(res["range_%d.npy" % r]) for r in range(3)] == [[0, 20, 20], [20, 40, 20], [40, 61, 21]]
    F, I = O.structure_factor(Z, pos.astype(np.float64), q)
    np.testing.assert_allclose(res["full.npy"], np.stack([F.real, F.imag, I], axis=1), rtol=1e-12, atol=0)


def _balanced_gather(rank, world, out):
    costs = [5.0, 1.0, 1.0, 1.0, 1.0]  # rank 0 takes unit 0, rank 1 the other four
    local = D.forward_sharded(len(costs), lambda i: torch.full((3,), float(i)), costs=costs)
    np.save(os.path.join(out, "mine_%d.npy" % rank), np.array(sorted(local)))
    full = D.gather_to(local, len(costs), (3,), torch.float32)
    if rank == 0:
        np.save(os.path.join(out, "full.npy"), full.numpy())


def test_gather_of_cost_balanced_units():
    # non-contiguous unit sets of different sizes per rank, reassembled in order on rank 0
    res = _run(_balanced_gather)
    mine = [list(res["mine_%d.npy" % r]) for r in range(2)]
    assert mine == [[0], [1, 2, 3, 4]]
    np.testing.assert_array_equal(res["full.npy"], np.repeat(np.arange(5, dtype=np.float32)[:, None], 3, axis=1))


def _gradient_allreduce(rank, world, out):
    from oracle import oracle as O

    Z, pos, R, q0 = _case()
    s, e = D.slab_range(len(R), rank, world)
    q = np.concatenate([q0 @ r.T for r in R[s:e]])
    g = np.linspace(-1, 1, q.shape[0])
    dp, do, db = O.structure_factor_vjp(Z, pos.astype(np.float64), q, g, nthreads=1)
    t = [torch.from_numpy(dp.copy()), torch.from_numpy(do.copy())]
    D.allreduce_(*t)
    np.save(os.path.join(out, "dpos_%d.npy" % rank), t[0].numpy())
    # the autograd hook: identity forward, summed gradient backward
    x = torch.ones(3, dtype=torch.float64, requires_grad=True)
    y = D._AllReduceGrad.apply(x, None)
    (y * (rank + 1)).sum().backward()
    np.save(os.path.join(out, "xgrad_%d.npy" % rank), x.grad.numpy())


def test_gradient_allreduce_equals_global_vjp():
    from oracle import oracle as O

    res = _run(_gradient_allreduce)
    Z, pos, R, q0 = _case()
    parts = []
    for rank in range(2):
        s, e = D.slab_range(len(R), rank, 2)
        parts.append(np.concatenate([q0 @ r.T for r in R[s:e]]))
    g = np.concatenate([np.linspace(-1, 1, p.shape[0]) for p in parts])
    dp, _, _ = O.structure_factor_vjp(Z, pos.astype(np.float64), np.concatenate(parts), g)
    for rank in range(2):
        np.testing.assert_allclose(res["dpos_%d.npy" % rank], dp, rtol=1e-10, atol=1e-12 * np.abs(dp).max())
        np.testing.assert_allclose(res["xgrad_%d.npy" % rank], np.full(3, 3.0))


def _rank_dies(rank, world, out):
    import time

    if rank == 1:
        raise SystemExit(0)  # leaves before the collective, between steps
    t = torch.ones(4)
    t0 = time.time()
    try:
        dist.all_reduce(t)
        np.save(os.path.join(out, "status.npy"), np.array(["completed"]))
    except Exception as exc:  # noqa: BLE001 - the failure is the point
        np.save(os.path.join(out, "status.npy"), np.array(["error: %s" % type(exc).__name__, time.time() - t0]))


def test_dead_rank_surfaces_as_collective_error():
    with tempfile.TemporaryDirectory() as td:
        port = _free_port()
        ctx = mp.get_context("spawn")
        procs = [ctx.Process(target=_worker, args=(r, 2, port, _rank_dies, td)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(60)
        for p in procs:
            if p.is_alive():
                p.kill()
        st = np.load(os.path.join(td, "status.npy"), allow_pickle=True)
    assert str(st[0]).startswith("error"), st
