"""Multi-GPU work distribution over torch.distributed (one process per GPU).

The forward path shards: orientations, molecules and pixel slabs are
independent, so ranks split the units and compute with no collective on the
data path (weak or strong scaling).  The only exchange is the adjoint's sum of
per-rank gradients (one all-reduce), plus an optional gather of patterns to
one rank, the analogue of spsim's MPI gather to the master
(src/mpi.c:50-60, :96-117).

Unit assignment:
  slab_range          contiguous equal slabs, spsim's own split (src/mpi.c:30-48)
  balanced_assignment cost-balanced (longest-processing-time first) for
                      uneven units such as molecules of different sizes

One large pattern (sharded_pixels) is split into contiguous pixel slabs, one
per rank, as spsim's MPI build splits its HKL list; gathers move each rank's
own slab only (gather_to, gather_slab): rank dst receives world slabs of the
largest slab's size, every other rank sends just its own.
"""
import heapq

import torch
import torch.distributed as dist

__all__ = ["slab_range", "balanced_assignment", "rank_world", "forward_sharded", "sharded_orientations",
           "sharded_pixels", "gather_slab", "gather_to", "allreduce_", "sharded_intensity"]


def rank_world(group=None):
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(group), dist.get_world_size(group)
    return 0, 1


def slab_range(size, rank, world):
    """[start, end) of `rank`'s contiguous slab; the last rank takes the remainder (src/mpi.c:30-48)."""
    start = rank * size // world
    end = size if rank == world - 1 else (rank + 1) * size // world
    return start, end


def balanced_assignment(costs, world):
    """Unit indices per rank: each unit, largest first, goes to the least-loaded rank.
    Deterministic, so every rank computes the same assignment without communicating."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(world)]
    out = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(v) for v in out]


def forward_sharded(units, compute, costs=None, group=None):
    """Run compute(unit_index) for this rank's units; returns {index: result}.

    With costs, units are cost-balanced across ranks, else split in contiguous
    slabs.  No collective is issued."""
    rank, world = rank_world(group)
    n = len(units) if hasattr(units, "__len__") else int(units)
    if costs is not None:
        mine = balanced_assignment(costs, world)[rank]
    else:
        s, e = slab_range(n, rank, world)
        mine = range(s, e)
    return {i: compute(i) for i in mine}


def sharded_orientations(rots, compute_batch, group=None):
    """This rank's contiguous slab of orientations in one batched call, e.g.
    compute_batch = lambda r: core.forward_nufft_batch(mol, qs, r)[1] (one NUFFT
    grid per rank for all its orientations) or a core.forward_batch call.
    Returns ({index: pattern}, (start, end)); no collective is issued."""
    rank, world = rank_world(group)
    s, e = slab_range(len(rots), rank, world)
    if e <= s:
        return {}, (s, e)
    out = compute_batch(rots[s:e])
    return {s + i: out[i] for i in range(e - s)}, (s, e)


def gather_slab(local, size, dst=0, group=None):
    """Reassemble a unit axis of length `size` split by slab_range on rank dst.

    local: this rank's contiguous slab, a tensor of shape (end - start, ...).
    Every rank knows every slab's extent from slab_range, so each sends one
    buffer of the largest slab's length (its own rows, then padding) and rank
    dst keeps the first (end - start) rows of each (spsim's mpi_receive_pattern,
    src/mpi.c:96-117).  Returns the (size, ...) tensor on dst, None elsewhere."""
    rank, world = rank_world(group)
    if world == 1:
        return local
    ranges = [slab_range(size, r, world) for r in range(world)]
    s, e = ranges[rank]
    if local.shape[0] != e - s:
        raise ValueError("rank %d holds %d rows of its slab [%d, %d)" % (rank, local.shape[0], s, e))
    width = max(b - a for a, b in ranges)
    buf = torch.zeros((width,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    buf[: e - s] = local
    parts = [torch.empty_like(buf) for _ in range(world)] if rank == dst else None
    dist.gather(buf, parts, dst=dst, group=group)
    if rank != dst:
        return None
    return torch.cat([parts[r][: b - a] for r, (a, b) in enumerate(ranges)])


def sharded_pixels(npix, compute_slab, dst=0, group=None, gather=True):
    """One pattern split across ranks in contiguous pixel slabs, spsim's own
    split of its HKL list (get_my_loop_start_and_end, src/mpi.c:30-48): this
    rank computes compute_slab(start, end) -> tensor (end - start, ...) for
    [start, end) = slab_range(npix, rank, world), e.g.
        lambda s, e: core.forward(mol, core.QSet.from_list(hkl[s:e]))[1]
    and, with gather, the slabs are reassembled on rank dst (gather_slab).
    Returns (full pattern on dst or None, local slab, (start, end)); the only
    collective is the gather."""
    rank, world = rank_world(group)
    s, e = slab_range(npix, rank, world)
    local = compute_slab(s, e)
    full = gather_slab(local, npix, dst=dst, group=group) if gather else None
    return full, local, (s, e)


def gather_to(local, n_units, shape, dtype, dst=0, group=None, device=None):
    """Gather {index: tensor} from all ranks into one (n_units, *shape) tensor on rank dst.

    The assignment may be any (contiguous slabs or cost-balanced): each rank
    packs its own units and their indices into buffers of the largest rank's
    unit count (one small all-reduce finds it) and rank dst scatters what it
    gathers into place, so no rank but dst holds more than its own units."""
    rank, world = rank_world(group)
    dev = device or (next(iter(local.values())).device if local else torch.device("cpu"))
    if world == 1:
        buf = torch.zeros((n_units,) + tuple(shape), dtype=dtype, device=dev)
        for i, t in local.items():
            buf[i] = t
        return buf
    cnt = torch.tensor([len(local)], dtype=torch.int64, device=dev)
    dist.all_reduce(cnt, op=dist.ReduceOp.MAX, group=group)
    width = max(int(cnt.item()), 1)
    vals = torch.zeros((width,) + tuple(shape), dtype=dtype, device=dev)
    idx = torch.full((width,), -1, dtype=torch.int64, device=dev)
    for k, (i, t) in enumerate(sorted(local.items())):
        vals[k] = t
        idx[k] = i
    pv = [torch.empty_like(vals) for _ in range(world)] if rank == dst else None
    pi = [torch.empty_like(idx) for _ in range(world)] if rank == dst else None
    dist.gather(idx, pi, dst=dst, group=group)
    dist.gather(vals, pv, dst=dst, group=group)
    if rank != dst:
        return None
    out = torch.zeros((n_units,) + tuple(shape), dtype=dtype, device=dev)
    for v, ix in zip(pv, pi):
        keep = ix >= 0
        out[ix[keep]] = v[keep]
    return out


def allreduce_(*tensors, group=None):
    """Sum tensors over ranks in place (the adjoint's gradient exchange)."""
    _, world = rank_world(group)
    if world > 1:
        for t in tensors:
            if t is not None:
                dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return tensors


class _AllReduceGrad(torch.autograd.Function):
    """Identity in the forward; sums the incoming gradient over ranks in the backward."""

    @staticmethod
    def forward(ctx, x, group):
        ctx.group = group
        return x.view_as(x)

    @staticmethod
    def backward(ctx, g):
        g = g.contiguous().clone()
        allreduce_(g, group=ctx.group)
        return g, None


def sharded_intensity(mol, qs, pos, occ, bfac, rots, precision="f32", group=None):
    """Differentiable intensities of this rank's slab of orientations.

    Returns (I_local (n_local, npix), (start, end)).  Losses summed over the
    local patterns and backpropagated give every rank the gradient of the
    global loss (sum over ranks), through one all-reduce per parameter."""
    from .autograd import intensity

    rank, world = rank_world(group)
    if len(rots) < world:
        raise ValueError("every rank needs at least one orientation (%d orientations, %d ranks)" % (len(rots), world))
    s, e = slab_range(len(rots), rank, world)
    p = _AllReduceGrad.apply(pos, group)
    o = _AllReduceGrad.apply(occ, group) if occ is not None else None
    b = _AllReduceGrad.apply(bfac, group) if bfac is not None else None
    return intensity(mol, qs, p, o, b, rots=rots[s:e], precision=precision), (s, e)
