"""Partition of a plan's dose calculation across GPUs (one process per GPU).

Beams are independent in FastDose's dose path: a beamlet's Terma, CCCS and
column touch only its own BEV volumes and the shared, read-only density
(IMRTOpt/src/IMRTDoseMat.cu:26-140 loops over beams with nothing carried
between them).  So a plan shards by beams with no collective on the data
path:

- `beam_costs` prices a beam by the CCCS march it needs: the sum over its
  beamlets of (fluence-map pixels x long_dim), the voxels every zenith pass
  walks;
- `partition_beams` assigns beams to ranks greedily, largest first, each to
  the least loaded rank (longest-processing-time rule); ranks keep their
  beams in plan order, so each rank's CSR ensemble is a run of whole beams;
- `merge_ensembles` puts the ranks' CSR ensembles back into the plan's beam
  order on the host (the layout `MatCSREnsemble::tofile` writes, one matrix
  per beam), for a caller that wants the whole matrix in one place;
- `gather_ensembles` does that gather over a `torch.distributed` group
  (object collectives: gloo for host ranks, NCCL between GPU ranks).

The optimizer shards the other way, by rows of A (voxels): `row_blocks` cuts
the rows into contiguous blocks; A x is then local and the beamlet-space
gradient is the sum of the blocks' partial A^T g.  The solver makes one
all-reduce per objective evaluation, of the VOI-row objective terms and that
partial gradient in one FP64 buffer, through the reducer the problem is given
(`rank_reducer`, `optimize.Problem.set_reducer`); `allreduce_partials` is the
same exchange for host-side code.
"""
from __future__ import annotations

import numpy as np

from .types import BEAM_DTYPE


def beam_costs(beamlets_per_beam) -> np.ndarray:
    """Cost of each beam: sum over its beamlets of fmap pixels x long_dim."""
    out = np.zeros(len(beamlets_per_beam), np.float64)
    for i, b in enumerate(beamlets_per_beam):
        b = np.asarray(b, BEAM_DTYPE).reshape(-1)
        if b.size:
            px = b["fmap_size"][:, 0].astype(np.float64) * b["fmap_size"][:, 1].astype(np.float64)
            out[i] = float(np.sum(px * b["long_dim"].astype(np.float64)))
    return out


def partition_beams(costs, world: int) -> list[list[int]]:
    """Greedy longest-first assignment of beams to `world` ranks.

    Beams are taken in decreasing cost (ties by index) and each goes to the
    rank with the smallest load so far (ties to the lower rank).  Every beam is
    assigned exactly once; each rank's list is in increasing beam index.  The
    largest load is at most the mean load plus the largest single cost."""
    if world < 1:
        raise ValueError("world must be >= 1")
    costs = np.asarray(costs, np.float64)
    if np.any(costs < 0) or not np.all(np.isfinite(costs)):
        raise ValueError("beam costs must be finite and non-negative")
    order = sorted(range(costs.size), key=lambda i: (-costs[i], i))
    load = np.zeros(world, np.float64)
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = int(np.argmin(load))  # first minimum = lowest rank among ties
        parts[r].append(i)
        load[r] += costs[i]
    return [sorted(p) for p in parts]


def partition_loads(costs, parts) -> np.ndarray:
    costs = np.asarray(costs, np.float64)
    return np.array([float(costs[p].sum()) if len(p) else 0.0 for p in parts])


def merge_ensembles(parts, beams_of_rank, rows_per_beam):
    """Merge per-rank CSR ensembles into the plan's beam order.

    parts[r] = (row_offsets int64 [n_rows_r + 1], columns, values) of rank r's
    ensemble, whose rows are its beams' beamlets in the order of
    beams_of_rank[r]; rows_per_beam[b] = beamlets of beam b.  Returns
    (row_offsets, columns, values) of the whole plan, rows in beam order."""
    rows_per_beam = np.asarray(rows_per_beam, np.int64)
    n_beams = rows_per_beam.size
    seen = np.zeros(n_beams, bool)
    pieces = [None] * n_beams  # beam -> (row lengths, columns, values)
    for (ro, col, val), beams in zip(parts, beams_of_rank):
        ro = np.asarray(ro, np.int64)
        expect = int(rows_per_beam[list(beams)].sum()) if len(beams) else 0
        if ro.size != expect + 1 or ro[0] != 0:
            raise ValueError(f"rank ensemble has {ro.size - 1} rows, its beams have {expect}")
        r0 = 0
        for b in beams:
            if seen[b]:
                raise ValueError(f"beam {b} appears on two ranks")
            seen[b] = True
            r1 = r0 + int(rows_per_beam[b])
            lo, hi = int(ro[r0]), int(ro[r1])
            pieces[b] = (np.diff(ro[r0:r1 + 1]), col[lo:hi], val[lo:hi])
            r0 = r1
    if not seen.all():
        raise ValueError(f"beams {np.flatnonzero(~seen).tolist()} are on no rank")
    if n_beams == 0:
        return np.zeros(1, np.int64), np.zeros(0, np.int32), np.zeros(0, np.float32)
    lens = np.concatenate([p[0] for p in pieces]).astype(np.int64)
    ro = np.zeros(lens.size + 1, np.int64)
    np.cumsum(lens, out=ro[1:])
    col = np.concatenate([np.asarray(p[1]) for p in pieces])
    val = np.concatenate([np.asarray(p[2]) for p in pieces])
    return ro, col, val


def gather_ensembles(local, beams_of_rank, rows_per_beam, group=None, dst=0):
    """Gather every rank's CSR ensemble (row offsets, columns, values; numpy
    arrays or tensors) to rank `dst` and merge there in beam order; other
    ranks get None.  Every rank of the group must call it.

    The arrays move as tensors: one all-gather of their sizes, then
    point-to-point sends to `dst` -- device buffers over NCCL (the arrays are
    copied to this rank's GPU first when they are on the host), host buffers
    over gloo.  Values travel as float32."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" \
        else torch.device("cpu")

    def as_tensor(a, dtype):
        t = a if torch.is_tensor(a) else torch.from_numpy(np.ascontiguousarray(a))
        return t.to(device=dev, dtype=dtype).contiguous()

    ro, col, val = (as_tensor(a, dt) for a, dt in zip(local, (torch.int64, torch.int32, torch.float32)))
    sizes = torch.tensor([ro.numel(), col.numel()], dtype=torch.int64, device=dev)
    every = [torch.empty_like(sizes) for _ in range(world)]
    dist.all_gather(every, sizes, group=group)

    def peer(r):
        return r if group is None else dist.get_global_rank(group, r)

    if rank != dst:
        for t in (ro, col, val):
            dist.send(t, dst=peer(dst), group=group)
        return None
    parts = []
    for r in range(world):
        if r == rank:
            got = (ro, col, val)
        else:
            n_ro, n_nz = (int(v) for v in every[r].tolist())
            got = (torch.empty(n_ro, dtype=torch.int64, device=dev), torch.empty(n_nz, dtype=torch.int32, device=dev),
                   torch.empty(n_nz, dtype=torch.float32, device=dev))
            for t in got:
                dist.recv(t, src=peer(r), group=group)
        parts.append(tuple(t.cpu().numpy() for t in got))
    return merge_ensembles(parts, beams_of_rank, rows_per_beam)


def row_blocks(n_rows: int, world: int) -> list[tuple[int, int]]:
    """Contiguous row ranges [lo, hi) of near-equal size, one per rank."""
    if world < 1 or n_rows < 0:
        raise ValueError("need world >= 1 and n_rows >= 0")
    base, extra = divmod(n_rows, world)
    out, lo = [], 0
    for r in range(world):
        hi = lo + base + (1 if r < extra else 0)
        out.append((lo, hi))
        lo = hi
    return out


def rank_reducer(group=None):
    """The reducer a row-sharded optimizer problem takes
    (optimize.Problem.set_reducer): the sum of a float64 tensor over the
    group's ranks, in place (NCCL between GPU ranks)."""
    import torch.distributed as dist

    def fn(t):
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)

    return fn


def allreduce_partials(grad, terms, group=None):
    """Sum the partial beamlet-space gradient and the objective's scalar terms
    over the ranks in one collective: both are packed into one FP64 buffer
    (gradient, then terms), reduced, and unpacked in place."""
    import torch
    import torch.distributed as dist

    n = grad.numel()
    buf = torch.cat([grad.reshape(-1).to(torch.float64), terms.reshape(-1).to(torch.float64)])
    dist.all_reduce(buf, op=dist.ReduceOp.SUM, group=group)
    grad.copy_(buf[:n].reshape(grad.shape).to(grad.dtype))
    terms.copy_(buf[n:].reshape(terms.shape).to(terms.dtype))
    return grad, terms
