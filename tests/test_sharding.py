"""Multi-rank dose calculation: beam partition, the merge of per-rank CSR
ensembles in beam order, and the optimizer's row-sharded gradient sum, on
world-size-2 gloo ranks (CPU; the per-rank columns come from the oracle)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from fastdose_b200 import sharding
from oracle import oracle
from plan_cases import small_case

GANTRY = (0.6, 1.4, 2.5, 4.0)
KEEP = (16, 9, 5, 12)  # beamlets kept per beam, so the beams' costs differ


def _plan():
    """Four beams on one 32^3 phantom, ragged beamlet counts."""
    cases = [small_case(seed=5, gantry=g) for g in GANTRY]
    beams = [c["beams"][:k] for c, k in zip(cases, KEEP)]
    c0 = cases[0]
    return c0, beams


def _oracle_csr(c0, beams):
    """Oracle CSR ensemble (rows = beamlets in the given beam order)."""
    ph = c0["phantom"]
    if not beams:
        return np.zeros(1, np.int64), np.zeros(0, np.int64), np.zeros(0, np.float32)
    rows = oracle.dose_rows(np.concatenate(beams), c0["fluence"], ph.density, ph.volume, c0["spectrum"],
                            c0["kernel"], precision="float")
    return oracle.dense_to_csr(rows)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


# ---------------------------------------------------------------- partition
def test_partition_assigns_every_beam_once_and_balances():
    rng = np.random.default_rng(3)
    for world in (1, 2, 3, 8):
        for n in (0, 1, 5, 40, 401):
            costs = rng.integers(0, 1000, n).astype(np.float64) * rng.uniform(0.5, 2.0, n)
            parts = sharding.partition_beams(costs, world)
            assert len(parts) == world
            flat = sorted(i for p in parts for i in p)
            assert flat == list(range(n))
            assert all(p == sorted(p) for p in parts)
            loads = sharding.partition_loads(costs, parts)
            if n:
                assert loads.max() <= costs.sum() / world + costs.max() + 1e-9
            assert parts == sharding.partition_beams(costs, world)  # deterministic


def test_partition_largest_first_rule():
    # costs by index (3, 7, 1, 5, 4), taken as 7, 5, 4, 3, 1: 7 -> r0, 5 -> r1,
    # 4 -> r1 (5 < 7), 3 -> r0 (7 < 9), 1 -> r1 (9 < 10)
    parts = sharding.partition_beams([3, 7, 1, 5, 4], 2)
    assert parts == [[0, 1], [2, 3, 4]]
    assert sharding.partition_loads([3, 7, 1, 5, 4], parts).tolist() == [10.0, 10.0]
    with pytest.raises(ValueError):
        sharding.partition_beams([1.0, -1.0], 2)
    with pytest.raises(ValueError):
        sharding.partition_beams([1.0], 0)


def test_beam_costs_follow_march_length():
    _, beams = _plan()
    costs = sharding.beam_costs(beams)
    for b, c in zip(beams, costs):
        px = b["fmap_size"][:, 0].astype(float) * b["fmap_size"][:, 1]
        assert c == pytest.approx(float(np.sum(px * b["long_dim"])))
    assert sharding.beam_costs([np.zeros(0, beams[0].dtype)]).tolist() == [0.0]


def test_row_blocks_cover_rows():
    for n, w in ((0, 3), (10, 3), (7, 7), (5, 8)):
        blocks = sharding.row_blocks(n, w)
        assert blocks[0][0] == 0 and blocks[-1][1] == n
        assert all(a[1] == b[0] for a, b in zip(blocks, blocks[1:]))
        sizes = [hi - lo for lo, hi in blocks]
        assert max(sizes) - min(sizes) <= 1


def test_merge_rejects_inconsistent_parts():
    ro = np.array([0, 1, 2], np.int64)
    part = (ro, np.array([0, 1]), np.array([1.0, 2.0], np.float32))
    with pytest.raises(ValueError):
        sharding.merge_ensembles([part], [[0]], [1])  # 2 rows for a 1-row beam
    with pytest.raises(ValueError):
        sharding.merge_ensembles([part, part], [[0], [0]], [2])  # beam on two ranks
    with pytest.raises(ValueError):
        sharding.merge_ensembles([part], [[0]], [2, 1])  # beam 1 on no rank


# ----------------------------------------------------------- gloo ranks (2)
def _rank_main(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        c0, beams = _plan()
        parts = sharding.partition_beams(sharding.beam_costs(beams), world)
        mine = parts[rank]
        local = _oracle_csr(c0, [beams[b] for b in mine])
        merged = sharding.gather_ensembles(local, parts, [len(b) for b in beams])

        # optimizer: rows of A split across ranks; the partial A^T (w * (A x - d))
        # and the objective term are summed in one all-reduce
        rng = np.random.default_rng(11)
        n_rows, n_cols = 500, 40
        A = rng.random((n_rows, n_cols)) * (rng.random((n_rows, n_cols)) < 0.2)
        x = rng.random(n_cols)
        d = rng.random(n_rows)
        w = rng.uniform(0.5, 2.0, n_rows)
        lo, hi = sharding.row_blocks(n_rows, world)[rank]
        r = A[lo:hi] @ x - d[lo:hi]
        g = torch.from_numpy(A[lo:hi].T @ (w[lo:hi] * r)).to(torch.float32)
        terms = torch.tensor([0.5 * float(np.sum(w[lo:hi] * r * r)), float(hi - lo)], dtype=torch.float64)
        sharding.allreduce_partials(g, terms)
        rf = A @ x - d
        ok_grad = np.allclose(g.numpy(), (A.T @ (w * rf)).astype(np.float32), rtol=1e-6, atol=1e-5)
        ok_terms = abs(terms[0].item() - 0.5 * float(np.sum(w * rf * rf))) < 1e-9 and terms[1].item() == n_rows
        if rank == 0:
            q.put(("merged", merged, parts))
        q.put(("opt", rank, ok_grad, ok_terms))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_beams_and_rows():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    msgs = [q.get(timeout=300) for _ in range(3)]
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    merged = next(m for m in msgs if m[0] == "merged")
    _, (ro, col, val), parts = merged
    assert all(len(p) for p in parts)  # both ranks got beams
    c0, beams = _plan()
    ro_f, col_f, val_f = _oracle_csr(c0, beams)
    np.testing.assert_array_equal(ro, ro_f)
    np.testing.assert_array_equal(col, col_f)
    np.testing.assert_array_equal(val, val_f)
    opt = [m for m in msgs if m[0] == "opt"]
    assert len(opt) == 2 and all(m[2] and m[3] for m in opt)


# ------------------------------------------------------ GPU shards (one GPU)
@pytest.mark.gpu
def test_sharded_construction_merges_to_the_whole_plan(ctx):
    """Each rank's share built on its own (here one after another on one GPU,
    nothing waits on another launch) and merged in beam order equals the
    whole plan built at once, bit for bit."""
    from fastdose_b200 import api

    c0, beams = _plan()
    ph = c0["phantom"]
    dens = api.Density(ctx, ph.density, ph.volume)
    spec, kern = api.Spectrum(ctx, c0["spectrum"]), api.Kernel(ctx, c0["kernel"])

    def build(bs):
        m = api.DoseMatConstruction(ctx, bs, c0["fluence"], dens, spec, kern)
        out = m.to_host()
        m.close()
        return out

    whole = build(beams)
    for world in (2, 3):
        parts = sharding.partition_beams(sharding.beam_costs(beams), world)
        locals_ = [build([beams[b] for b in p]) if p else
                   (np.zeros(1, np.int64), np.zeros(0, np.int32), np.zeros(0, np.float32)) for p in parts]
        merged = sharding.merge_ensembles(locals_, parts, [len(b) for b in beams])
        for a, b in zip(merged, whole):
            np.testing.assert_array_equal(a, b)
