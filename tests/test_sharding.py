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
        # the solver's reducer: an FP64 buffer summed over the ranks in place
        buf = torch.full((5,), float(rank + 1), dtype=torch.float64)
        sharding.rank_reducer()(buf)
        ok_terms_r = bool(torch.all(buf == 3.0))
        rf = A @ x - d
        ok_grad = np.allclose(g.numpy(), (A.T @ (w * rf)).astype(np.float32), rtol=1e-6, atol=1e-5)
        ok_terms = (abs(terms[0].item() - 0.5 * float(np.sum(w * rf * rf))) < 1e-9 and terms[1].item() == n_rows
                    and ok_terms_r)
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


@pytest.mark.gpu
def test_row_sharded_optimizer_matches_the_whole_problem(ctx):
    """The optimizer with A's VOI rows split between two ranks -- here two host
    threads, each with its own context on the one GPU, exchanging partial sums
    through host memory (no kernel waits on another) -- takes the same steps as
    the whole problem: the same iterations and trials, costs within 1e-5 and the
    same fluence within 1e-4 of its max (the partial sums are added in a
    different order)."""
    import threading

    from fastdose_b200 import api, optimize

    rng = np.random.default_rng(21)
    n_beams, fd, per_beam, n_ptv, n_oar = 6, 8, 40, 500, 1500
    n, nv = n_beams * per_beam, n_ptv + n_oar
    dense = rng.random((nv, n)) * (rng.random((nv, n)) < 0.05)
    import scipy.sparse as sp

    A = sp.csr_matrix(dense.astype(np.float32))
    masks = []
    for _ in range(n_beams):
        m = np.zeros(fd * fd, np.uint8)
        m[rng.choice(fd * fd, per_beam, replace=False)] = 1
        masks.append(m)
    D = optimize.block_diag([optimize.fluence_grad(fd, m) for m in masks])
    w = dict(max_dose=np.concatenate([np.full(n_ptv, 1.05), rng.uniform(0.3, 0.7, n_oar)]).astype(np.float32),
             max_weights=np.concatenate([np.ones(n_ptv), rng.uniform(0.1, 1.0, n_oar)]).astype(np.float32),
             min_dose=np.ones(n_ptv, np.float32), min_weights=np.ones(n_ptv, np.float32),
             oar_weights=rng.uniform(0.0, 0.1, n_oar).astype(np.float32))
    groups = np.arange(0, n + 1, per_beam, dtype=np.int64)
    x0 = np.full(n, 0.01, np.float32)

    def problem(c, lo, hi):
        Ab = A[lo:hi]
        Am = optimize.Matrix.from_csr(c, Ab.indptr.astype(np.int64), Ab.indices.astype(np.int64), Ab.data, n)
        Dm = optimize.Matrix.from_csr(c, *D[:3], n)
        p_lo, p_hi = min(lo, n_ptv), min(hi, n_ptv)
        P = optimize.Problem(c, Am, Am.transpose(), Dm, Dm.transpose(), p_hi - p_lo, (hi - lo) - (p_hi - p_lo),
                             w["max_dose"][lo:hi], w["max_weights"][lo:hi], w["min_dose"][p_lo:p_hi],
                             w["min_weights"][p_lo:p_hi],
                             w["oar_weights"][max(lo, n_ptv) - n_ptv:max(hi, n_ptv) - n_ptv], 1.0, 0.1)
        return P, (Am, Dm)

    def solve(P):
        bw = 0.1 * P.beam_weights_init(groups)
        r = P.boo(groups, bw, x0, step_size=1e-3, iters=40, want=2, change_trigger=10)
        return dict(bw=bw, k=r["k"], trials=r["trials"], loss=r["loss"][:r["k"]], x=r["x"].cpu().numpy())

    whole, _keep = problem(ctx, 0, nv)
    ref = solve(whole)

    blocks = sharding.row_blocks(nv, 2)
    bar = threading.Barrier(2)
    slots = [None, None]
    out, errs = [None, None], []

    def reducer(rank):
        def fn(t):
            slots[rank] = t.cpu().numpy()
            bar.wait(timeout=60)
            total = slots[0] + slots[1]  # the same order on both ranks
            bar.wait(timeout=60)
            t.copy_(torch.from_numpy(total).to(t.device))
        return fn

    def rank_main(rank):
        try:
            c = api.Context(0)
            P, keep = problem(c, *blocks[rank])
            P.set_reducer(reducer(rank))
            out[rank] = solve(P)
            P.close()
            del keep
        except Exception as e:  # surfaced below
            errs.append(e)
            bar.abort()

    th = [threading.Thread(target=rank_main, args=(r,)) for r in range(2)]
    for t in th:
        t.start()
    for t in th:
        t.join(300)
    assert not errs, errs
    for r in range(2):
        got = out[r]
        np.testing.assert_allclose(got["bw"], ref["bw"], rtol=1e-6)
        assert got["k"] == ref["k"] and got["trials"] == ref["trials"]
        np.testing.assert_allclose(got["loss"], ref["loss"], rtol=1e-5)
        assert np.abs(got["x"] - ref["x"]).max() <= 1e-4 * np.abs(ref["x"]).max()
    np.testing.assert_array_equal(out[0]["x"], out[1]["x"])  # every rank takes the same steps
