"""A seeded optimization problem shared by the optimizer parity tests and
tests/golden/make_golden_opt.py (deterministic from its seed, so the fixture
made by the reference and the tests rebuild the same inputs).

The shape follows the reference's optimizer inputs (IMRTOptimize.cu:197-388):
A is VOI rows (PTV first, then OAR) x beamlets, its columns grouped by beam
with ragged beamlet counts; each beam has a fluence map whose on-pixels are
its beamlets in row-major order (the x2d operator); D is the block diagonal
of the per-beam fluence-gradient operators (fluenceGradInit, diagBlock)."""
import numpy as np
import scipy.sparse as sp

import oracle


def opt_case(seed=31, n_beams=24, fd=12, n_ptv=6000, n_oar=42000, count_range=(40, 121)):
    rng = np.random.default_rng(seed)
    counts = rng.integers(count_range[0], count_range[1], n_beams)
    masks = np.zeros((n_beams, fd * fd), np.uint8)
    for b, c in enumerate(counts):
        masks[b, rng.choice(fd * fd, int(c), replace=False)] = 1
    n = int(counts.sum())
    nv = n_ptv + n_oar
    # beams differ in usefulness, so the group prox has something to prune
    beam_scale = np.repeat(rng.uniform(0.3, 1.5, n_beams), counts).astype(np.float32)
    rows_l, cols_l, vals_l = [], [], []
    win = int(0.15 * n_oar)
    for j in range(n):
        r_ptv = np.flatnonzero(rng.random(n_ptv) < 0.05)
        start = int(rng.integers(0, n_oar - win))
        r_oar = n_ptv + start + np.flatnonzero(rng.random(win) < 0.15)
        r = np.concatenate([r_ptv, r_oar])
        v = np.concatenate([rng.uniform(0.005, 0.03, r_ptv.size), rng.uniform(0.001, 0.02, r_oar.size)])
        rows_l.append(r)
        cols_l.append(np.full(r.size, j))
        vals_l.append((v * beam_scale[j]).astype(np.float32))
    M = sp.csr_matrix((np.concatenate(vals_l), (np.concatenate(rows_l), np.concatenate(cols_l))), shape=(nv, n),
                      dtype=np.float32)
    M.sort_indices()
    A = (M.indptr.astype(np.int64), M.indices.astype(np.int64), M.data.astype(np.float32), n)
    Ds = [oracle.fluence_grad(fd, masks[b]) for b in range(n_beams)]
    D = _block_diag(Ds)
    d_rows = np.concatenate([[0], np.cumsum([len(d[0]) - 1 for d in Ds])]).astype(np.int64)
    w = dict(max_dose=np.concatenate([np.full(n_ptv, 1.05), rng.uniform(0.3, 0.7, n_oar)]).astype(np.float32),
             max_weights=np.concatenate([np.ones(n_ptv), rng.uniform(0.1, 1.0, n_oar)]).astype(np.float32),
             min_dose=np.ones(n_ptv, np.float32), min_weights=np.ones(n_ptv, np.float32),
             oar_weights=rng.uniform(0.0, 0.1, n_oar).astype(np.float32))
    beam_cols = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    return dict(A=A, D=D, Ds=Ds, masks=masks, counts=counts.astype(np.int64), beam_cols=beam_cols, d_rows=d_rows,
                w=w, n_ptv=n_ptv, n_oar=n_oar, n=n, fd=fd, gamma=1.0, eta=0.1, csr=M)


def _block_diag(blocks):
    offs, cols, vals = [np.zeros(1, np.int64)], [], []
    base_nnz = base_col = 0
    for off, col, val, nc in blocks:
        offs.append(np.asarray(off[1:], np.int64) + base_nnz)
        cols.append(np.asarray(col, np.int64) + base_col)
        vals.append(np.asarray(val, np.float32))
        base_nnz += len(col)
        base_col += nc
    return np.concatenate(offs), np.concatenate(cols), np.concatenate(vals), base_col


def select(case, beams):
    """A, D and fluence maps of the listed beams, in that order (the
    reference's parallelMatCoalesce and diagBlock over activeBeams)."""
    M = case["csr"]
    bc = case["beam_cols"]
    cols = np.concatenate([np.arange(bc[b], bc[b + 1]) for b in beams])
    As = M[:, cols].tocsr()
    As.sort_indices()
    A = (As.indptr.astype(np.int64), As.indices.astype(np.int64), As.data.astype(np.float32), len(cols))
    D = _block_diag([case["Ds"][b] for b in beams])
    return A, D, case["masks"][list(beams)]


def beam_blocks(case, beams=None):
    """Per-beam VOI x beamlet blocks (the VOIMatrices of beamWeightsInit_func)."""
    M = case["csr"]
    bc = case["beam_cols"]
    out = []
    for b in (range(len(bc) - 1) if beams is None else beams):
        B = M[:, bc[b]:bc[b + 1]].tocsr()
        B.sort_indices()
        out.append((B.indptr.astype(np.int64), B.indices.astype(np.int64), B.data.astype(np.float32),
                    int(bc[b + 1] - bc[b])))
    return out


# the runs recorded in tests/golden/opt_ref.npz
BOO = dict(beam_weight=0.1, step_size=1e-3, iters=100, change_trigger=20, want=0)
OUTER = dict(beam_weight=0.1, step_size=1e-3, max_iter=100, change_trigger=20, want=8, prune=(30, 60))
POLISH = dict(step_size=1e-3, iters=100)


def eval_points(case):
    """The fluence vectors the objective and gradient are pinned at."""
    rng = np.random.default_rng(101)
    n = case["n"]
    return [np.zeros(n, np.float32), (0.02 * rng.random(n)).astype(np.float32), rng.random(n).astype(np.float32)]


def prox_input(case):
    """A prox input over the beam x pixel operator with a zero-norm group and a
    group whose squared norm (5e-5) falls under the 1e-4 guard."""
    rng = np.random.default_rng(102)
    n, counts = case["n"], case["counts"]
    g0 = (0.3 * rng.standard_normal(n)).astype(np.float32)
    bc = case["beam_cols"]
    g0[bc[3]:bc[4]] = 0.0
    seg = rng.standard_normal(counts[5])
    g0[bc[5]:bc[6]] = (seg / np.linalg.norm(seg) * np.sqrt(5e-5)).astype(np.float32)
    tau = rng.uniform(0.01, 1.0, len(counts)).astype(np.float32)
    return g0, tau


def dim_reduction(active, counts, weights, x, v, nrm, n_keep):
    """DimReduction (IMRTOptUtils.cu:726-793): keep the n_keep beams of largest
    norm, strongest first, with their weights and fluence segments."""
    offs = np.concatenate([[0], np.cumsum([counts[b] for b in active])]).astype(np.int64)
    rank = sorted(range(len(active)), key=lambda j: -float(nrm[j]))[:n_keep]
    keep = [active[j] for j in rank]
    seg = lambda a: (np.concatenate([a[offs[j]:offs[j + 1]] for j in rank]).astype(np.float32)  # noqa: E731
                     if rank else np.zeros(0, np.float32))
    return keep, np.array([weights[j] for j in rank], np.float32), seg(x), seg(v)


def oracle_outer(case, x0, beam_weights, prm=OUTER):
    """BeamOrientationOptimization (IMRTOptimize.cu:197-388) over the oracle's
    BOO: phases ended by the prune triggers, each followed by DimReduction."""
    w = case["w"]
    active = list(range(len(case["counts"])))
    x = v = x0
    weights = beam_weights
    state = None
    costs = np.zeros(prm["max_iter"], np.float32)
    phases = []
    while True:
        A, D, _ = select(case, active)
        O = oracle.Problem(A, D, case["n_ptv"], case["n_oar"], w["max_dose"], w["max_weights"], w["min_dose"],
                           w["min_weights"], w["oar_weights"], case["gamma"], case["eta"])
        go = np.concatenate([[0], np.cumsum([case["counts"][b] for b in active])]).astype(np.int64)
        st = None if state is None else (state[0], state[1], state[2], v)
        r = O.boo(go, weights, x, prm["step_size"], prm["max_iter"], prune=prm["prune"], want=prm["want"],
                  change_trigger=prm["change_trigger"], state=st, loss=costs)
        state = (r["k"], r["theta"], r["t"])
        phases.append((list(active), r["k"], r["active"]))
        active, weights, x, v = dim_reduction(active, case["counts"], r["weights"], r["x"], r["v"], r["nrm"],
                                              int(r["active"]))
        if r["stop"] or not active:
            break
    return dict(active=np.array(active, np.int32), x=x, v=v, weights=weights, costs=costs, state=state,
                phases=phases)
