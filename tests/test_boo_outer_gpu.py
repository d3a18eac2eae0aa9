"""Beam selection on device matrices and the beam-orientation loop
(BeamOrientationOptimization + DimReduction, IMRTOptimize.cu:197-388,
IMRTOptUtils.cu:726-793) against the oracle: the oracle's BOO restatement
driven through the same phases by a host loop that selects the active beams
with scipy and ranks them as DimReduction does.

Tolerances: selections bit-exact; costs 1e-3 relative over the common
iterations; the kept beams and their order identical; fluence 1e-2 of its max."""
import numpy as np
import pytest
import scipy.sparse as sp

import oracle
from fastdose_b200 import optimize

pytestmark = pytest.mark.gpu


def _case(seed=21, n_beams=6, fd=8, n_ptv=400, n_oar=1600):
    """Beams with ragged beamlet counts; A = VOI x beamlets (beam-major columns)."""
    rng = np.random.default_rng(seed)
    counts = rng.integers(20, 50, n_beams)
    masks = []
    for c in counts:
        m = np.zeros(fd * fd, np.uint8)
        m[rng.choice(fd * fd, int(c), replace=False)] = 1
        masks.append(m)
    n = int(counts.sum())
    nv = n_ptv + n_oar
    dense = rng.random((nv, n)) * (rng.random((nv, n)) < 0.05)
    # make beams differ in usefulness so that the group prox prunes some
    scale = np.repeat(rng.uniform(0.2, 1.5, n_beams), counts)
    A = sp.csr_matrix((dense * scale).astype(np.float32))
    Ds = [optimize.fluence_grad(fd, m) for m in masks]
    D = optimize.block_diag(Ds)
    beam_cols = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    d_rows = np.concatenate([[0], np.cumsum([len(d[0]) - 1 for d in Ds])]).astype(np.int64)
    w = dict(max_dose=np.concatenate([np.full(n_ptv, 1.05), rng.uniform(0.3, 0.7, n_oar)]).astype(np.float32),
             max_weights=np.concatenate([np.ones(n_ptv), rng.uniform(0.1, 1.0, n_oar)]).astype(np.float32),
             min_dose=np.ones(n_ptv, np.float32), min_weights=np.ones(n_ptv, np.float32),
             oar_weights=rng.uniform(0.0, 0.1, n_oar).astype(np.float32))
    return A, D, beam_cols, d_rows, w, n_ptv, n_oar


def _csr_tuple(M):
    M = sp.csr_matrix(M)
    M.sort_indices()
    return (M.indptr.astype(np.int64), M.indices.astype(np.int64), M.data.astype(np.float32), M.shape[1])


def _oracle_outer(A, D, beam_cols, d_rows, w, n_ptv, n_oar, x0, prm):
    """BeamOrientationOptimization over the oracle's BOO, phase by phase."""
    n_beams = len(beam_cols) - 1
    Dm = sp.csr_matrix((D[2], D[1], D[0]), shape=(d_rows[-1], D[3]))
    active = list(range(n_beams))
    x = x0.copy()
    state = (0, 0.0, prm["step_size"], x0.copy())
    costs = np.zeros(prm["max_iter"], np.float32)
    weights = None
    while True:
        cols = np.concatenate([np.arange(beam_cols[b], beam_cols[b + 1]) for b in active])
        rows = np.concatenate([np.arange(d_rows[b], d_rows[b + 1]) for b in active])
        As = A[:, cols]
        Dsel = Dm[rows][:, cols]
        O = oracle.Problem(_csr_tuple(As), _csr_tuple(Dsel), n_ptv, n_oar, w["max_dose"], w["max_weights"],
                           w["min_dose"], w["min_weights"], w["oar_weights"], prm["gamma"], prm["eta"])
        lens = np.array([beam_cols[b + 1] - beam_cols[b] for b in active], np.int64)
        go = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
        if weights is None:
            blocks = [_csr_tuple(A[:, beam_cols[b]:beam_cols[b + 1]]) for b in active]
            weights = prm["beam_weight"] * oracle.beam_weights_init(blocks, n_ptv)
        r = O.boo(go, weights, x, prm["step_size"], prm["max_iter"], prune=prm["prune"], want=prm["want"],
                  change_trigger=prm["change"], state=state, loss=costs)
        nrm, weights = r["nrm"], r["weights"]
        keep = int(r["active"])
        rank = sorted(range(len(active)), key=lambda j: (-nrm[j], j))[:keep]
        segs_x = [r["x"][go[j]:go[j + 1]] for j in rank]
        segs_v = [r["v"][go[j]:go[j + 1]] for j in rank]
        active = [active[j] for j in rank]
        weights = np.array([weights[j] for j in rank], np.float32)
        norms = np.array([nrm[j] for j in rank], np.float32)
        x = np.concatenate(segs_x) if segs_x else np.zeros(0, np.float32)
        v = np.concatenate(segs_v) if segs_v else np.zeros(0, np.float32)
        state = (r["k"], r["theta"], r["t"], v)
        if r["stop"] or keep == 0:
            return dict(active=np.array(active), norms=norms, x=x, costs=costs, k=r["k"])


@pytest.mark.parametrize("vt,fmt", [("f32", "i32"), ("f16", "packed16")])
def test_select_blocks_reorders_beams_bit_exact(ctx, vt, fmt):
    A, D, beam_cols, d_rows, w, n_ptv, n_oar = _case()
    AT = sp.csr_matrix(A.T)
    ATm = optimize.Matrix.from_csr(ctx, *_csr_tuple(AT)[:3], A.shape[0], value_type=vt, index_format=fmt)
    off, col, val = ATm.to_host()  # the stored values (16-bit rounded, scale applied)
    stored = sp.csr_matrix((val, col, off), shape=AT.shape)
    for order in ([3, 0, 5], [5, 4, 3, 2, 1, 0], [2], []):
        S = ATm.select_blocks(beam_cols, order)
        rows = np.concatenate([np.arange(beam_cols[b], beam_cols[b + 1]) for b in order]) if order else []
        ref = stored[rows] if order else sp.csr_matrix((0, AT.shape[1]), dtype=np.float32)
        so, sc, sv = S.to_host()
        ref.sort_indices()
        np.testing.assert_array_equal(so, ref.indptr)
        np.testing.assert_array_equal(sc, ref.indices)
        np.testing.assert_array_equal(sv, ref.data.astype(np.float32))
        assert S.info()["index_format"] == fmt and S.info()["value_type"] == ATm.info()["value_type"]


def test_select_blocks_renumbers_block_diagonal_columns(ctx):
    A, D, beam_cols, d_rows, w, n_ptv, n_oar = _case()
    Dm = optimize.Matrix.from_csr(ctx, *D[:3], D[3])
    ref_full = sp.csr_matrix((D[2], D[1], D[0]), shape=(d_rows[-1], D[3]))
    order = [4, 1, 2]
    S = Dm.select_blocks(d_rows, order, block_cols=beam_cols)
    rows = np.concatenate([np.arange(d_rows[b], d_rows[b + 1]) for b in order])
    cols = np.concatenate([np.arange(beam_cols[b], beam_cols[b + 1]) for b in order])
    ref = ref_full[rows][:, cols]
    ref.sort_indices()
    so, sc, sv = S.to_host()
    assert S.shape == ref.shape
    np.testing.assert_array_equal(so, ref.indptr)
    np.testing.assert_array_equal(sc, ref.indices)
    np.testing.assert_array_equal(sv, ref.data)
    # a matrix that is not block-diagonal as declared is refused
    from fastdose_b200 import _lib

    wrong = np.array([0] + [int(beam_cols[-1])] * (len(beam_cols) - 1), np.int64)  # block 0 takes every column
    with pytest.raises(_lib.FD2Error) as e:
        Dm.select_blocks(d_rows, order, block_cols=wrong)
    assert e.value.status == -1  # FD2_ERR_INVALID_ARGUMENT
    assert "block-diagonal" in str(e.value)


def test_beam_orientation_matches_oracle(ctx):
    A, D, beam_cols, d_rows, w, n_ptv, n_oar = _case()
    AT = sp.csr_matrix(A.T)
    ATm = optimize.Matrix.from_csr(ctx, *_csr_tuple(AT)[:3], A.shape[0])
    Dm = optimize.Matrix.from_csr(ctx, *D[:3], D[3])
    x0 = optimize.reference_x0(A.shape[1]) * np.float32(0.02)
    prm = dict(beam_weight=0.5, step_size=1e-3, gamma=1.0, eta=0.1, max_iter=150, change=20, want=2, prune=[40, 90])
    got = optimize.beam_orientation_optimization(
        ctx, ATm, Dm, beam_cols, d_rows, n_ptv, n_oar, w["max_dose"], w["max_weights"], w["min_dose"],
        w["min_weights"], w["oar_weights"], x0, beam_weight=prm["beam_weight"], step_size=prm["step_size"],
        gamma=prm["gamma"], eta=prm["eta"], max_iter=prm["max_iter"], change_weights_trigger=prm["change"],
        n_beams_want=prm["want"], prune_trigger=prm["prune"])
    ref = _oracle_outer(A, D, beam_cols, d_rows, w, n_ptv, n_oar, x0, prm)
    assert got["phases"] >= 2  # at least one prune phase ran
    assert len(got["active"]) < len(beam_cols) - 1  # and it dropped beams
    np.testing.assert_array_equal(got["active"], ref["active"])
    k = min(got["iterations"], ref["k"])
    np.testing.assert_allclose(got["costs_full"][:k], ref["costs"][:k], rtol=1e-3)
    np.testing.assert_allclose(got["norms"], ref["norms"], rtol=1e-2)
    x = got["x"].cpu().numpy()
    assert x.shape == ref["x"].shape
    assert np.abs(x - ref["x"]).max() <= 1e-2 * max(np.abs(ref["x"]).max(), 1e-6)


def _dvh_reference(dose, structures, n_bins, width):
    """Binned cumulative DVH in numpy float32 (the same bin rule)."""
    out = np.zeros((len(structures), n_bins), np.uint64)
    for s, vox in enumerate(structures):
        d = dose[np.asarray(vox, np.int64)].astype(np.float32)
        q = np.floor(d / np.float32(width))
        k = np.clip(q, 0, n_bins - 1).astype(np.int64)
        counts = np.bincount(k, minlength=n_bins).astype(np.uint64)
        out[s] = np.cumsum(counts[::-1])[::-1]
    return out


def test_dvh_counts_match_numpy(ctx):
    rng = np.random.default_rng(4)
    n = 300_000
    dose = (rng.gamma(2.0, 0.6, n)).astype(np.float32)
    dose[:100] = -0.5  # clamps to the first bin
    dose[100:200] = 1e6  # clamps to the last
    structures = [rng.choice(n, 50_000, replace=False), np.arange(0, n, 7), np.arange(10), np.zeros(0, np.int64),
                  np.arange(n)]  # overlapping, tiny, empty, everything
    counts, frac = optimize.dvh(ctx, dose, structures, n_bins=400, bin_width=0.01)
    np.testing.assert_array_equal(counts, _dvh_reference(dose, structures, 400, 0.01))
    assert frac[0, 0] == 1.0 and counts[3].sum() == 0
    from fastdose_b200 import _lib

    with pytest.raises(_lib.FD2Error):
        optimize.dvh(ctx, dose, [np.array([0, n])], n_bins=10, bin_width=1.0)  # voxel n is outside the dose


def test_final_dose_and_dvh_of_the_kept_beams(ctx):
    """resultDoseCalc: the kept beams' fluence through the all-beam matrix equals
    the product over the kept beams' columns alone; its DVHs per structure."""
    import torch

    A, D, beam_cols, d_rows, w, n_ptv, n_oar = _case()
    Am = optimize.Matrix.from_csr(ctx, *_csr_tuple(A)[:3], A.shape[1])
    active = [4, 0, 2]
    rng = np.random.default_rng(9)
    n_keep = int(sum(beam_cols[b + 1] - beam_cols[b] for b in active))
    x = rng.random(n_keep).astype(np.float32)
    dose = optimize.final_dose(Am, beam_cols, active, torch.from_numpy(x).cuda()).cpu().numpy()
    cols = np.concatenate([np.arange(beam_cols[b], beam_cols[b + 1]) for b in active])
    ref = A[:, cols].astype(np.float64) @ x.astype(np.float64)
    bound = abs(A[:, cols]).astype(np.float64) @ np.abs(x.astype(np.float64))
    assert np.all(np.abs(dose - ref) <= 2e-5 * bound + 1e-30)
    structures = [np.arange(n_ptv), np.arange(n_ptv, n_ptv + n_oar)]
    counts, frac = optimize.dvh(ctx, dose, structures, n_bins=200, bin_width=float(dose.max()) / 199)
    np.testing.assert_array_equal(counts, _dvh_reference(dose, structures, 200, float(dose.max()) / 199))
