"""Optimizer on the GPU against the oracle (double-precision restatement of
IMRTOptUtils.cu / IMRTOptimize_var1.cu / IMRTOptimize.cu) and against exact
numpy arithmetic for the matrix operations.

Tolerances: SpMV in FP32 accumulation vs an FP64 product, 2e-5 relative to the
row's |A||x| sum; objective 1e-5 relative; gradient 1e-4 of its max; solver
loss trajectories 1e-3 relative (the line search compares FP64 sums, the
oracle's are FP64 too, so only FP32 rounding of the products differs)."""
import numpy as np
import pytest

import oracle
from fastdose_b200 import api, optimize
from plan_cases import small_case

pytestmark = pytest.mark.gpu


def _random_csr(rng, rows, cols, density, long_rows=(), empty_frac=0.1):
    offs = [0]
    cols_l, vals_l = [], []
    for r in range(rows):
        if r in long_rows:
            k = cols
        elif rng.random() < empty_frac:
            k = 0
        else:
            k = rng.binomial(cols, density)
        c = np.sort(rng.choice(cols, size=k, replace=False))
        cols_l.append(c)
        vals_l.append(rng.random(k).astype(np.float32) + 0.01)
        offs.append(offs[-1] + k)
    return (np.array(offs, np.int64), np.concatenate(cols_l).astype(np.int64), np.concatenate(vals_l), cols)


def _dense(m, rows):
    off, col, val, nc = m[0], m[1], m[2], m[3]
    d = np.zeros((rows, nc))
    for r in range(rows):
        d[r, col[off[r]:off[r + 1]]] = val[off[r]:off[r + 1]]
    return d


@pytest.mark.parametrize("cols,density", [(6000, 0.01), (60000, 0.001)])
@pytest.mark.parametrize("fmt", ["i32", "packed16"])
@pytest.mark.parametrize("vt", ["f32", "f16", "bf16"])
def test_spmv_matches_exact_product(ctx, vt, fmt, cols, density):
    """Both SpMV instances: x of 6000 floats is gathered from shared memory,
    x of 60000 floats (over 200 KiB) from global memory."""
    import scipy.sparse as sp
    import torch

    rng = np.random.default_rng(3)
    rows = 700  # rows 3 and 400 span many 256-nonzero chunks and several warps
    m = _random_csr(rng, rows, cols, density, long_rows=(3, 400))
    M = optimize.Matrix.from_csr(ctx, *m[:3], cols, value_type=vt, index_format=fmt)
    info = M.info()
    assert info["index_format"] == fmt
    assert info["x_in_shared"] == (cols * 4 <= 200 * 1024)
    off, col, val = M.to_host()  # the stored (rounded) values, scale applied
    np.testing.assert_array_equal(off, m[0])
    np.testing.assert_array_equal(col, m[1])
    rel = {"f32": 0.0, "f16": 2.0 ** -11, "bf16": 2.0 ** -8}[vt]
    assert np.all(np.abs(val - m[2]) <= rel * np.abs(m[2]) + 1e-12)
    x = rng.standard_normal(cols).astype(np.float32)
    y = M.spmv(torch.from_numpy(x).cuda()).cpu().numpy()
    D = sp.csr_matrix((val.astype(np.float64), col, off), shape=(rows, cols))
    ref = D @ x.astype(np.float64)
    bound = abs(D) @ np.abs(x.astype(np.float64))
    assert np.all(np.abs(y - ref) <= 2e-5 * bound + 1e-30)
    # empty rows are written as zero and repeated products are bit-identical
    empty = np.diff(off) == 0
    assert empty.any() and np.all(y[empty] == 0)
    y2 = M.spmv(torch.from_numpy(x).cuda()).cpu().numpy()
    np.testing.assert_array_equal(y, y2)


@pytest.mark.parametrize("vt,fmt", [("f32", "i32"), ("f16", "packed16")])
def test_spmv_at_scale_matches_cusparse_and_its_adjoint(ctx, vt, fmt):
    """400k VOI rows x 4000 beamlets, 3.2e7 nonzeros: A x against cuSPARSE
    (through torch) on the same stored values, and <A x, y> = <x, A^T y> with
    A^T generated independently."""
    import torch

    rows, cols = 400_000, 4000
    A, AT = optimize.Matrix.synthetic(ctx, rows, cols, rows // 25, 0.5, seed=5, value_type=vt, index_format=fmt)
    g = torch.Generator(device="cuda").manual_seed(1)
    x = torch.rand(cols, device="cuda", generator=g)
    y = torch.rand(rows, device="cuda", generator=g)
    Ax, ATy = A.spmv(x), AT.spmv(y)
    torch.cuda.synchronize()
    lhs = torch.dot(Ax.double(), y.double()).item()
    rhs = torch.dot(x.double(), ATy.double()).item()
    assert abs(lhs - rhs) <= 1e-6 * abs(lhs)
    off, col, val = A.to_host()
    S = torch.sparse_csr_tensor(torch.from_numpy(off).cuda(), torch.from_numpy(col.astype(np.int64)).cuda(),
                                torch.from_numpy(val).cuda(), size=(rows, cols))
    ref = (S @ x.unsqueeze(1)).squeeze(1)
    bound = (torch.sparse_csr_tensor(S.crow_indices(), S.col_indices(), S.values().abs(), size=(rows, cols))
             @ x.abs().unsqueeze(1)).squeeze(1)
    assert torch.all((Ax - ref).abs() <= 2e-5 * bound + 1e-30)


def test_packed_columns_with_wide_chunks(ctx):
    """Columns spread over 300k: most chunks span more than 65536 columns and
    keep int32 columns; short rows (many row starts per chunk) and empty rows."""
    import torch

    rng = np.random.default_rng(8)
    rows, cols = 4000, 300_000
    m = _random_csr(rng, rows, cols, 2e-4, long_rows=(17,), empty_frac=0.3)
    ref = optimize.Matrix.from_csr(ctx, *m[:3], cols, value_type="f32", index_format="i32")
    M = optimize.Matrix.from_csr(ctx, *m[:3], cols, value_type="f32", index_format="packed16")
    info = M.info()
    assert 0 < info["exception_chunks"] < (m[0][-1] + 255) // 256
    for a, b in zip(M.to_host(), ref.to_host()):
        np.testing.assert_array_equal(a, b)
    x = torch.from_numpy(rng.standard_normal(cols).astype(np.float32)).cuda()
    np.testing.assert_array_equal(M.spmv(x).cpu().numpy(), ref.spmv(x).cpu().numpy())
    # its transpose (300k rows, columns < 4000) packs without exceptions
    T = M.transpose()
    assert T.info()["index_format"] == "packed16" and T.info()["exception_chunks"] == 0
    for a, b in zip(T.to_host(), ref.transpose().to_host()):
        np.testing.assert_array_equal(a, b)


def test_transpose_is_exact(ctx):
    rng = np.random.default_rng(4)
    m = _random_csr(rng, 300, 2500, 0.02, long_rows=(7,))
    for vt in ("f32", "f16"):
        M = optimize.Matrix.from_csr(ctx, *m[:3], 2500, value_type=vt)
        T = M.transpose()
        assert T.shape == (2500, 300)
        assert T.info()["scale_axis"] == ("rows" if vt == "f16" else "none")
        off, col, val = M.to_host()
        t_off, t_col, t_val = T.to_host()
        r_off, r_col, r_val, _ = oracle.csr_transpose((off, col.astype(np.int64), val, 2500))
        np.testing.assert_array_equal(t_off, r_off)
        np.testing.assert_array_equal(t_col, r_col)
        np.testing.assert_array_equal(t_val, r_val)


@pytest.mark.parametrize("fmt", ["i32", "packed16"])
def test_synthetic_pair_is_an_exact_transpose(ctx, fmt):
    for vt in ("f32", "f16"):
        A, AT = optimize.Matrix.synthetic(ctx, 6000, 300, 900, 0.3, seed=7, value_type=vt, index_format=fmt)
        ia, it = A.info(), AT.info()
        assert ia["nnz"] == it["nnz"] > 0 and (ia["rows"], ia["cols"]) == (it["cols"], it["rows"])
        T = A.transpose()
        for a, b in zip(T.to_host(), AT.to_host()):
            np.testing.assert_array_equal(a, b)


def _problem_case(seed=11, n_beams=6, fd=8, per_beam=40, n_ptv=500, n_oar=1500):
    rng = np.random.default_rng(seed)
    n = n_beams * per_beam
    nv = n_ptv + n_oar
    A = _random_csr(rng, nv, n, 0.05, empty_frac=0.05)
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
    return A, D, w, groups, n_ptv, n_oar, n


def _gpu_problem(ctx, A, D, w, n_ptv, n_oar, n, vt="f32", gamma=1.0, eta=0.1, fmt="i32"):
    Am = optimize.Matrix.from_csr(ctx, *A[:3], n, value_type=vt, index_format=fmt)
    ATm = Am.transpose()
    Dm = optimize.Matrix.from_csr(ctx, *D[:3], n)
    DTm = Dm.transpose()
    return optimize.Problem(ctx, Am, ATm, Dm, DTm, n_ptv, n_oar, w["max_dose"], w["max_weights"], w["min_dose"],
                            w["min_weights"], w["oar_weights"], gamma, eta)


def _oracle_problem(A, D, w, n_ptv, n_oar, gamma=1.0, eta=0.1):
    return oracle.Problem(A, D, n_ptv, n_oar, w["max_dose"], w["max_weights"], w["min_dose"], w["min_weights"],
                          w["oar_weights"], gamma, eta)


def test_objective_and_gradient_match_oracle(ctx):
    A, D, w, groups, n_ptv, n_oar, n = _problem_case()
    P = _gpu_problem(ctx, A, D, w, n_ptv, n_oar, n)
    O = _oracle_problem(A, D, w, n_ptv, n_oar)
    rng = np.random.default_rng(0)
    for scale in (0.0, 0.02, 0.1):
        x = (scale * rng.random(n)).astype(np.float32)
        g_ref = O.eval_g(x)
        assert abs(P.eval_g(x) - g_ref) <= 1e-5 * abs(g_ref)
        v, g = P.eval_grad(x)
        v_ref, g_ref_vec = O.eval_grad(x)
        assert abs(v - v_ref) <= 1e-5 * abs(v_ref)
        g = g.cpu().numpy()
        assert np.abs(g - g_ref_vec).max() <= 1e-4 * np.abs(g_ref_vec).max()


def test_prox_matches_oracle(ctx):
    rng = np.random.default_rng(5)
    groups = np.array([0, 10, 10, 60, 61, 200], np.int64)  # includes an empty group
    g0 = rng.standard_normal(200).astype(np.float32) * 0.3
    g0[60] = 0.0  # zero-norm guard
    tau = np.array([0.1, 0.5, 0.05, 0.2, 2.0], np.float32)
    prox, nrm = optimize.prox_l2onehalf(ctx, groups, g0, tau)
    p_ref, n_ref = oracle.prox_l2onehalf(groups, g0, tau)
    np.testing.assert_allclose(prox.cpu().numpy(), p_ref, rtol=1e-5, atol=1e-7)
    np.testing.assert_allclose(nrm.cpu().numpy(), n_ref, rtol=1e-5, atol=1e-7)


def test_beam_weights_match_oracle(ctx):
    A, D, w, groups, n_ptv, n_oar, n = _problem_case()
    P = _gpu_problem(ctx, A, D, w, n_ptv, n_oar, n)
    blocks = []
    dense = _dense(A, n_ptv + n_oar)
    for b in range(len(groups) - 1):
        blk = dense[:, groups[b]:groups[b + 1]]
        blocks.append(oracle.dense_to_csr(blk) + (blk.shape[1],))
    ref = oracle.beam_weights_init(blocks, n_ptv)
    np.testing.assert_allclose(P.beam_weights_init(groups), ref, rtol=1e-6)


def test_boo_matches_oracle(ctx):
    A, D, w, groups, n_ptv, n_oar, n = _problem_case()
    P = _gpu_problem(ctx, A, D, w, n_ptv, n_oar, n)
    O = _oracle_problem(A, D, w, n_ptv, n_oar)
    bw = 0.1 * P.beam_weights_init(groups)
    x0 = np.full(n, 0.01, np.float32)
    iters = 60
    got = P.boo(groups, bw, x0, step_size=1e-3, iters=iters, want=2, change_trigger=20)
    ref = O.boo(groups, bw, x0, step_size=1e-3, iters=iters, want=2, change_trigger=20)
    k = min(got["k"], ref["k"])
    assert k >= 20
    np.testing.assert_allclose(got["loss"][:k], ref["loss_full"][:k], rtol=1e-3)
    np.testing.assert_allclose(got["weights"], ref["weights"], rtol=1e-6)
    x = got["x"].cpu().numpy()
    assert np.abs(x - ref["x"]).max() <= 1e-2 * max(np.abs(ref["x"]).max(), 1e-6)


def test_trials_from_a_captured_graph_match_direct_launches(ctx):
    """BOO and polish give the same bits whether each line-search trial is
    replayed from the captured CUDA graph or launched kernel by kernel."""
    A, D, w, groups, n_ptv, n_oar, n = _problem_case(seed=14)
    x0 = np.full(n, 0.01, np.float32)
    out = []
    for graph in (True, False):
        P = _gpu_problem(ctx, A, D, w, n_ptv, n_oar, n)
        P.set_graph(graph)
        bw = 0.1 * P.beam_weights_init(groups)
        r = P.boo(groups, bw, x0, step_size=1e-3, iters=40, want=2, change_trigger=10)
        q = P.polish(x0, step_size=1e-3, iters=30)
        out.append((r["loss"], r["x"].cpu().numpy(), r["nrm"], r["trials"], q["loss"], q["x"].cpu().numpy()))
    for a, b in zip(*out):
        np.testing.assert_array_equal(a, b)


def test_polish_matches_oracle(ctx):
    A, D, w, groups, n_ptv, n_oar, n = _problem_case(seed=12)
    P = _gpu_problem(ctx, A, D, w, n_ptv, n_oar, n)
    O = _oracle_problem(A, D, w, n_ptv, n_oar)
    x0 = np.random.default_rng(1).random(n).astype(np.float32) * 0.02
    got = P.polish(x0, step_size=1e-3, iters=80)
    ref = O.polish(x0, step_size=1e-3, iters=80)
    np.testing.assert_allclose(got["loss"], ref["loss"], rtol=1e-3)
    assert got["loss"][-1] < got["loss"][0]


def test_half_precision_objective_within_a_tenth_percent(ctx):
    A, D, w, groups, n_ptv, n_oar, n = _problem_case(seed=13)
    x0 = np.random.default_rng(2).random(n).astype(np.float32) * 0.02
    res = {}
    for vt, fmt in (("f32", "i32"), ("f32", "packed16"), ("f16", "packed16"), ("bf16", "packed16")):
        P = _gpu_problem(ctx, A, D, w, n_ptv, n_oar, n, vt=vt, fmt=fmt)
        res[vt, fmt] = P.polish(x0, step_size=1e-3, iters=100)["loss"][-1]
    f32 = res["f32", "i32"]
    assert abs(res["f32", "packed16"] - f32) <= 1e-6 * abs(f32)  # same values, same order per row
    assert abs(res["f16", "packed16"] - f32) <= 1e-3 * abs(f32)
    assert abs(res["bf16", "packed16"] - f32) <= 1e-2 * abs(f32)


@pytest.mark.parametrize("vt,fmt", [("f32", "i32"), ("f16", "packed16")])
def test_voi_restriction_of_a_dose_matrix(ctx, vt, fmt):
    case = small_case()
    ph = case["phantom"]
    dens, sp, kn = api.Density(ctx, ph.density, ph.volume), api.Spectrum(ctx, case["spectrum"]), \
        api.Kernel(ctx, case["kernel"])
    ens = api.DoseMatConstruction(ctx, [case["beams"]], case["fluence"], dens, sp, kn, value_type=vt)
    ro, col, val = ens.to_host()
    nvox = ph.density.size
    rng = np.random.default_rng(9)
    vox = rng.permutation(nvox)
    ptv, oar = np.sort(vox[:3000]), np.sort(vox[3000:9000])
    voxel_row = np.full(nvox, -1, np.int32)
    voxel_row[ptv] = np.arange(len(ptv))
    voxel_row[oar] = len(ptv) + np.arange(len(oar))
    n_voi = len(ptv) + len(oar)
    A, AT = optimize.Matrix.voi(ctx, ens, voxel_row, n_voi, value_type=vt, index_format=fmt)
    assert A.shape == (n_voi, len(ro) - 1)
    # exact restriction on the host: keep, renumber, transpose
    rows = np.repeat(np.arange(len(ro) - 1), np.diff(ro))
    keep = voxel_row[col] >= 0
    dense = np.zeros((n_voi, len(ro) - 1), np.float32)
    dense[voxel_row[col[keep]], rows[keep]] = val[keep]
    a_off, a_col, a_val = A.to_host()
    got = np.zeros_like(dense)
    got[np.repeat(np.arange(n_voi), np.diff(a_off)), a_col] = a_val
    tol = 0.0 if vt == "f32" else 1e-6 * np.abs(dense).max()
    assert np.abs(got - dense).max() <= tol
    # the transpose holds the same values
    t_off, t_col, t_val = AT.to_host()
    got_t = np.zeros((len(ro) - 1, n_voi), np.float32)
    got_t[np.repeat(np.arange(len(ro) - 1), np.diff(t_off)), t_col] = t_val
    np.testing.assert_array_equal(got_t, got.T)
