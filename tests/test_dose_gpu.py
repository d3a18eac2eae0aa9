"""CUDA dose path vs the CPU oracle: Terma, CCCS, BEV->PVCS, dose matrix.

Each stage is fed the same inputs on both sides, so the comparison isolates
that stage.  Tolerances: Terma and CCCS share every discrete decision with the
oracle (same float boundary arithmetic), so only rounding of the physics
differs (float vs double); the column stage point-samples, where a rounding
flip moves one of ss^3 samples to a neighbouring texel.  The whole-plan check
uses the dose tolerance of the parity gate: 0.5% of Dmax for the maximum
difference and 0.1% of Dmax for the mean over voxels above 10% of Dmax.
"""
import numpy as np
import pytest

import oracle
from fastdose_b200 import api

from plan_cases import c1_case, small_case

pytestmark = pytest.mark.gpu


def _setup(ctx, case, spectrum=None, kernel=None):
    ph = case["phantom"]
    spec = spectrum or case.get("spectrum") or case["cfg"]["spectrum"]
    kern = kernel or case.get("kernel") or case["cfg"]["kernel"]
    return (api.Density(ctx, ph.density, ph.volume), api.Spectrum(ctx, spec), api.Kernel(ctx, kern), spec, kern)


def _run_bev(ctx, case, idx, schedule=None):
    import torch

    dens, sp, kn, spec, kern = _setup(ctx, case)
    beams = case["beams"][idx]
    batch = api.BEVBatch(beams)
    api.TermaComputeCollective(ctx, batch, case["fluence"], dens, sp)
    api.DoseComputeCollective(ctx, batch, kn)
    torch.cuda.synchronize()
    out = []
    for i in range(len(beams)):
        out.append((batch.get("terma", i).cpu().numpy(), batch.get("dens", i).cpu().numpy(),
                    batch.get("dose", i).cpu().numpy()))
    return batch.beams, out, spec, kern


@pytest.mark.parametrize("case_fn,idx", [(small_case, [0, 5, 10, 15]), (c1_case, [0, 44, 93])])
def test_terma_matches_oracle(ctx, case_fn, idx):
    case = case_fn()
    beams, out, spec, _ = _run_bev(ctx, case, idx)
    for b, (T, R, _) in zip(beams, out):
        To, Ro = oracle.terma(b, case["fluence"], case["phantom"].density, case["phantom"].volume, spec)
        assert np.abs(T - To).max() <= 1e-4 * np.abs(To).max()
        assert np.abs(R - Ro).max() <= 1e-4 * np.abs(Ro).max()


@pytest.mark.parametrize("case_fn,idx", [(small_case, [0, 5, 10, 15]), (c1_case, [0, 44, 93])])
def test_cccs_matches_oracle(ctx, case_fn, idx):
    """The oracle marches with the device's cone directions; its boundary
    arithmetic is correctly rounded where the kernel reproduces the
    reference's fast division, so the two agree in the mean and up to the
    march's floating-point sensitivity at isolated voxels."""
    case = case_fn()
    beams, out, _, kern = _run_bev(ctx, case, idx)
    dirs = api.cone_directions(ctx, api.Kernel(ctx, kern), beams)
    for i, (b, (T, R, D)) in enumerate(zip(beams, out)):
        Do = oracle.cccs(b, T, R, kern, dirs=dirs[i])
        assert np.abs(D - Do).mean() <= 5e-4 * np.abs(Do).max()
        assert np.abs(D - Do).max() <= 5e-2 * np.abs(Do).max()


@pytest.mark.parametrize("case_fn", [small_case, c1_case], ids=["8x8", "16x16"])
def test_cccs_schedules_agree_bitwise(ctx, case_fn):
    """One block per beamlet and one block per (beamlet, zenith bin): the same
    matrix, bit for bit (the 8x8 map with 4x4 cones, and the 16x16 march with
    the 8x6 kernel)."""
    import torch

    case = case_fn()
    dens, sp, kn, _, _ = _setup(ctx, case)
    res = []
    for sched in (0, 1):
        m = api.DoseMatConstruction(ctx, [case["beams"]], case["fluence"], dens, sp, kn, cccs_schedule=sched)
        res.append(m.to_host())
        m.close()
    torch.cuda.synchronize()
    for a, b in zip(*res):
        np.testing.assert_array_equal(a, b)


def _dense(ro, col, val, n_rows, n_cols):
    out = np.zeros((n_rows, n_cols), np.float32)
    for r in range(n_rows):
        out[r, col[ro[r]:ro[r + 1]]] = val[ro[r]:ro[r + 1]]
    return out


def test_context_release_then_rebuild(ctx):
    """fd2_context_release hands the context's idle memory back; the next
    construction regrows its buffers and gives the same matrix, bit for bit."""
    c2 = api.Context(0)
    case = small_case()
    dens, sp, kn, _, _ = _setup(c2, case)
    ref = api.DoseMatConstruction(c2, [case["beams"]], case["fluence"], dens, sp, kn).to_host()
    c2.release()
    c2.release()  # nothing left to release: still fine
    again = api.DoseMatConstruction(c2, [case["beams"]], case["fluence"], dens, sp, kn)
    for a, b in zip(again.to_host(), ref):
        np.testing.assert_array_equal(a, b)
    again.close()


def test_rule_cccs_schedule(ctx):
    """cccs_schedule = -2 picks a schedule by rule, without a timing run: the
    same matrix as either fixed schedule, bit for bit, and nothing tuned."""
    from fastdose_b200 import _lib

    c2 = api.Context(0)
    case = small_case()
    dens, sp, kn, _, _ = _setup(c2, case)
    ref = api.DoseMatConstruction(c2, [case["beams"]], case["fluence"], dens, sp, kn, cccs_schedule=0).to_host()
    rule = api.DoseMatConstruction(c2, [case["beams"]], case["fluence"], dens, sp, kn, cccs_schedule=-2)
    for a, b in zip(rule.to_host(), ref):
        np.testing.assert_array_equal(a, b)
    assert c2.tuned_schedules() == ({}, 0)
    with pytest.raises(_lib.FD2Error):
        api.DoseMatConstruction(c2, [case["beams"]], case["fluence"], dens, sp, kn, cccs_schedule=-3)
    rule.close()


def test_tuned_cccs_schedule(ctx):
    """The automatic schedule times both schedules on the first batch of a
    shape, then reuses the choice; every build gives the same matrix as either
    fixed schedule, bit for bit."""
    from fastdose_b200 import api as _api

    c2 = _api.Context(0)  # a fresh context: no tuned shapes yet
    case = small_case()
    dens, sp, kn, _, _ = _setup(c2, case)
    fixed = [_api.DoseMatConstruction(c2, [case["beams"]], case["fluence"], dens, sp, kn, cccs_schedule=s)
             for s in (0, 1)]
    ref = [m.to_host() for m in fixed]
    for a, b in zip(*ref):
        np.testing.assert_array_equal(a, b)
    assert c2.tuned_schedules() == ({}, 0)
    for k in range(2):
        m = _api.DoseMatConstruction(c2, [case["beams"]], case["fluence"], dens, sp, kn)
        for a, b in zip(m.to_host(), ref[0]):
            np.testing.assert_array_equal(a, b)
        m.close()
        sched, runs = c2.tuned_schedules()
        assert runs == 1 and len(sched) == 1 and list(sched.values())[0] in (0, 1)
    for h in fixed + [dens, sp, kn]:
        h.close()
    c2.close()


@pytest.mark.parametrize("vt,sched", [("f32", 0), ("f16", 1), ("f32", -1)])
def test_graph_captured_construction_matches_direct(vt, sched):
    """Batches launched as captured CUDA graphs give the matrix of direct
    launches bit for bit, over several batches of one shape (the executable
    graph is instantiated once and updated in place for the others) and over
    a second plan on the same context."""
    from fastdose_b200 import api as _api

    c2 = _api.Context(0)
    case = c1_case()
    dens, sp, kn, _, _ = _setup(c2, case)
    beams = [case["beams"][i:i + 10] for i in range(0, 100, 10)]  # 10 beams of 10 beamlets
    fixed = -2 if sched < 0 else sched  # graph mode fixes the schedule per batch
    ref = _api.DoseMatConstruction(c2, beams, case["fluence"], dens, sp, kn, value_type=vt, cccs_schedule=fixed,
                                   batch_beamlets=30)
    want = ref.to_host()
    rows_want = ref.mat_rows()
    for rep in range(2):
        m = _api.DoseMatConstruction(c2, beams, case["fluence"], dens, sp, kn, value_type=vt, cccs_schedule=sched,
                                     batch_beamlets=30, graph=True)
        for a, b in zip(m.to_host(), want):
            np.testing.assert_array_equal(a, b)
        np.testing.assert_array_equal(m.mat_rows(), rows_want)
        m.close()
    launches, inst, updates = c2.graph_counts()
    # four batches per plan (30, 30, 30, 10 beamlets), two plans
    assert launches == 8 and inst >= 1 and inst + updates == 8
    assert inst <= 2, f"{inst} instantiations: the in-place update was refused"
    for h in (ref, dens, sp, kn):
        h.close()
    c2.close()


def test_graph_construction_refuses_host_out(ctx):
    from fastdose_b200 import _lib

    case = small_case()
    dens, sp, kn, _, _ = _setup(ctx, case)
    host = api.HostCSR(len(case["beams"]), 10 ** 6)
    with pytest.raises(_lib.FD2Error):
        api.DoseMatConstruction(ctx, [case["beams"]], case["fluence"], dens, sp, kn, host_out=host, graph=True)


def test_columns_match_oracle(ctx):
    case = small_case()
    beams, out, _, _ = _run_bev(ctx, case, list(range(16)))
    dens, sp, kn, _, _ = _setup(ctx, case)
    m = api.DoseMatConstruction(ctx, [case["beams"]], case["fluence"], dens, sp, kn)
    ro, col, val = m.to_host()
    nv = case["phantom"].density.size
    A = _dense(ro, col, val, 16, nv)
    for i, b in enumerate(beams):
        row = oracle.beamlet_column(b, out[i][2], case["phantom"].volume)
        mx = np.abs(row).max()
        assert np.abs(A[i] - row).max() <= 0.01 * mx
        assert np.abs(A[i] - row).mean() <= 1e-4 * mx
        # same support except where the oracle value is within a sample flip of 0
        diff = (A[i] != 0) != (row != 0)
        assert np.all(np.abs(row[diff]) <= 0.01 * mx)


def test_csr_structure_and_file_round_trip(ctx, tmp_path):
    case = small_case()
    dens, sp, kn, _, _ = _setup(ctx, case)
    m = api.DoseMatConstruction(ctx, [case["beams"][:7], case["beams"][7:]], case["fluence"], dens, sp, kn)
    info = m.info()
    assert info["n_mats"] == 2 and info["n_rows"] == 16
    ro, col, val = m.to_host()
    assert ro[0] == 0 and np.all(np.diff(ro) >= 0) and ro[-1] == info["nnz"]
    for r in range(16):
        c = col[ro[r]:ro[r + 1]]
        assert np.all(np.diff(c) > 0)
        assert c.min() >= 0 and c.max() < info["n_cols"]
    assert np.all(val != 0)
    np.testing.assert_array_equal(m.mat_rows(), [0, 7, 16])
    m.tofile(tmp_path)
    # the reference layout: uint64 per-matrix arrays, local offsets, uint64 columns
    nnz = np.fromfile(tmp_path / "NonZeroElements.bin", np.uint64)
    np.testing.assert_array_equal(nnz, [ro[7] - ro[0], ro[16] - ro[7]])
    np.testing.assert_array_equal(np.fromfile(tmp_path / "CumuNonZeroElements.bin", np.uint64), np.cumsum(nnz))
    np.testing.assert_array_equal(np.fromfile(tmp_path / "numRowsPerMat.bin", np.uint64), [7, 9])
    np.testing.assert_array_equal(np.fromfile(tmp_path / "CumuNumRowsPerMat.bin", np.uint64), [7, 16])
    np.testing.assert_array_equal(np.fromfile(tmp_path / "OffsetBufferIdx.bin", np.uint64), [0, 8])
    offs = np.fromfile(tmp_path / "offsetsBuffer.bin", np.uint64)
    np.testing.assert_array_equal(offs[:8], ro[:8] - ro[0])
    np.testing.assert_array_equal(offs[8:], ro[7:] - ro[7])
    np.testing.assert_array_equal(np.fromfile(tmp_path / "columnsBuffer.bin", np.uint64), col)
    np.testing.assert_array_equal(np.fromfile(tmp_path / "valuesBuffer.bin", np.float32), val)
    m2 = api.MatCSREnsemble.fromfile(ctx, tmp_path, info["n_cols"])
    for a, b in zip(m2.to_host(), (ro, col, val)):
        np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(m2.mat_rows(), [0, 7, 16])


@pytest.mark.parametrize("vt,rel", [("f16", 2 ** -11), ("bf16", 2 ** -8)])
def test_half_precision_matrix(ctx, vt, rel):
    case = small_case()
    dens, sp, kn, _, _ = _setup(ctx, case)
    ref = api.DoseMatConstruction(ctx, [case["beams"]], case["fluence"], dens, sp, kn).to_host()
    half = api.DoseMatConstruction(ctx, [case["beams"]], case["fluence"], dens, sp, kn, value_type=vt)
    ro, col, val = half.to_host()
    np.testing.assert_array_equal(ro, ref[0])
    np.testing.assert_array_equal(col, ref[1])
    for r in range(len(ro) - 1):
        a, b = val[ro[r]:ro[r + 1]], ref[2][ro[r]:ro[r + 1]]
        assert np.abs(a - b).max() <= rel * np.abs(b).max() * 1.01


@pytest.mark.parametrize("vt", ["f16", "bf16"])
def test_half_precision_file_round_trip(ctx, tmp_path, vt):
    """A 16-bit ensemble written to a doseMatFolder: the reference's files hold
    the decoded float32 values, the sidecars the stored bits; loading the
    sidecars gives back the same ensemble bit for bit.  A folder without them
    (the reference's own) is refused for a 16-bit load."""
    case = small_case()
    dens, sp, kn, _, _ = _setup(ctx, case)
    half = api.DoseMatConstruction(ctx, [case["beams"]], case["fluence"], dens, sp, kn, value_type=vt)
    ro, col, val = half.to_host()
    half.tofile(tmp_path / "m")
    np.testing.assert_array_equal(np.fromfile(tmp_path / "m" / "valuesBuffer.bin", np.float32), val)
    assert (tmp_path / "m" / f"valuesBuffer.{vt}.bin").stat().st_size == 2 * len(val)
    back = api.MatCSREnsemble.fromfile(ctx, tmp_path / "m", case["phantom"].density.size, value_type=vt)
    assert back.info()["value_type"] == half.info()["value_type"]
    for a, b in zip(back.to_host(), (ro, col, val)):
        np.testing.assert_array_equal(a, b)
    f32 = api.DoseMatConstruction(ctx, [case["beams"]], case["fluence"], dens, sp, kn)
    f32.tofile(tmp_path / "r")
    from fastdose_b200 import _lib

    with pytest.raises(_lib.FD2Error) as e:
        api.MatCSREnsemble.fromfile(ctx, tmp_path / "r", case["phantom"].density.size, value_type=vt)
    assert "sidecar" in str(e.value)
    for m in (half, back, f32):
        m.close()


def test_dose_matrix_c1_matches_oracle(ctx):
    """Whole config-1 plan (100 beamlets, 6 azimuths) against the FP64 oracle:
    the mean criterion of the parity gate; the maximum is bounded by the
    march's floating-point sensitivity (see test_reference_parity.py)."""
    case = c1_case()
    dens, sp, kn, spec, kern = _setup(ctx, case)
    m = api.DoseMatConstruction(ctx, [case["beams"]], case["fluence"], dens, sp, kn)
    ro, col, val = m.to_host()
    nv = case["phantom"].density.size
    gpu = np.zeros(nv, np.float64)
    np.add.at(gpu, col, val)
    rows = oracle.dose_rows(case["beams"], case["fluence"], case["phantom"].density, case["phantom"].volume, spec,
                            kern, threads=8)
    ref = rows.sum(0).astype(np.float64)
    dmax = ref.max()
    sel = ref > 0.1 * dmax
    assert np.abs(gpu - ref).max() <= 5e-2 * dmax
    assert np.abs(gpu - ref)[sel].mean() <= 1e-3 * dmax


def _decode16(words, scale, ro, vt):
    w = np.asarray(words).view(np.uint16)
    v = w.view(np.float16).astype(np.float32) if vt == "f16" else (w.astype(np.uint32) << 16).view(np.float32)
    rows = np.repeat(np.arange(len(ro) - 1), np.diff(ro))
    return (v * np.asarray(scale, np.float32)[rows]).astype(np.float32)


@pytest.mark.parametrize("vt", ["f32", "f16", "bf16"])
def test_host_copy_while_building(ctx, vt):
    """host_out receives the matrix batch by batch during the construction
    (small batches force several overlapped copies): the same arrays as the
    finished ensemble's read-back, bit for bit.  A buffer that is too small
    is refused with a capacity error and nothing is left in flight."""
    from fastdose_b200 import _lib

    case = c1_case()
    dens, sp, kn, _, _ = _setup(ctx, case)
    beams = [case["beams"][i:i + 10] for i in range(0, len(case["beams"]), 10)]
    ref = api.DoseMatConstruction(ctx, beams, case["fluence"], dens, sp, kn, value_type=vt)
    ro_r, col_r, val_r = ref.to_host()
    nnz = int(ro_r[-1])
    host = api.HostCSR(len(ro_r) - 1, nnz + 17, value_type=vt)
    for batch in (0, 16, 33):
        m = api.DoseMatConstruction(ctx, beams, case["fluence"], dens, sp, kn, value_type=vt, batch_beamlets=batch,
                                    host_out=host)
        ro, col, val, sc = host.arrays()
        assert host.nnz == nnz and host.n_rows == len(ro_r) - 1
        np.testing.assert_array_equal(ro, ro_r)
        np.testing.assert_array_equal(col, col_r)
        if vt == "f32":
            np.testing.assert_array_equal(val, val_r)
        else:
            np.testing.assert_array_equal(_decode16(val, sc, ro, vt), val_r)
        assert host.nbytes() == (len(ro_r)) * 8 + nnz * (4 + (4 if vt == "f32" else 2)) + \
            (0 if vt == "f32" else (len(ro_r) - 1) * 4)
        m.close()
    small = api.HostCSR(len(ro_r) - 1, nnz // 2, value_type=vt)
    with pytest.raises(_lib.FD2Error) as e:
        api.DoseMatConstruction(ctx, beams, case["fluence"], dens, sp, kn, value_type=vt, batch_beamlets=16,
                                host_out=small)
    assert "host_out holds" in str(e.value)
    # the context is still usable
    again = api.DoseMatConstruction(ctx, beams, case["fluence"], dens, sp, kn, value_type=vt)
    np.testing.assert_array_equal(again.to_host()[0], ro_r)
    for mm in (ref, again):
        mm.close()


@pytest.mark.parametrize("vt", ["f32", "f16"])
def test_overlapped_column_stage_matches_one_stream(ctx, vt):
    """The column stage of each batch on the context's second stream, beside
    the next batch's Terma and CCCS in the other BEV buffer (the default), and
    the whole construction on one stream: the same matrix, bit for bit, for
    one batch and for several (batches of 10, 20 and 30 beamlets, so BEV
    buffers are reused and regrown while a column stage may still read them)."""
    case = c1_case()
    dens, sp, kn, _, _ = _setup(ctx, case)
    beams = [case["beams"][i:i + 10] for i in range(0, len(case["beams"]), 10)]
    ref = api.DoseMatConstruction(ctx, beams, case["fluence"], dens, sp, kn, value_type=vt, overlap=False)
    ref_h = ref.to_host()
    for batch in (0, 30, 10, 20):
        m = api.DoseMatConstruction(ctx, beams, case["fluence"], dens, sp, kn, value_type=vt, batch_beamlets=batch)
        for a, b in zip(m.to_host(), ref_h):
            np.testing.assert_array_equal(a, b)
        np.testing.assert_array_equal(m.mat_rows(), ref.mat_rows())
        m.close()
    ref.close()


def test_construction_with_empty_beams(ctx):
    """Beams without beamlets (a beam whose flags are all off) anywhere in the
    plan add no rows and repeat their neighbour's row boundary; the rows are
    those of the plan without them, bit for bit, with and without the column
    overlap and over several batchings.  A plan of empty beams only gives an
    empty matrix."""
    from fastdose_b200.types import BEAM_DTYPE

    case = c1_case()
    dens, sp, kn, _, _ = _setup(ctx, case)
    b = case["beams"]
    empty = np.zeros(0, BEAM_DTYPE)
    ref = api.DoseMatConstruction(ctx, [b[:30], b[30:]], case["fluence"], dens, sp, kn)
    ref_h = ref.to_host()
    plan = [empty, b[:30], empty, empty, b[30:], empty]
    for overlap in (True, False):
        for batch in (0, 16):
            m = api.DoseMatConstruction(ctx, plan, case["fluence"], dens, sp, kn, overlap=overlap,
                                        batch_beamlets=batch)
            for x, y in zip(m.to_host(), ref_h):
                np.testing.assert_array_equal(x, y)
            np.testing.assert_array_equal(m.mat_rows(), [0, 0, 30, 30, 30, 100, 100])
            m.close()
    for overlap in (True, False):
        z = api.DoseMatConstruction(ctx, [empty, empty], case["fluence"], dens, sp, kn, overlap=overlap)
        ro, col, val = z.to_host()
        assert z.info()["nnz"] == 0 and len(col) == 0 and ro.tolist() == [0]
        np.testing.assert_array_equal(z.mat_rows(), [0, 0, 0])
        z.close()
    ref.close()


def test_density_outlives_its_context(ctx):
    """A density is freed after its context was destroyed (the Python objects
    of a caller can go in any order): no error, and later work on another
    context is unaffected."""
    import torch

    case = small_case()
    c2 = api.Context(0)
    d2 = api.Density(c2, case["phantom"].density, case["phantom"].volume)
    c2.close()
    d2.close()
    dens, sp, kn, _, _ = _setup(ctx, case)
    m = api.DoseMatConstruction(ctx, [case["beams"]], case["fluence"], dens, sp, kn)
    torch.cuda.synchronize()
    assert m.info()["nnz"] > 0
    m.close()


def _write_folder(path, mats, vals_dtype=np.float32):
    """A doseMatFolder (the reference's layout) from host CSR matrices."""
    path.mkdir(parents=True, exist_ok=True)
    nrows = np.array([len(ro) - 1 for ro, _, _ in mats], np.uint64)
    nnz = np.array([ro[-1] for ro, _, _ in mats], np.uint64)
    nrows.tofile(path / "numRowsPerMat.bin")
    np.cumsum(nrows).astype(np.uint64).tofile(path / "CumuNumRowsPerMat.bin")
    nnz.tofile(path / "NonZeroElements.bin")
    np.cumsum(nnz).astype(np.uint64).tofile(path / "CumuNonZeroElements.bin")
    np.concatenate([[0], np.cumsum(nrows + 1)[:-1]]).astype(np.uint64).tofile(path / "OffsetBufferIdx.bin")
    np.concatenate([np.asarray(ro, np.uint64) for ro, _, _ in mats]).tofile(path / "offsetsBuffer.bin")
    np.concatenate([np.asarray(c, np.uint64) for _, c, _ in mats]).tofile(path / "columnsBuffer.bin")
    np.concatenate([np.asarray(v, vals_dtype) for _, _, v in mats]).tofile(path / "valuesBuffer.bin")


def test_fromfile_streams_large_folders(ctx, tmp_path):
    """A folder of 9.4M nonzeros in two matrices loads in several streamed
    chunks: the same row offsets, columns and values as written.  A column
    outside the volume is refused."""
    rng = np.random.default_rng(21)
    n_cols = 2_000_000
    mats = []
    for rows, per in ((300, 20_000), (170, 20_000)):
        lens = rng.integers(per // 2, per * 3 // 2, rows)
        ro = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
        col = np.concatenate([np.sort(rng.integers(0, n_cols, l)) for l in lens]).astype(np.int64)
        val = rng.random(ro[-1]).astype(np.float32)
        mats.append((ro, col, val))
    _write_folder(tmp_path / "big", mats)
    m = api.MatCSREnsemble.fromfile(ctx, tmp_path / "big", n_cols)
    ro, col, val = m.to_host()
    assert m.info()["nnz"] == sum(int(x[0][-1]) for x in mats) > 8_400_000
    ro_ref = np.concatenate([mats[0][0], mats[1][0][1:] + mats[0][0][-1]])
    np.testing.assert_array_equal(ro, ro_ref)
    np.testing.assert_array_equal(col, np.concatenate([mats[0][1], mats[1][1]]))
    np.testing.assert_array_equal(val, np.concatenate([mats[0][2], mats[1][2]]))
    np.testing.assert_array_equal(m.mat_rows(), [0, 300, 470])
    m.close()
    from fastdose_b200 import _lib

    bad = [(mats[0][0], mats[0][1].copy(), mats[0][2])]
    bad[0][1][-1] = n_cols  # one index past the volume, in the last chunk
    _write_folder(tmp_path / "bad", bad)
    with pytest.raises(_lib.FD2Error) as e:
        api.MatCSREnsemble.fromfile(ctx, tmp_path / "bad", n_cols)
    assert "outside" in str(e.value)
    # an index of 2^31 would wrap negative as int32: a volume that large is
    # refused before any column is read
    huge = [(mats[1][0], mats[1][1].copy(), mats[1][2])]
    huge[0][1][-1] = 2**31
    _write_folder(tmp_path / "huge", huge)
    with pytest.raises(_lib.FD2Error) as e:
        api.MatCSREnsemble.fromfile(ctx, tmp_path / "huge", 2**31 + 1)
    assert "int32" in str(e.value)
