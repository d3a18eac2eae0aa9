"""Multi-isocentre plan features (the head-and-neck configuration at a small
scale): one dose-loading matrix per isocentre, each with its own BEV grid
(12x12, 16x16, 20x20 sub-beam maps), beams of uneven beamlet counts including
one of 400 beamlets (the reference aborts above 327, IMRTDoseMat.cu:64-70),
concatenated on the device and optimized jointly with a 16-bit matrix."""
import numpy as np
import pytest

import oracle
from fastdose_b200 import api, optimize, phantoms
from fastdose_b200.types import make_bundle

pytestmark = pytest.mark.gpu


def _plan(ctx):
    cfg = phantoms.config4(n_per_iso=3, dim=(64, 64, 50))
    ph = cfg["phantom"]
    isos = []
    for k, iso in enumerate(cfg["isos"]):
        bundles = [make_bundle(iso["isocenter"], a, sad=cfg["sad"], fluence_dim=int(fd),
                               beamlet_size=cfg["beamlet_size"], sub_fluence_dim=iso["sub_fluence_dim"],
                               sub_fluence_on=cfg["sub_fluence_on"], long_spacing=cfg["long_spacing"])
                   for a, fd in zip(iso["angles"], iso["fluence_dims"])]
        if k == 0:  # a beam of 20x20 open beamlets (0.25 cm, inside this small phantom), all kept: 400 > 327
            bundles.append(make_bundle(iso["isocenter"], iso["angles"][0], sad=cfg["sad"], fluence_dim=20,
                                       beamlet_size=0.25, sub_fluence_dim=iso["sub_fluence_dim"],
                                       sub_fluence_on=cfg["sub_fluence_on"], long_spacing=cfg["long_spacing"]))
        bundles = np.array(bundles)
        # beamletFlagInit takes one fluence dimension per call (IMRTBeamBundle.cu:130)
        flags = [api.beamletFlagInit(ctx, bundles[j:j + 1], iso["mask"], ph.volume)[0] for j in range(len(bundles))]
        if k == 0:
            flags[-1][:] = 1
        beams = [api.bundle_beamlets(b, f, ph.volume) for b, f in zip(bundles, flags)]
        keep = [j for j, b in enumerate(beams) if len(b)]
        isos.append(dict(beams=[beams[j] for j in keep], flags=[np.asarray(flags[j]).reshape(-1) for j in keep],
                         fluence_dims=[int(bundles[j]["fluence_dim"][0]) for j in keep],
                         fluence=api.beamlet_fluence(bundles[0]), mask=iso["mask"]))
    return cfg, isos


def test_multi_isocentre_matrices_and_joint_optimization(ctx):
    cfg, isos = _plan(ctx)
    ph = cfg["phantom"]
    dens = api.Density(ctx, ph.density, ph.volume)
    spec, kern = api.Spectrum(ctx, cfg["spectrum"]), api.Kernel(ctx, cfg["kernel"])
    assert max(len(b) for b in isos[0]["beams"]) == 400
    parts, hosts = [], []
    for iso in isos:
        m = api.DoseMatConstruction(ctx, iso["beams"], iso["fluence"], dens, spec, kern)
        parts.append(m)
        hosts.append(m.to_host())
        # each beam alone gives the same rows, bit for bit
        ro, col, val = hosts[-1]
        r0 = 0
        for b in iso["beams"]:
            s = api.DoseMatConstruction(ctx, [b], iso["fluence"], dens, spec, kern)
            sro, scol, sval = s.to_host()
            s.close()
            a, z = ro[r0], ro[r0 + len(b)]
            np.testing.assert_array_equal(ro[r0:r0 + len(b) + 1] - a, sro)
            np.testing.assert_array_equal(col[a:z], scol)
            np.testing.assert_array_equal(val[a:z], sval)
            r0 += len(b)
    # one ensemble of all isocentres, in order
    joint = api.MatCSREnsemble.concat(ctx, parts)
    jro, jcol, jval = joint.to_host()
    np.testing.assert_array_equal(jcol, np.concatenate([h[1] for h in hosts]))
    np.testing.assert_array_equal(jval, np.concatenate([h[2] for h in hosts]))
    starts = np.cumsum([0] + [h[0][-1] for h in hosts[:-1]])
    np.testing.assert_array_equal(jro, np.concatenate([[0]] + [h[0][1:] + s0 for h, s0 in zip(hosts, starts)]))
    assert len(joint.mat_rows()) - 1 == sum(len(i["beams"]) for i in isos)

    # the 20x20 BEV grid (general march) against the FP64 oracle, one beam
    iso = isos[2]
    b = iso["beams"][0]
    ro, col, val = hosts[2]
    nv = ph.density.size
    gpu = np.zeros(nv, np.float64)
    np.add.at(gpu, col[:ro[len(b)]], val[:ro[len(b)]])
    ref = oracle.dose_rows(b, iso["fluence"], ph.density, ph.volume, cfg["spectrum"], cfg["kernel"],
                           threads=8).sum(0).astype(np.float64)
    dmax = ref.max()
    sel = ref > 0.1 * dmax
    assert np.abs(gpu - ref).max() <= 5e-2 * dmax
    assert np.abs(gpu - ref)[sel].mean() <= 1e-3 * dmax

    # joint optimization over all isocentres' beams with the FP16 matrix: PTV
    # rows (the union of the segments) then a ring of healthy tissue
    ptv = np.zeros(ph.density.shape, bool)
    for i in isos:
        ptv |= i["mask"].astype(bool)
    ring = (ph.density > 0.5) & ~ptv
    ring_idx = np.flatnonzero(ring.reshape(-1))[::5]
    ptv_idx = np.flatnonzero(ptv.reshape(-1))
    voxel_row = np.full(nv, -1, np.int32)
    voxel_row[ptv_idx] = np.arange(len(ptv_idx))
    voxel_row[ring_idx] = len(ptv_idx) + np.arange(len(ring_idx))
    n_ptv, n_oar = len(ptv_idx), len(ring_idx)
    A, AT = optimize.Matrix.voi(ctx, joint, voxel_row, n_ptv + n_oar, value_type="f16", index_format="packed16")
    beams_all = [bb for i in isos for bb in i["beams"]]
    n = A.shape[1]
    assert n == sum(len(bb) for bb in beams_all)
    D = optimize.block_diag([optimize.fluence_grad(fd, f) for i in isos
                             for fd, f in zip(i["fluence_dims"], i["flags"])])
    assert D[3] == n
    Dm = optimize.Matrix.from_csr(ctx, *D[:3], D[3])
    P = optimize.Problem(ctx, A, AT, Dm, Dm.transpose(), n_ptv, n_oar, np.full(n_ptv + n_oar, 1.1, np.float32),
                         np.ones(n_ptv + n_oar, np.float32), np.ones(n_ptv, np.float32), np.ones(n_ptv, np.float32),
                         np.full(n_oar, 0.05, np.float32), 1.0, 0.1)
    groups = np.concatenate([[0], np.cumsum([len(bb) for bb in beams_all])]).astype(np.int64)
    bw = 0.1 * P.beam_weights_init(groups)
    r = P.boo(groups, bw, np.full(n, 0.01, np.float32), step_size=1e-3, iters=30, want=0, change_trigger=10 ** 9)
    assert r["k"] == 30 and r["loss"][29] < r["loss"][0]
    for m in parts + [joint]:
        m.close()
