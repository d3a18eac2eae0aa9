"""Generates the dose-path golden fixtures by running the REFERENCE's own CUDA
kernels (oracle/_ref/libfdref.so, built from the reference sources by
oracle/build_ref.sh) on a GPU:

  dose_c1_ref.npz     config 1 (64^3 slab phantom, 100 beamlets): Terma, density
                      and dose BEV of four beamlets, their dose columns, the
                      summed dose of all 100 columns, per-beamlet nnz, timings
  dose_small_ref.npz  a small oblique case (all 16 beamlets)
  bev2pvcs_ref.npz    fastdose::BEV2PVCS of one beamlet's dose (texture path)
  flags_c2_ref.npz    beamletFlagInit of the 4pi torso bundles
  dose_c2_ref.npz     the 4pi torso plan (config 2): two beamlets from each of
                      six oblique beams -- Terma and dose BEV of the first,
                      the interpolated dose column of both
  bev2pvcs_ss_ref.npz fastdose::BEV2PVCS_SuperSampling of config-1 beamlet 44
  dose_c4_ref.npz     the multi-isocentre case: two beamlets each from two
                      isocentres with 24x24 sub-beam maps (Terma, density and
                      dose BEV, columns)
  reference_timings.json  kernel times, and IMRT::DoseMatConstruction's steps
                      over the whole 4pi plan (part "c2full")

Usage (on a GPU machine): python tests/golden/make_golden_dose.py OUTDIR [part ...]
with parts from c1 small flags c2timing c2 ss c2full c4 (default: all).  The
fixtures are then copied next to this script; reference_timings.json is
updated in place, keeping the keys of parts not rerun.
"""
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from fastdose_b200 import phantoms  # noqa: E402
from fastdose_b200.types import make_bundle  # noqa: E402
from oracle import ref  # noqa: E402
from plan_cases import c1_case, small_case  # noqa: E402

PICK = [0, 44, 55, 93]


def ref_kernel():
    """The CCCS kernel used for every reference run: 8 zenith x 8 azimuth bins
    (the reference's default nPhi, IMRTOpt/src/IMRTArgs.cpp:47).  With 6
    azimuths one cone lies at phi = 90 degrees, where the reference's fast-math
    direction has a zero component and its ray march divides by zero and never
    finishes a slice; it is not run that way."""
    return phantoms.synthetic_kernel(n_theta=8, n_phi=8)


def log(*a):
    print(*a, flush=True)


def _csr_rows(dense, rows):
    out = {}
    for r in rows:
        nz = np.nonzero(dense[r])[0]
        out[f"col_{r}"] = nz.astype(np.int32)
        out[f"val_{r}"] = dense[r, nz]
    return out


def c1(outdir):
    case = c1_case()
    cfg = case["cfg"]
    ph = case["phantom"]
    kern = ref_kernel()
    log("c1: reference batch of", len(case["beams"]), "beamlets")
    r = ref.dose_batch(case["beams"], case["fluence"], ph.density, ph.volume, cfg["spectrum"], kern,
                       extent=cfg["extent"], dense=True, repeats=1)
    assert r["status"] == 0, r["status"]
    log("c1: done, timing")
    # timing of the reference kernels on the same batch (three repeats)
    t = ref.dose_batch(case["beams"], case["fluence"], ph.density, ph.volume, cfg["spectrum"], kern,
                       extent=cfg["extent"], dense=True, repeats=3)["times_ms"]
    log("c1: times", t)
    dense = r["dense"]
    keep = {}
    for i in PICK:
        L = int(case["beams"][i]["long_dim"])
        keep[f"terma_{i}"] = r["terma"][i, :L]
        keep[f"dens_{i}"] = r["dens"][i, :L]
        keep[f"dose_{i}"] = r["dose"][i, :L]
    nx, ny, nz = (int(v) for v in ph.volume["dim"])
    np.savez_compressed(os.path.join(outdir, "dose_c1_ref.npz"), beams=case["beams"], pick=np.array(PICK),
                        kernel_theta=kern.theta, kernel_A=kern.A, kernel_a=kern.a, kernel_B=kern.B,
                        kernel_b=kern.b, kernel_phi=kern.phi,
                        dose_sum=dense.sum(0).reshape(nz, ny, nx).astype(np.float32),
                        nnz=(dense != 0).sum(1).astype(np.int64), times_ms=t, **keep, **_csr_rows(dense, PICK))
    # dense trilinear resampling of beamlet 44's dose
    b = case["beams"][44]
    st, vol = ref.bev2pvcs(b, r["dose"][44, : int(b["long_dim"])], ph.volume)
    assert st == 0
    np.savez_compressed(os.path.join(outdir, "bev2pvcs_ref.npz"), beam=b, bev=r["dose"][44, : int(b["long_dim"])],
                        out=vol)
    return dict(c1_terma_ms=float(t[0]), c1_cccs_ms=float(t[1]), c1_interp_ms=float(t[2]),
                c1_beamlets=int(len(case["beams"])))


def small(outdir):
    case = small_case()
    ph = case["phantom"]
    log("small: reference batch")
    r = ref.dose_batch(case["beams"], case["fluence"], ph.density, ph.volume, case["spectrum"], case["kernel"],
                       extent=2.0, dense=True)
    assert r["status"] == 0
    L = case["beams"]["long_dim"]
    keep = {f"{k}_{i}": r[k][i, : int(L[i])] for k in ("terma", "dens", "dose") for i in range(len(L))}
    np.savez_compressed(os.path.join(outdir, "dose_small_ref.npz"), beams=case["beams"], dense=r["dense"], **keep)


def flags(outdir):
    cfg = phantoms.config2()
    ph = cfg["phantom"]
    bundles = np.array([make_bundle(cfg["isocenter"], a, sad=cfg["sad"], fluence_dim=cfg["fluence_dim"],
                                    beamlet_size=cfg["beamlet_size"], sub_fluence_dim=cfg["sub_fluence_dim"],
                                    sub_fluence_on=cfg["sub_fluence_on"], long_spacing=cfg["long_spacing"])
                        for a in cfg["angles"]])
    log("flags: reference beamletFlagInit of", len(bundles), "bundles")
    st, fl = ref.beamlet_flags(bundles, ph.masks["PTV"], ph.volume, ph.density)
    assert st == 0
    np.savez_compressed(os.path.join(outdir, "flags_c2_ref.npz"), bundles=bundles, flags=fl)
    return dict(c2_beams=int(len(bundles)), c2_active_beamlets=int(fl.sum()))


def c2_timing(outdir, n_beams=8):
    """Reference Terma + CCCS of whole 4pi beams (its interpolation stage is
    not run on this volume: its supervoxel pass writes past its flag array when
    the volume is not a multiple of 32 voxels)."""
    cfg = phantoms.config2()
    ph = cfg["phantom"]
    fl = np.load(os.path.join(outdir, "flags_c2_ref.npz"))["flags"]
    from fastdose_b200 import api

    tot_b, tot_ms = 0, 0.0
    for i in range(0, len(cfg["angles"]), max(1, len(cfg["angles"]) // n_beams))[:n_beams]:
        bb = make_bundle(cfg["isocenter"], cfg["angles"][i], sad=cfg["sad"], fluence_dim=cfg["fluence_dim"],
                         beamlet_size=cfg["beamlet_size"], sub_fluence_dim=cfg["sub_fluence_dim"],
                         sub_fluence_on=cfg["sub_fluence_on"], long_spacing=cfg["long_spacing"])
        beams = api.bundle_beamlets(bb, fl[i], ph.volume)
        if len(beams) == 0:
            continue
        log("c2 timing: beam", i, len(beams), "beamlets")
        t = ref.dose_batch(beams, api.beamlet_fluence(bb), ph.density, ph.volume, cfg["spectrum"], ref_kernel(),
                           dense=False, repeats=1)["times_ms"]
        tot_b += len(beams)
        tot_ms += float(t[0] + t[1])
    return dict(c2_sample_beams=n_beams, c2_sample_beamlets=tot_b, c2_terma_cccs_ms=tot_ms,
                c2_ref_beamlets_per_s=tot_b / (tot_ms * 1e-3) if tot_ms else None)


C2_PICK_BEAMS = (0, 67, 134, 201, 268, 335)


def _c2_plan():
    cfg = phantoms.config2()
    bundles = np.array([make_bundle(cfg["isocenter"], a, sad=cfg["sad"], fluence_dim=cfg["fluence_dim"],
                                    beamlet_size=cfg["beamlet_size"], sub_fluence_dim=cfg["sub_fluence_dim"],
                                    sub_fluence_on=cfg["sub_fluence_on"], long_spacing=cfg["long_spacing"])
                        for a in cfg["angles"]])
    fl = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "flags_c2_ref.npz"))["flags"]
    return cfg, bundles, fl


def c2(outdir):
    """Sampled beamlets of the 4pi torso plan through the reference's Terma,
    CCCS and batched interpolation (8x8 cone kernel)."""
    from fastdose_b200 import api

    cfg, bundles, fl = _c2_plan()
    ph = cfg["phantom"]
    kern = ref_kernel()
    keep = {}
    beams_all = []
    for bi in C2_PICK_BEAMS:
        beams = api.bundle_beamlets(bundles[bi], fl[bi], ph.volume)
        assert len(beams) >= 2, (bi, len(beams))
        sel = beams[[len(beams) // 2, 0]]
        log("c2: beam", bi, "beamlets", len(beams), "picked long_dim", sel["long_dim"])
        r = ref.dose_batch(sel, api.beamlet_fluence(bundles[bi]), ph.density, ph.volume, cfg["spectrum"], kern,
                           extent=cfg["extent"], dense=True)
        assert r["status"] == 0, r["status"]
        j = len(beams_all)
        L = int(sel[0]["long_dim"])
        keep[f"terma_{j}"] = r["terma"][0, :L]
        keep[f"dose_{j}"] = r["dose"][0, :L]
        for k in range(2):
            nz = np.nonzero(r["dense"][k])[0]
            keep[f"col_{j + k}"] = nz.astype(np.int32)
            keep[f"val_{j + k}"] = r["dense"][k, nz]
        beams_all.extend(sel)
    np.savez_compressed(os.path.join(outdir, "dose_c2_ref.npz"), beams=np.array(beams_all),
                        beam_index=np.repeat(C2_PICK_BEAMS, 2), kernel_phi=kern.phi, **keep)


def ss(outdir):
    """BEV2PVCS_SuperSampling of config-1 beamlet 44's dose BEV."""
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "dose_c1_ref.npz"))
    case = c1_case()
    b = case["beams"][44]
    bev = g["dose_44"]
    out = {}
    for ssf, ext in ((5, 2.0), (3, 0.6)):
        st, vol = ref.bev2pvcs_ss(b, bev, case["phantom"].volume, ssfactor=ssf, extent=ext)
        assert st == 0
        out[f"out_{ssf}"] = vol
    np.savez_compressed(os.path.join(outdir, "bev2pvcs_ss_ref.npz"), beam=b, **out)


def c2full(outdir):
    """IMRT::DoseMatConstruction's steps over the whole 4pi plan."""
    cfg, bundles, fl = _c2_plan()
    ph = cfg["phantom"]
    t0 = time.time()
    r = ref.dose_mat_steps(bundles, fl, ph.density, ph.volume, cfg["spectrum"], ref_kernel(), extent=cfg["extent"])
    wall = time.time() - t0
    assert r["status"] == 0, r["status"]
    t = r["times_ms"]
    log("c2full:", r["beamlets"], "beamlets", t, "ms, nnz", int(r["nnz"].sum()))
    return dict(c2full_beamlets=int(r["beamlets"]), c2full_terma_ms=float(t[0]), c2full_cccs_ms=float(t[1]),
                c2full_interp_ms=float(t[2]), c2full_dense_to_csr_ms=float(t[3]), c2full_total_ms=float(t[4]),
                c2full_nnz=int(r["nnz"].sum()), c2full_wall_s=wall,
                c2full_beamlets_per_s=r["beamlets"] / (float(t[4]) * 1e-3))


C4_MAPS = (24, 16, 24, 16)


def c4(outdir):
    """Two beamlets each from isocentres 0 and 2 of the small multi-isocentre
    head-and-neck case, with 24x24 sub-beam maps, through the reference's
    Terma, CCCS and batched interpolation with the 8x8 kernel.

    The reference's CCCS block has one thread per map pixel rounded up to a
    warp, and the threads past the map return (DoseComp.cu:236) before the
    block-wide barriers and the block-wide async slice copy (DoseComp.cu:295,
    305-309, 382).  Maps whose pixel count is not a multiple of 32 (12x12,
    20x20) are therefore outside its defined behaviour and are not run here.
    24x24 (576 pixels) is, and at 8 azimuths its dynamic shared memory
    (20 x 576 x 4 + 192 bytes) stays under the 48 KB the launch gets without
    an opt-in (DoseComp.cu:203-205)."""
    from fastdose_b200 import api

    cfg = phantoms.config4(n_per_iso=3, dim=(64, 64, 50), sub_fluence_dims=C4_MAPS)
    ph = cfg["phantom"]
    kern = ref_kernel()
    keep = {}
    for k in (0, 2):
        iso = cfg["isos"][k]
        fd = int(iso["fluence_dims"][1])
        bb = make_bundle(iso["isocenter"], iso["angles"][1], sad=cfg["sad"], fluence_dim=fd,
                         beamlet_size=cfg["beamlet_size"], sub_fluence_dim=iso["sub_fluence_dim"],
                         sub_fluence_on=cfg["sub_fluence_on"], long_spacing=cfg["long_spacing"])
        flags = np.zeros(fd * fd, np.uint8)
        flags[(fd // 2) * fd + fd // 2] = flags[(fd // 2 - 1) * fd + fd // 2 - 1] = 1  # two central beamlets
        beams = api.bundle_beamlets(bb, flags, ph.volume)
        log("c4: isocentre", k, "map", iso["sub_fluence_dim"], "long_dim", beams["long_dim"])
        r = ref.dose_batch(beams, api.beamlet_fluence(bb), ph.density, ph.volume, cfg["spectrum"], kern,
                           extent=cfg["extent"], dense=True)
        assert r["status"] == 0, r["status"]
        keep[f"beams_{k}"] = beams
        keep[f"fluence_{k}"] = api.beamlet_fluence(bb)
        for j in range(2):
            L = int(beams[j]["long_dim"])
            keep[f"terma_{k}_{j}"] = r["terma"][j, :L]
            keep[f"dens_{k}_{j}"] = r["dens"][j, :L]
            keep[f"dose_{k}_{j}"] = r["dose"][j, :L]
            nz = np.nonzero(r["dense"][j])[0]
            keep[f"col_{k}_{j}"] = nz.astype(np.int32)
            keep[f"val_{k}_{j}"] = r["dense"][j, nz]
    np.savez_compressed(os.path.join(outdir, "dose_c4_ref.npz"), kernel_phi=kern.phi, **keep)


PARTS = ("c1", "small", "flags", "c2timing", "c2", "ss", "c2full", "c4")


def main():
    outdir = sys.argv[1] if len(sys.argv) > 1 else os.path.dirname(os.path.abspath(__file__))
    parts = sys.argv[2:] or PARTS
    os.makedirs(outdir, exist_ok=True)
    if not ref.available():
        raise SystemExit("oracle/_ref/libfdref.so missing: run oracle/build_ref.sh")
    t0 = time.time()
    path = os.path.join(outdir, "reference_timings.json")
    meta = {}
    if os.path.exists(path):
        with open(path) as f:
            meta = json.load(f)
    fns = dict(c1=c1, small=small, flags=flags, c2timing=c2_timing, c2=c2, ss=ss, c2full=c2full, c4=c4)
    for p in parts:
        got = fns[p](outdir)
        if got:
            meta.update(got)
    meta["wall_s"] = time.time() - t0
    with open(path, "w") as f:
        json.dump(meta, f, indent=1)
    print(json.dumps(meta))


if __name__ == "__main__":
    main()
