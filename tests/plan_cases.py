"""Shared synthetic planning cases for the tests (seeded, deterministic)."""
import numpy as np

from fastdose_b200 import api, phantoms
from fastdose_b200.types import make_bundle, make_volume


def c1_case():
    """Config 1: 64^3 slab phantom, one gantry-0 beam, 10x10 beamlets."""
    cfg = phantoms.config1()
    ph = cfg["phantom"]
    bund = make_bundle(cfg["isocenter"], cfg["angles"][0], sad=cfg["sad"], fluence_dim=cfg["fluence_dim"],
                       beamlet_size=cfg["beamlet_size"], sub_fluence_dim=cfg["sub_fluence_dim"],
                       sub_fluence_on=cfg["sub_fluence_on"], long_spacing=cfg["long_spacing"])
    beams = api.bundle_beamlets(bund, np.ones(100, np.uint8), ph.volume)
    return dict(cfg=cfg, phantom=ph, bundle=bund, beams=beams, fluence=api.beamlet_fluence(bund))


def small_case(seed=5, n=32, gantry=0.6, couch=0.3):
    """A small oblique case: n^3 heterogeneous phantom, one 4x4 bundle with
    8x8 sub-maps (fast enough for the double-precision oracle)."""
    rng = np.random.default_rng(seed)
    vox = 0.25
    d = (1.0 + 0.2 * rng.standard_normal((n, n, n))).clip(0.05, 2.5).astype(np.float32)
    d[:, : n // 4, :] = 0.3
    vol = make_volume((n, n, n), (vox, vox, vox))
    ph = phantoms.Phantom(d, vol)
    iso = ph.centre()
    bund = make_bundle(iso, (gantry, couch, 0.1), sad=100.0, fluence_dim=4, beamlet_size=0.4, sub_fluence_dim=8,
                       sub_fluence_on=2, long_spacing=0.25)
    beams = api.bundle_beamlets(bund, np.ones(16, np.uint8), vol)
    spec = phantoms.synthetic_spectrum(seed=11, n_bins=6)
    kern = phantoms.synthetic_kernel(seed=12, n_theta=4, n_phi=4)
    return dict(phantom=ph, bundle=bund, beams=beams, fluence=api.beamlet_fluence(bund), spectrum=spec,
                kernel=kern)
