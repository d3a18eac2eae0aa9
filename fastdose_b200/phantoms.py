"""Seeded synthetic planning inputs: phantoms, spectra, CCCS kernels, beam lists.

These stand in for the reference's patient datasets (which are external to its
repository); every generator is deterministic in its seed.  Arrays follow the
reference layouts: density float32[z][y][x] (FastDoseLib/include/density.cuh:12),
masks uint8 of the same shape, angles in radians.
"""
import math
from dataclasses import dataclass, field

import numpy as np

from .types import make_volume


@dataclass
class Spectrum:
    """SPECTRUM_h after read_spectrum_file (fluence normalised to sum 1)."""
    energy: np.ndarray
    fluence: np.ndarray
    mu: np.ndarray
    mu_en: np.ndarray

    @property
    def n(self):
        return int(self.energy.size)


@dataclass
class CCCSKernel:
    """KERNEL_h after read_kernel_file: per zenith bin (theta_mid, A, a, B, b), phi list."""
    theta: np.ndarray
    A: np.ndarray
    a: np.ndarray
    B: np.ndarray
    b: np.ndarray
    phi: np.ndarray

    @property
    def n_theta(self):
        return int(self.theta.size)

    @property
    def n_phi(self):
        return int(self.phi.size)


@dataclass
class Phantom:
    density: np.ndarray            # float32 [z][y][x]
    volume: np.ndarray             # VOLUME_DTYPE record
    masks: dict = field(default_factory=dict)   # name -> uint8 [z][y][x]

    @property
    def dim(self):
        return tuple(int(v) for v in self.volume["dim"])

    @property
    def voxel(self):
        return tuple(float(v) for v in self.volume["voxel_size"])

    def centre(self):
        return tuple(d * v * 0.5 for d, v in zip(self.dim, self.voxel))


def _phi_angles(n_phi):
    # KERNEL_h::read_kernel_file, FastDoseLib/src/kernel.cu:44-49 (float arithmetic)
    interval = np.float32(2.0 * np.float32(math.pi) / n_phi)
    return np.array([np.float32((i + 0.5) * float(interval)) for i in range(n_phi)], np.float32)


def synthetic_spectrum(seed=1, n_bins=12, e_lo=0.2, e_hi=6.0, e0=2.0):
    """Log-spaced bins with a seeded decaying weight profile and a smooth
    power-law mass attenuation coefficient (cm^2/g)."""
    rng = np.random.default_rng(seed)
    e = np.geomspace(e_lo, e_hi, n_bins)
    w = np.exp(-e / e0) * rng.uniform(0.8, 1.2, n_bins)
    w = w / w.sum()
    mu = 0.0707 * e ** -0.47
    mu_en = 0.0310 * e ** -0.22
    return Spectrum(e.astype(np.float32), w.astype(np.float32), mu.astype(np.float32),
                    mu_en.astype(np.float32))


def synthetic_kernel(seed=2, n_theta=8, n_phi=6):
    """Zenith bins spanning [0, pi/2] (all forward), two-exponential parameters
    A, B in [0.1, 1], a in [1, 5] /cm, b in [0.1, 0.8] /cm."""
    rng = np.random.default_rng(seed)
    edges = np.linspace(0.0, np.float32(math.pi) / 2, n_theta + 1).astype(np.float32)
    theta = ((edges[:-1] + edges[1:]) / np.float32(2)).astype(np.float32)
    A = rng.uniform(0.1, 1.0, n_theta).astype(np.float32)
    a = rng.uniform(1.0, 5.0, n_theta).astype(np.float32)
    B = rng.uniform(0.1, 1.0, n_theta).astype(np.float32)
    b = rng.uniform(0.1, 0.8, n_theta).astype(np.float32)
    return CCCSKernel(theta, A, a, B, b, _phi_angles(n_phi))


def parse_spectrum_text(text):
    """SPECTRUM_h::read_spectrum_file semantics (FastDoseLib/src/spectrum.cu:14-60):
    rows 'E fluence mu mu_en label', fluence normalised to sum 1."""
    rows = [ln.split() for ln in text.splitlines() if ln.strip()]
    e = np.array([float(r[0]) for r in rows], np.float32)
    f = np.array([float(r[1]) for r in rows], np.float32)
    mu = np.array([float(r[2]) for r in rows], np.float32)
    mu_en = np.array([float(r[3]) for r in rows], np.float32)
    s = np.float32(0)
    for v in f:
        s = np.float32(s + v)
    return Spectrum(e, (f / s).astype(np.float32), mu, mu_en)


def parse_kernel_text(text, n_phi):
    """KERNEL_h::read_kernel_file semantics (FastDoseLib/src/kernel.cu:13-72): a
    header line, then rows 'theta_begin theta_end A a B b'; theta_mid is the mean."""
    lines = [ln for ln in text.splitlines() if ln.strip()]
    rows = [[float(v) for v in ln.split()] for ln in lines[1:]]
    tb = np.array([r[0] for r in rows], np.float32)
    te = np.array([r[1] for r in rows], np.float32)
    theta = ((tb + te) / np.float32(2)).astype(np.float32)
    col = lambda k: np.array([r[k] for r in rows], np.float32)
    return CCCSKernel(theta, col(2), col(3), col(4), col(5), _phi_angles(n_phi))


def slab_phantom(n=64, voxel=0.25, bone=(4.0, 2.0, 1.85), lung=(8.0, 3.0, 0.25)):
    """Water cube with a bone and a lung slab perpendicular to +y (the gantry-0
    beam axis; the source sits at -y).  (depth_cm, thickness_cm, density)."""
    d = np.ones((n, n, n), np.float32)
    yc = (np.arange(n) + 0.5) * voxel
    for depth, thick, rho in (bone, lung):
        sel = (yc >= depth) & (yc < depth + thick)
        d[:, sel, :] = rho
    return Phantom(d, make_volume((n, n, n), (voxel, voxel, voxel)))


def _grid(dim, voxel):
    nx, ny, nz = dim
    x = (np.arange(nx) + 0.5) * voxel
    y = (np.arange(ny) + 0.5) * voxel
    z = (np.arange(nz) + 0.5) * voxel
    return np.meshgrid(z, y, x, indexing="ij")  # Z, Y, X arrays of shape [z][y][x]


def torso_phantom(seed=3, dim=(200, 200, 160), voxel=0.25, ptv_radius=3.0,
                  ptv_offset=(3.0, 1.5, 0.0), noise=0.03):
    """Ellipsoidal body (density 1 + N(0, noise)), two lung ellipsoids at 0.25, a
    spine cylinder at 1.5, and a PTV sphere; air outside at 0.001."""
    rng = np.random.default_rng(seed)
    Z, Y, X = _grid(dim, voxel)
    cx, cy, cz = (dim[0] * voxel / 2, dim[1] * voxel / 2, dim[2] * voxel / 2)
    ax, ay, az = cx * 0.9, cy * 0.62, cz * 0.95
    body = ((X - cx) / ax) ** 2 + ((Y - cy) / ay) ** 2 + ((Z - cz) / az) ** 2 <= 1.0
    d = np.full(X.shape, 0.001, np.float32)
    d[body] = (1.0 + noise * rng.standard_normal(int(body.sum()))).astype(np.float32)
    for sx in (-1, 1):
        lung = (((X - (cx + sx * ax * 0.45)) / (ax * 0.3)) ** 2 + ((Y - (cy - ay * 0.1)) / (ay * 0.55)) ** 2
                + ((Z - cz) / (az * 0.6)) ** 2) <= 1.0
        d[lung & body] = 0.25
    spine = ((X - cx) ** 2 + (Y - (cy + ay * 0.7)) ** 2 <= (1.2) ** 2) & body
    d[spine] = 1.5
    pc = (cx + ptv_offset[0], cy + ptv_offset[1], cz + ptv_offset[2])
    ptv = ((X - pc[0]) ** 2 + (Y - pc[1]) ** 2 + (Z - pc[2]) ** 2) <= ptv_radius ** 2
    masks = {"PTV": ptv.astype(np.uint8), "BODY": body.astype(np.uint8)}
    bstart, bdim = _bbox(body)
    vol = make_volume(dim, (voxel,) * 3, bstart, bdim)
    return Phantom(d, vol, masks)


def head_neck_phantom(seed=4, dim=(256, 256, 200), voxel=0.25):
    """Skin ellipsoid, bone, air cavities at 0.001 and four PTV spheres of radius
    1.5-3 cm at separate isocentres."""
    rng = np.random.default_rng(seed)
    Z, Y, X = _grid(dim, voxel)
    cx, cy, cz = (dim[0] * voxel / 2, dim[1] * voxel / 2, dim[2] * voxel / 2)
    ax, ay, az = cx * 0.7, cy * 0.8, cz * 0.95
    skin = ((X - cx) / ax) ** 2 + ((Y - cy) / ay) ** 2 + ((Z - cz) / az) ** 2 <= 1.0
    d = np.full(X.shape, 0.001, np.float32)
    d[skin] = (1.0 + 0.03 * rng.standard_normal(int(skin.sum()))).astype(np.float32)
    bone = skin & ((X - cx) ** 2 + (Y - (cy + ay * 0.6)) ** 2 <= 1.5 ** 2)
    d[bone] = 1.8
    for k in range(3):
        c = (cx + rng.uniform(-0.3, 0.3) * ax, cy + rng.uniform(-0.5, 0.0) * ay, cz + rng.uniform(-0.4, 0.4) * az)
        r = rng.uniform(0.8, 1.5)
        cav = ((X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2 <= r * r) & skin
        d[cav] = 0.001
    masks = {"SKIN": skin.astype(np.uint8)}
    for k in range(4):
        c = (cx + rng.uniform(-0.4, 0.4) * ax, cy + rng.uniform(-0.3, 0.3) * ay, cz + (k - 1.5) * az * 0.35)
        r = rng.uniform(1.5, 3.0)
        masks[f"PTVSeg{k}"] = (((X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2 <= r * r) & skin).astype(np.uint8)
    bstart, bdim = _bbox(skin)
    return Phantom(d, make_volume(dim, (voxel,) * 3, bstart, bdim), masks)


def _bbox(mask):
    """getBBox semantics: start and size (x, y, z) of the mask's bounding box."""
    idx = np.nonzero(mask)
    zs, ys, xs = (int(i.min()) for i in idx)
    ze, ye, xe = (int(i.max()) + 1 for i in idx)
    return (xs, ys, zs), (xe - xs, ye - ys, ze - zs)


def mask_centroid(mask, voxel):
    """PTV centroid in cm (IMRT::BeamBundleInit, IMRTOpt/src/IMRTBeamBundle.cu:36-61)."""
    idx = np.nonzero(mask)
    zs, ys, xs = (i.astype(np.float64) + 0.5 for i in idx)
    n = xs.size
    return (xs.sum() / n * voxel[0], ys.sum() / n * voxel[1], zs.sum() / n * voxel[2])


def sphere_beam_angles(n_target=400, min_axis_sep_deg=35.0, seed=0):
    """4pi candidate beams: directions on a sphere by the latitude-ring scheme of
    the reference's angle generator (dockerScripts/HeadNeck/scripts.py:21-44),
    converted to (gantry, couch) (scripts.py:47-61), pruned by a couch/gantry
    clearance rule that rejects directions within `min_axis_sep_deg` of the
    patient's long axis.  Returns float32 [n, 3] (gantry, couch, coll) radians."""
    res = math.radians(6.0)
    out = []
    for _ in range(40):
        dirs = []
        n_th = round(math.pi / res)
        for it in range(n_th + 1):
            th = it * res
            n_ph = max(1, int(math.ceil(2 * math.pi * math.sin(th) / res)))
            for ip in range(n_ph):
                ph = ip * 2 * math.pi / n_ph
                dirs.append((math.sin(th) * math.cos(ph), math.sin(th) * math.sin(ph), math.cos(th)))
        keep = [d for d in dirs if abs(d[2]) < math.cos(math.radians(min_axis_sep_deg))]
        if len(keep) >= n_target:
            out = keep
            break
        res *= 0.97
    out = out[:: max(1, len(out) // n_target)][:n_target]
    angles = []
    for d in out:
        cg = d[1]
        sg = math.sqrt(max(0.0, 1 - cg * cg))
        gantry = math.acos(max(-1.0, min(1.0, cg)))
        if sg < 1e-4:
            mc = 0.0
        else:
            smc = d[2] / sg
            cmc = max(-1.0, min(1.0, -d[0] / sg))
            mc = math.acos(cmc)
            if smc < 0:
                mc = -mc
        angles.append((gantry, -mc, 0.0))
    return np.array(angles, np.float32)


def config1():
    """Plain CCCS, single beam: 64^3 slab phantom, gantry 0, SAD 100, iso at
    the centre, 10x10 open 0.5 cm beamlets (16x16 sub-maps, 4x4 open)."""
    ph = slab_phantom()
    return dict(phantom=ph, spectrum=synthetic_spectrum(), kernel=synthetic_kernel(),
                isocenter=ph.centre(), angles=np.zeros((1, 3), np.float32), fluence_dim=10,
                beamlet_size=0.5, sad=100.0, sub_fluence_dim=16, sub_fluence_on=4,
                long_spacing=0.25, extent=2.0)


def config4(n_per_iso=300, dim=(256, 256, 200), seed=4, sub_fluence_dims=(12, 16, 20, 16)):
    """Multi-isocentre head-and-neck plan: the head_neck_phantom's four PTV
    segments, each with its own isocentre and n_per_iso candidate beams from
    the 4pi sphere; per beam a fluence map of 6..20 beamlets a side (PTV
    masking leaves 20-400 per beam); per isocentre its own BEV grid (sub-beam
    map of sub_fluence_dims[k] pixels a side), so the plan is built as one
    dose-loading matrix per isocentre."""
    ph = head_neck_phantom(seed=seed, dim=dim)
    rng = np.random.default_rng(seed + 100)
    angles = sphere_beam_angles(n_per_iso)
    isos = []
    for k in range(4):
        mask = ph.masks[f"PTVSeg{k}"]
        # each isocentre sees the sphere from its own rotation of the couch axis
        shift = rng.uniform(0.0, 2.0 * math.pi)
        a = angles.copy()
        a[:, 1] = ((a[:, 1] + shift + math.pi) % (2.0 * math.pi) - math.pi).astype(np.float32)
        isos.append(dict(mask=mask, isocenter=mask_centroid(mask, ph.voxel), angles=a,
                         fluence_dims=rng.integers(6, 21, size=len(a)), sub_fluence_dim=int(sub_fluence_dims[k])))
    return dict(phantom=ph, spectrum=synthetic_spectrum(), kernel=synthetic_kernel(), isos=isos, beamlet_size=0.5,
                sad=100.0, sub_fluence_on=4, long_spacing=0.25, extent=2.0)


def config2(n_beams=400):
    """Batched 4pi CCCS: 200x200x160 torso, up to 400 candidate beams,
    16x16 beamlet grid of 0.5 cm, beamlets kept where they see the PTV."""
    ph = torso_phantom()
    iso = mask_centroid(ph.masks["PTV"], ph.voxel)
    return dict(phantom=ph, spectrum=synthetic_spectrum(), kernel=synthetic_kernel(),
                isocenter=iso, angles=sphere_beam_angles(n_beams), fluence_dim=16,
                beamlet_size=0.5, sad=100.0, sub_fluence_dim=16, sub_fluence_on=4,
                long_spacing=0.25, extent=2.0)
