"""numpy views of the POD structs declared in include/fd2.h.

The beam record is byte-compatible with the reference's ``fastdose::d_BEAM_d``
(FastDoseLib/include/beam.cuh:84-133); the volume and bundle records carry the
fields of ``DENSITY_h`` (FastDoseLib/include/density.cuh:9-27) and
``IMRT::BeamBundle`` (IMRTOpt/include/IMRTBeamBundle.cuh:9-31).
"""
import numpy as np

BEAM_DTYPE = np.dtype(
    [
        ("isocenter", "<f4", (3,)),
        ("pad0", "<u4"),
        ("beamlet_size", "<f4", (2,)),
        ("fmap_size", "<u4", (2,)),
        ("sad", "<f4"),
        ("angles", "<f4", (3,)),
        ("long_spacing", "<f4"),
        ("lim_min", "<f4"),
        ("lim_max", "<f4"),
        ("long_dim", "<u4"),
        ("source", "<f4", (3,)),
        ("pad1", "<u4"),
        ("TermaBEV_pitch", "<u8"),
        ("DensityBEV_pitch", "<u8"),
    ]
)
assert BEAM_DTYPE.itemsize == 96

VOLUME_DTYPE = np.dtype(
    [
        ("dim", "<u4", (3,)),
        ("voxel_size", "<f4", (3,)),
        ("bbox_start", "<u4", (3,)),
        ("bbox_dim", "<u4", (3,)),
    ]
)
assert VOLUME_DTYPE.itemsize == 48

BUNDLE_DTYPE = np.dtype(
    [
        ("isocenter", "<f4", (3,)),
        ("beamlet_size", "<f4", (2,)),
        ("fluence_dim", "<i4", (2,)),
        ("sad", "<f4"),
        ("angles", "<f4", (3,)),
        ("long_spacing", "<f4"),
        ("sub_fluence_dim", "<i4", (2,)),
        ("sub_fluence_on", "<i4", (2,)),
    ]
)
assert BUNDLE_DTYPE.itemsize == 64


def make_volume(dim, voxel_size, bbox_start=(0, 0, 0), bbox_dim=None):
    """One VOLUME_DTYPE record; dim and voxel_size are (x, y, z)."""
    v = np.zeros((), VOLUME_DTYPE)
    v["dim"] = dim
    v["voxel_size"] = voxel_size
    v["bbox_start"] = bbox_start
    v["bbox_dim"] = dim if bbox_dim is None else bbox_dim
    return v


def make_bundle(isocenter, angles, sad=100.0, fluence_dim=20, beamlet_size=0.5,
                sub_fluence_dim=16, sub_fluence_on=4, long_spacing=0.25):
    """One BUNDLE_DTYPE record with the reference's argument defaults
    (IMRTOpt/src/IMRTArgs.cpp:47-62)."""
    b = np.zeros((), BUNDLE_DTYPE)
    b["isocenter"] = isocenter
    b["beamlet_size"] = (beamlet_size, beamlet_size)
    b["fluence_dim"] = (fluence_dim, fluence_dim)
    b["sad"] = sad
    b["angles"] = angles
    b["long_spacing"] = long_spacing
    b["sub_fluence_dim"] = (sub_fluence_dim, sub_fluence_dim)
    b["sub_fluence_on"] = (sub_fluence_on, sub_fluence_on)
    return b
