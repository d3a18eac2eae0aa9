"""fd2_dose_compute_static: the CCCS entry point that allocates nothing.

It serves callers that may not allocate device memory while they run (all of
their device memory comes from a pool fixed at start-up, or belongs to another
runtime).  The test calls it through the C-ABI and compares it with
fd2_dose_compute on the same Terma/density inputs.  Two static calls run back
to back on different batches (8x8 maps on the general march, 16x16 maps on
the 16x16 march), so a direction table or status word left over from the first
call would show in the second.  The file name sorts last, so a run that stops
at its first failure has run every other test before this one.
"""
import ctypes as C

import numpy as np
import pytest

from fastdose_b200 import _lib, api
from plan_cases import c1_case, small_case

FD2_ERR_INVALID_ARGUMENT = -1
FD2_ERR_CAPACITY = -6
STATIC_DIR_BYTES = 256 * 1024


def _prepared(ctx, case, idx):
    ph = case["phantom"]
    spec = case.get("spectrum") or case["cfg"]["spectrum"]
    kern = case.get("kernel") or case["cfg"]["kernel"]
    dens, sp, kn = api.Density(ctx, ph.density, ph.volume), api.Spectrum(ctx, spec), api.Kernel(ctx, kern)
    batch = api.BEVBatch(case["beams"][idx])
    api.TermaComputeCollective(ctx, batch, case["fluence"], dens, sp)
    return batch, kn


def _static(lib, batch, kernel, status, stream):
    return lib.fd2_dose_compute_static(batch.P, len(batch.beams), C.c_void_p(batch.d_beams.data_ptr()),
                                       batch.ptrs("terma"), batch.ptrs("dens"), batch.ptrs("dose"), kernel.h,
                                       C.byref(status), stream)


@pytest.mark.gpu
def test_static_entry_matches_dose_compute(ctx):
    import torch

    lib = _lib.get()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    batches = [_prepared(ctx, small_case(), list(range(16))), _prepared(ctx, c1_case(), list(range(0, 100, 3)))]
    assert [b.shape2 for b, _ in batches] == [(8, 8), (16, 16)]

    expected = []
    for batch, kn in batches:
        batch.dose.zero_()
        api.DoseComputeCollective(ctx, batch, kn)
        torch.cuda.synchronize()
        expected.append(batch.dose.cpu().numpy())
        batch.dose.zero_()
    torch.cuda.synchronize()

    statuses = [C.c_int(12345), C.c_int(12345)]
    for (batch, kn), st in zip(batches, statuses):
        _lib.check(_static(lib, batch, kn, st, stream), "dose_compute_static")
    torch.cuda.synchronize()
    for (batch, _), st, ref in zip(batches, statuses, expected):
        assert st.value == 0
        got = batch.dose.cpu().numpy()
        assert np.abs(ref).max() > 0
        # same kernel, same summation order: equal bit for bit
        np.testing.assert_array_equal(got, ref)


@pytest.mark.gpu
def test_static_entry_rejects_oversize_batches(ctx):
    lib = _lib.get()
    batch, kn = _prepared(ctx, small_case(), [0, 1])
    n_cones = int(np.sum(kn.src.theta.astype(np.float64) <= np.pi / 2)) * kn.src.n_phi
    limit = STATIC_DIR_BYTES // (16 * n_cones)
    st = C.c_int(0)
    # rejected on the host before the descriptors are read, so the 2-beam
    # descriptor array is never read past its end
    rc = lib.fd2_dose_compute_static(batch.P, limit + 1, C.c_void_p(batch.d_beams.data_ptr()), batch.ptrs("terma"),
                                     batch.ptrs("dens"), batch.ptrs("dose"), kn.h, C.byref(st), None)
    assert rc == FD2_ERR_CAPACITY
    msg = lib.fd2_last_error().decode()
    assert "fixed scratch" in msg and f"at most {limit} beams" in msg
    rc = lib.fd2_dose_compute_static(0, 2, C.c_void_p(batch.d_beams.data_ptr()), batch.ptrs("terma"),
                                     batch.ptrs("dens"), batch.ptrs("dose"), kn.h, C.byref(st), None)
    assert rc == FD2_ERR_INVALID_ARGUMENT
