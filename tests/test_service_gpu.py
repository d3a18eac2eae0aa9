"""Served dose calculation: requests through the service give the same
matrices as direct constructions, in any completion order, with consistent
timing; requests beyond the HBM budget are refused at submission."""
import numpy as np
import pytest

from fastdose_b200 import _lib, api, service
from plan_cases import c1_case, small_case

pytestmark = pytest.mark.gpu


def _direct(ctx, case):
    ph = case["phantom"]
    spec = case.get("spectrum") or case["cfg"]["spectrum"]
    kern = case.get("kernel") or case["cfg"]["kernel"]
    m = api.DoseMatConstruction(ctx, [case["beams"]], case["fluence"], api.Density(ctx, ph.density, ph.volume),
                                api.Spectrum(ctx, spec), api.Kernel(ctx, kern))
    out = m.to_host()
    m.close()
    return out


def _submit(svc, case):
    spec = case.get("spectrum") or case["cfg"]["spectrum"]
    kern = case.get("kernel") or case["cfg"]["kernel"]
    return svc.submit(case["phantom"], [case["beams"]], case["fluence"], spec, kern)


def test_service_matches_direct_construction(ctx):
    cases = [small_case(seed=5), c1_case(), small_case(seed=7, gantry=1.2, couch=-0.4), small_case(seed=9)]
    expected = [_direct(ctx, c) for c in cases]
    svc = service.Service(device=0, workers=2)
    try:
        tickets = [_submit(svc, c) for c in cases]
        for t, exp, c in zip(reversed(tickets), reversed(expected), reversed(cases)):
            m, st = svc.wait(t)
            got = m.to_host()
            m.close()
            for a, b in zip(got, exp):
                np.testing.assert_array_equal(a, b)
            assert st["status"] == 0 and st["beamlets"] == len(c["beams"]) and st["nnz"] == len(exp[1])
            assert st["submit_ms"] <= st["start_ms"] <= st["end_ms"] <= svc.clock_ms()
            assert st["worker"] in (0, 1) and st["est_bytes"] > 0
    finally:
        svc.close()


def test_service_refuses_requests_over_budget(ctx):
    svc = service.Service(device=0, workers=1, hbm_budget=1 << 20)
    try:
        with pytest.raises(_lib.FD2Error) as e:
            _submit(svc, small_case())
        assert e.value.status == -9  # FD2_ERR_ADMISSION
        assert "budget" in str(e.value)
    finally:
        svc.close()
