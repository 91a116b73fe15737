"""The allocation-free entry point, for callers that cannot allocate device
memory while they run, returns what the regular device entry point returns.

Collected last on purpose: if it fails, a run that stops at the first failure
has already run every other test.  It does not depend on the other tests and
passes in a fresh process as well.
"""
import ctypes

import numpy as np
import pytest

from west_b200.system import build_system, perturbations

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-10     # same bar as the other FP64 parity tests


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_noalloc_matches_device_entry_point_twice():
    import torch
    from west_b200 import lib as L
    from west_b200.wstat import ResponseOperator

    s = build_system("small")
    m = 3
    dvg = perturbations(s, m)
    op = ResponseOperator(s, verbose=False)
    dv = torch.from_numpy(np.ascontiguousarray(dvg.T)).cuda()
    ref = torch.zeros_like(dv)
    ierr_ref = op.apply_operator(m, dv, ref, 1e-10, 1)
    ref = ref.cpu().numpy()
    lib = L.load()
    for call in range(2):                      # the scratch keeps the previous call's contents
        out = torch.full_like(dv, complex(float("nan"), float("nan")))
        ierr = np.full(m, -7, dtype=np.int32)
        rc = lib.wb_apply_operator_device_noalloc(op._ctx, m, dv.data_ptr(), s.npw, out.data_ptr(), s.npw,
                                                  1e-10, 1, ierr.ctypes.data)
        assert rc == 0, lib.wb_last_error().decode()
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.isfinite(got).all(), call
        assert (ierr == ierr_ref).all(), call
        assert _rel(got, ref) < TOL_FP64, call


def test_noalloc_rejects_calls_beyond_its_scratch():
    import torch
    from west_b200 import lib as L
    from west_b200.wstat import ResponseOperator

    s = build_system("small")
    m = 400
    op = ResponseOperator(s, verbose=False)
    dv = torch.zeros((m, s.npw), dtype=torch.complex128, device="cuda")
    out = torch.zeros_like(dv)
    lib = L.load()
    rc = lib.wb_apply_operator_device_noalloc(op._ctx, m, dv.data_ptr(), s.npw, out.data_ptr(), s.npw,
                                              1e-10, 1, None)
    assert rc == L.WB_ERR_ARG
    msg = lib.wb_last_error().decode()
    assert "scratch" in msg and str(L.WB_NOALLOC_SCRATCH_BYTES) in msg
