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


def _noalloc(op, m, dv, ld, tr2):
    import torch
    from west_b200 import lib as L
    lib = L.load()
    out = torch.full((m, ld), complex(float("nan"), float("nan")), dtype=torch.complex128, device="cuda")
    ierr = np.full(m, -7, dtype=np.int32)
    rc = lib.wb_apply_operator_device_noalloc(op._ctx, m, dv.data_ptr(), ld, out.data_ptr(), ld, tr2, 1,
                                              ierr.ctypes.data)
    assert rc == 0, lib.wb_last_error().decode()
    torch.cuda.synchronize()
    return out.cpu().numpy(), ierr


def _device(op, m, dv, tr2):
    import torch
    ref = torch.zeros((m, dv.shape[1]), dtype=torch.complex128, device="cuda")
    ierr = op.apply_operator(m, dv[:m].contiguous(), ref, tr2, 1)
    return ref.cpu().numpy(), ierr


def test_noalloc_smaller_call_after_a_larger_one():
    """m = 5 then m = 2 on one context: the second call's pieces of the shared
    array start at other offsets over the first call's leftovers."""
    import torch
    from west_b200.wstat import ResponseOperator

    s = build_system("small")
    dvg = perturbations(s, 5, seed=5)
    op = ResponseOperator(s, verbose=False)
    dv = torch.from_numpy(np.ascontiguousarray(dvg.T)).cuda()
    for m in (5, 2):
        ref, eref = _device(op, m, dv, 1e-10)
        got, ierr = _noalloc(op, m, dv[:m].contiguous(), s.npw, 1e-10)
        assert (ierr == eref).all(), m
        assert _rel(got, ref) < TOL_FP64, m


def test_noalloc_two_contexts_in_turn():
    """Two contexts of different systems share the one array, called one after the other."""
    import torch
    from west_b200.wstat import ResponseOperator

    cases = []
    for name, m in (("tiny", 3), ("small", 2)):
        s = build_system(name)
        dv = torch.from_numpy(np.ascontiguousarray(perturbations(s, m).T)).cuda()
        op = ResponseOperator(s, verbose=False)
        cases.append((s, op, m, dv, _device(op, m, dv, 1e-12)))
    for rnd in range(2):
        for s, op, m, dv, (ref, eref) in cases:
            got, ierr = _noalloc(op, m, dv, s.npw, 1e-12)
            assert (ierr == eref).all(), (s.nr, rnd)
            assert _rel(got, ref) < TOL_FP64, (s.nr, rnd)


def test_noalloc_kinetic_only():
    import torch
    from west_b200.wstat import ResponseOperator

    s = build_system("tiny")
    dv = torch.from_numpy(np.ascontiguousarray(perturbations(s, 2).T)).cuda()
    op = ResponseOperator(s, verbose=False, n_dfpt_maxiter=6, l_kinetic_only=True)
    ref, eref = _device(op, 2, dv, 0.0)
    got, ierr = _noalloc(op, 2, dv, s.npw, 0.0)
    assert (ierr == eref).all()
    assert _rel(got, ref) < TOL_FP64


def test_noalloc_rejects_the_mixed_form():
    import torch
    from west_b200 import lib as L
    from west_b200.wstat import ResponseOperator

    s = build_system("tiny")
    op = ResponseOperator(s, verbose=False)
    op.set_precision("mixed")
    dv = torch.zeros((1, s.npw), dtype=torch.complex128, device="cuda")
    out = torch.zeros_like(dv)
    lib = L.load()
    rc = lib.wb_apply_operator_device_noalloc(op._ctx, 1, dv.data_ptr(), s.npw, out.data_ptr(), s.npw, 1e-10, 1,
                                              None)
    assert rc == L.WB_ERR_UNSUPPORTED
    assert "FP64" in lib.wb_last_error().decode()
