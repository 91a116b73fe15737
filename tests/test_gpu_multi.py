"""Several ground states of uneven size in one call (wb_apply_operator_multi):
each system's result equals its own apply_operator call and the oracle."""
import numpy as np
import pytest

from oracle import west_oracle as O
from west_b200.system import build_system, perturbations

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_multi_system_call(tiny, small, precision):
    from west_b200.wstat import ResponseOperator, apply_operator_multi
    systems = [tiny, small, build_system("c1")]
    ms = [2, 5, 3]
    ops, dvgs, dngs = [], [], []
    for s, m in zip(systems, ms):
        op = ResponseOperator(s, verbose=False)
        op.set_precision(precision)
        ops.append(op)
        dvgs.append(perturbations(s, m))
        dngs.append(np.zeros((s.npw, m), dtype=np.complex128, order="F"))
    # a tight threshold: at a loose one a system whose residual sits on tr2 may stop
    # one iteration apart in the oracle, which compares the threshold, not the path
    tr2 = 1e-16
    ierrs = apply_operator_multi(ops, dvgs, dngs, tr2)
    for op, dvg, dng, ierr, s in zip(ops, dvgs, dngs, ierrs, systems):
        assert (ierr == 0).all()
        single = np.zeros_like(dng)
        op.apply_operator(dvg.shape[1], dvg, single, tr2, 1)
        tol = 1e-12 if precision == "fp64" else 1e-8
        assert _rel(dng, single) < tol
    for s, dvg, dng in zip(systems[:2], dvgs[:2], dngs[:2]):
        ref, _ = O.apply_operator(s, dvg, tr2)
        assert _rel(dng, ref) < (1e-10 if precision == "fp64" else 1e-7)


def test_multi_device_pointers(tiny, small):
    import torch
    from west_b200.wstat import ResponseOperator, apply_operator_multi
    ops, dvgs, dngs, hosts = [], [], [], []
    for s, m in ((tiny, 3), (small, 2)):
        ops.append(ResponseOperator(s, verbose=False))
        h = perturbations(s, m)
        hosts.append(h)
        dvgs.append(torch.from_numpy(np.ascontiguousarray(h.T)).cuda())
        dngs.append(torch.zeros_like(dvgs[-1]))
    apply_operator_multi(ops, dvgs, dngs, 1e-10)
    for op, h, d in zip(ops, hosts, dngs):
        single = np.zeros_like(h, order="F")
        op.apply_operator(h.shape[1], h, single, 1e-10, 1)
        assert _rel(d.cpu().numpy().T, single) < 1e-12


def test_multi_rejects_duplicate_context(tiny):
    from west_b200.lib import WestB200Error
    from west_b200.wstat import ResponseOperator, apply_operator_multi
    op = ResponseOperator(tiny, verbose=False)
    d = perturbations(tiny, 1)
    with pytest.raises(WestB200Error):
        apply_operator_multi([op, op], [d, d], [np.zeros_like(d, order="F"), np.zeros_like(d, order="F")], 1e-10)
