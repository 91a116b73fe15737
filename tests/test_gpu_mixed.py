"""Mixed form (FP32 PCG corrections inside FP64 iterative refinement) against
the FP64 oracle.  Bar: dng within 1e-7 relative (2-norm over the batch), every
system converged on the FP64 residual test, PDEP eigenvalues within 1e-6."""
import numpy as np
import pytest

from oracle import west_oracle as O
from west_b200.system import build_system, perturbations, randomized_basis

pytestmark = pytest.mark.gpu

TOL_MIXED = 1e-7


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _op(s, **kw):
    from west_b200.wstat import ResponseOperator
    op = ResponseOperator(s, verbose=False, **kw)
    op.set_precision("mixed")
    return op


@pytest.mark.parametrize("name", ["tiny", "small", "c1"])
def test_mixed_matches_fp64_oracle(name):
    s = build_system(name)
    dvg = perturbations(s, 4)
    ref, _ = O.apply_operator(s, dvg, 1e-10)
    op = _op(s)
    dng = np.zeros_like(dvg, order="F")
    ierr = op.apply_operator(4, dvg, dng, 1e-10, 1)
    st = op.stats()
    assert (ierr == 0).all()
    assert st["refinements"] >= 1
    assert _rel(dng, ref) < TOL_MIXED


def test_mixed_lite_solver_is_fp64(small):
    """tr2 < 0 runs no PCG, so the mixed form returns the FP64 result."""
    s = small
    dvg = perturbations(s, 3)
    ref, _ = O.apply_operator(s, dvg, -1.0)
    dng = np.zeros_like(dvg, order="F")
    _op(s).apply_operator(3, dvg, dng, -1.0, 1)
    assert _rel(dng, ref) < 1e-12


def test_mixed_kinetic_only(tiny):
    s = tiny
    dvg = perturbations(s, 2)
    ref, _ = O.apply_operator(s, dvg, 1e-12, kinetic_only=True, maxiter=400)
    dng = np.zeros_like(dvg, order="F")
    ierr = _op(s, l_kinetic_only=True, n_dfpt_maxiter=400).apply_operator(2, dvg, dng, 1e-12, 1)
    assert (ierr == 0).all()
    assert _rel(dng, ref) < TOL_MIXED


def test_mixed_davidson_eigenvalues(small):
    s = small
    dvg0 = randomized_basis(s, 4)
    rev, rconv, _, _ = O.davidson_diago_gamma(s, dvg0, 4, 16, tr2_dfpt=1e-12, trev_pdep=1e-6)
    ev, conv, _, info = _op(s).davidson(dvg0, 4, n_pdep_times=4, tr2_dfpt=1e-12, trev_pdep=1e-6)
    assert info["converged"] == 1 and rconv.all()
    assert np.abs((ev - rev) / rev).max() < 1e-6
