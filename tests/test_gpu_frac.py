"""Fractional occupations (l_frac_occ, DFPT_kernel/dfpt_module.f90:328-401) at
Gamma through the C ABI against the oracle, whose restatement matches the
sum over all states (tests/test_oracle.py).  Bars as in the other parity
tests: 1e-10 (FP64) and 1e-7 (mixed) relative 2-norm, identical ierr."""
import dataclasses

import numpy as np
import pytest

from oracle import west_oracle as O
from west_b200.system import SPECS, build_system, perturbations

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _gpu(s, dvg, tr2, precision="fp64", **kw):
    from west_b200.wstat import ResponseOperator
    op = ResponseOperator(s, verbose=False, **kw)
    op.set_precision(precision)
    dng = np.zeros_like(dvg, order="F")
    ierr = op.apply_operator(dvg.shape[1], dvg, dng, tr2, 1)
    op.close()
    return dng, ierr


@pytest.mark.parametrize("name,frac", [("tiny", (0.5,)), ("small", (0.8, 0.35)), ("c1", (0.9, 0.6, 0.25))])
def test_fractional_occupations(name, frac):
    s = build_system(dataclasses.replace(SPECS[name], frac_occ=frac), "cuda")
    assert O.nbnd_occ_full(s) == s.nbnd_occ - len(frac)
    dvg = perturbations(s, 3)
    ref, rerr = O.apply_operator(s, dvg, 1e-14, maxiter=400)
    got, ierr = _gpu(s, dvg, 1e-14, n_dfpt_maxiter=400)
    assert (ierr == rerr).all() and (ierr == 0).all()
    assert _rel(got, ref) < 1e-10, _rel(got, ref)
    got, ierr = _gpu(s, dvg, 1e-14, "mixed", n_dfpt_maxiter=400)
    assert (ierr == 0).all()
    assert _rel(got, ref) < 1e-7, _rel(got, ref)
    fixed, ferr = O.apply_operator(s, dvg, 0.0, maxiter=5)
    got, ierr = _gpu(s, dvg, 0.0, n_dfpt_maxiter=5)
    assert (ierr == ferr).all()
    assert _rel(got, fixed) < 1e-10
    # lite solver: the 1 / (e_i - e_j) of the correction amplifies the bra-ket
    # rounding (2.6e-12 at c1), so the FP64 bar rather than the integer case's 1e-12
    lite, _ = O.apply_operator(s, dvg, -1.0)
    got, _ = _gpu(s, dvg, -1.0)
    assert _rel(got, lite) < 1e-10


def test_fractional_degenerate_orbitals_rejected():
    """dfpt stops on degenerate orbitals with different occupations
    (dfpt_module.f90:387); the context creation reports it."""
    from west_b200.lib import WestB200Error
    from west_b200.wstat import ResponseOperator
    s = build_system(dataclasses.replace(SPECS["tiny"], frac_occ=(0.5,)), "cuda")
    s.et = s.et.copy()
    s.et[2] = s.et[1] + 1e-4
    with pytest.raises(WestB200Error, match="degenerate"):
        ResponseOperator(s, verbose=False)
