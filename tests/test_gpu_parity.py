"""Parity of the CUDA apply_operator (through the C ABI) with the CPU oracle.

Tolerance: dng agrees with the oracle to 1e-10 in relative 2-norm over the
whole batch, ||dng - ref|| / ||ref||, in the FP64 form (1e-12 for the lite
solver, which runs no PCG).  For scale: the oracle's own output moves by up to
~1e-10 (max-norm) when its input is perturbed by one ulp on the fixed-iteration
cases, so the PCG's conditioning, not the kernels, sets this floor.
"""
import os

import numpy as np
import pytest

from oracle import west_oracle as O
from west_b200.system import build_system, perturbations

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL_FP64 = 1e-10


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _op(s, **kw):
    from west_b200.wstat import ResponseOperator
    return ResponseOperator(s, verbose=False, **kw)


def _gpu_apply(op, dvg, tr2, m=None, ld=None):
    m = dvg.shape[1] if m is None else m
    ld = dvg.shape[0] if ld is None else ld
    dng = np.zeros((ld, m), dtype=np.complex128, order="F")
    din = np.zeros((ld, m), dtype=np.complex128, order="F")
    din[: dvg.shape[0]] = dvg[:, :m]
    ierr = op.apply_operator(m, din, dng, tr2, 1)
    return dng, ierr


@pytest.mark.parametrize("name", ["tiny", "small"])
def test_lite_solver_parity(name):
    s = build_system(name)
    dvg = perturbations(s, 4)
    ref, _ = O.apply_operator(s, dvg, -1.0)
    got, ierr = _gpu_apply(_op(s), dvg, -1.0)
    assert (ierr == 0).all()
    assert _rel(got, ref) < 1e-12


@pytest.mark.parametrize("name,steps", [("tiny", 5), ("small", 8)])
def test_fixed_iteration_parity(name, steps):
    """tr2 = 0: no system converges, both sides run exactly n_dfpt_maxiter steps
    (step counts where the PCG iterate is well conditioned)."""
    s = build_system(name)
    dvg = perturbations(s, 3)
    ref, rerr = O.apply_operator(s, dvg, 0.0, maxiter=steps)
    got, ierr = _gpu_apply(_op(s, n_dfpt_maxiter=steps), dvg, 0.0)
    assert (ierr == rerr).all() and (ierr == s.nbnd_occ).all()
    assert _rel(got, ref) < TOL_FP64


@pytest.mark.parametrize("name", ["tiny", "small"])
def test_converged_parity(name):
    s = build_system(name)
    dvg = perturbations(s, 5)
    ref, rerr = O.apply_operator(s, dvg, 1e-22, maxiter=400)
    got, ierr = _gpu_apply(_op(s, n_dfpt_maxiter=400), dvg, 1e-22)
    assert (ierr == 0).all() and (rerr == 0).all()
    assert _rel(got, ref) < TOL_FP64


def test_production_threshold_parity(small):
    s = small
    dvg = perturbations(s, 4, seed=99)
    ref, rerr = O.apply_operator(s, dvg, 1e-10)
    got, ierr = _gpu_apply(_op(s), dvg, 1e-10)
    assert (ierr == rerr).all()
    assert _rel(got, ref) < TOL_FP64


def test_golden_fixture(tiny):
    g = np.load(os.path.join(GOLDEN, "oracle_tiny.npz"))
    s = build_system("tiny")
    s.evc = g["evc"]; s.et = g["et"]
    for tag, tr2, maxit in (("lite", -1.0, 250), ("tr2_1e-12", 1e-12, 250), ("fixed5", 0.0, 5)):
        got, ierr = _gpu_apply(_op(s, n_dfpt_maxiter=maxit), g["dvg"], tr2)
        assert _rel(got, g["dng_" + tag]) < TOL_FP64, tag
        assert (ierr == g["ierr_" + tag]).all(), tag


def test_kinetic_only_parity(tiny):
    s = tiny
    dvg = perturbations(s, 2)
    ref, rerr = O.apply_operator(s, dvg, 0.0, maxiter=6, kinetic_only=True)
    got, ierr = _gpu_apply(_op(s, n_dfpt_maxiter=6, l_kinetic_only=True), dvg, 0.0)
    assert (ierr == rerr).all()
    assert _rel(got, ref) < TOL_FP64


@pytest.mark.parametrize("m", [0, 1, 3])
def test_small_batches(small, m):
    s = small
    dvg = perturbations(s, max(m, 1))
    op = _op(s)
    if m == 0:
        dng = np.zeros((s.npw, 1), dtype=np.complex128, order="F")
        ierr = op.apply_operator(0, dvg, dng, 1e-10, 1)
        assert ierr.size == 0 and not dng.any()
        return
    ref, _ = O.apply_operator(s, dvg[:, :m], 1e-14)
    got, _ = _gpu_apply(op, dvg, 1e-14, m=m)
    assert _rel(got, ref) < TOL_FP64


def test_chunking_invariance(small):
    """Splitting the perturbations into device batches changes only FFT pairing."""
    s = small
    dvg = perturbations(s, 5)
    op = _op(s)
    a, ea = _gpu_apply(op, dvg, 1e-14)
    op.set_batch(2)
    b, eb = _gpu_apply(op, dvg, 1e-14)
    assert (ea == eb).all()
    assert _rel(b, a) < 1e-12


def test_leading_dimension_padding(tiny):
    s = tiny
    dvg = perturbations(s, 2)
    ref, _ = O.apply_operator(s, dvg, 1e-14)
    got, _ = _gpu_apply(_op(s), dvg, 1e-14, ld=s.npw + 7)
    assert _rel(got[: s.npw], ref) < TOL_FP64
    assert not got[s.npw:].any()


def test_device_pointer_path_matches_host(small):
    import torch
    s = small
    dvg = perturbations(s, 3)
    op = _op(s)
    h, eh = _gpu_apply(op, dvg, 1e-12)
    dv = torch.from_numpy(np.ascontiguousarray(dvg.T)).cuda()
    dn = torch.zeros_like(dv)
    ed = op.apply_operator(3, dv, dn, 1e-12, 1)
    assert (ed == eh).all()
    assert np.array_equal(dn.cpu().numpy().T, h)


def test_errors_raise(tiny):
    from west_b200.lib import WestB200Error
    s = tiny
    op = _op(s)
    dvg = perturbations(s, 1)
    dng = np.zeros_like(dvg)
    with pytest.raises(WestB200Error, match="iq"):
        op.apply_operator(1, dvg, dng, 1e-10, 2)
    with pytest.raises(WestB200Error, match="NaN"):
        op.apply_operator(1, dvg, dng, float("nan"), 1)


def test_unconverged_reported(small):
    s = small
    dvg = perturbations(s, 2)
    _, ierr = _gpu_apply(_op(s, n_dfpt_maxiter=2), dvg, 1e-10)
    _, rerr = O.apply_operator(s, dvg, 1e-10, maxiter=2)
    assert (ierr == rerr).all() and (ierr > 0).all()


def test_c1_parity():
    """The 48^3 workload (L=15 bohr, 20 Ry, 8 bands), two perturbations, tr2 = 1e-10."""
    s = build_system("c1")
    dvg = perturbations(s, 2)
    ref, rerr = O.apply_operator(s, dvg, 1e-10)
    got, ierr = _gpu_apply(_op(s), dvg, 1e-10)
    assert (ierr == rerr).all()
    assert _rel(got, ref) < TOL_FP64
