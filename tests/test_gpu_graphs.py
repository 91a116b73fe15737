"""The graph-captured PCG loops (one CUDA graph launch per batch, convergence
tested on the device by a conditional WHILE node) against the eager loops
(host readback of the active count every iteration) and the FP64 oracle.

The two paths run the same kernels; the graph path sizes grids for the
workspace capacity and strides over the active systems, and its split-K
GEMMs may use a different split count, so FP64 results agree to rounding
(1e-12) and the iteration counts agree exactly."""
import numpy as np
import pytest

from oracle import west_oracle as O
from west_b200.system import perturbations

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _run(op, dvg, tr2, m=None):
    m = dvg.shape[1] if m is None else m
    dng = np.zeros((dvg.shape[0], m), dtype=np.complex128, order="F")
    ierr = op.apply_operator(m, dvg, dng, tr2, 1)
    return dng, ierr, op.stats()


def _op(s, **kw):
    from west_b200.wstat import ResponseOperator
    return ResponseOperator(s, verbose=False, **kw)


@pytest.mark.parametrize("tr2", [1e-10, 1e-20])
def test_graph_matches_eager_fp64(small, tr2):
    """tr2 = 1e-20 runs into n_dfpt_maxiter, so the device loop bound is exercised."""
    s = small
    dvg = perturbations(s, 5)
    op_g = _op(s, n_dfpt_maxiter=40)
    op_e = _op(s, n_dfpt_maxiter=40)
    op_e.set_graphs(False)
    for op in (op_g, op_e):  # the same launch shapes (split counts) in both contexts
        op.set_autotune(False)
    dg, eg, sg = _run(op_g, dvg, tr2)
    de, ee, se = _run(op_e, dvg, tr2)
    assert sg["cg_iterations"] == se["cg_iterations"]
    assert sg["cg_active_sum"] == se["cg_active_sum"]
    assert (eg == ee).all()
    assert _rel(dg, de) < 1e-12
    if tr2 == 1e-10:
        ref, _ = O.apply_operator(s, dvg, tr2)
        assert _rel(dg, ref) < 1e-10


def test_graph_reused_across_batch_sizes(small):
    """A batch smaller than the captured capacity reuses the graph (device
    batch size) and still matches the oracle."""
    s = small
    op = _op(s)
    dvg = perturbations(s, 6)
    _run(op, dvg, 1e-10)
    small_dvg = np.asfortranarray(dvg[:, :3])
    dng, ierr, _ = _run(op, small_dvg, 1e-10)
    ref, _ = O.apply_operator(s, small_dvg, 1e-10)
    assert (ierr == 0).all()
    assert _rel(dng, ref) < 1e-10


def test_graph_matches_eager_mixed(small):
    s = small
    dvg = perturbations(s, 4)
    op_g = _op(s)
    op_e = _op(s)
    for op in (op_g, op_e):
        op.set_precision("mixed")
    op_e.set_graphs(False)
    dg, eg, sg = _run(op_g, dvg, 1e-10)
    de, ee, se = _run(op_e, dvg, 1e-10)
    ref, _ = O.apply_operator(s, dvg, 1e-10)
    assert (eg == 0).all() and (ee == 0).all()
    assert sg["refinements"] == se["refinements"]
    assert _rel(dg, ref) < 1e-7 and _rel(de, ref) < 1e-7


def test_graph_kinetic_only(tiny):
    s = tiny
    dvg = perturbations(s, 2)
    ref, _ = O.apply_operator(s, dvg, 1e-12, kinetic_only=True, maxiter=400)
    dng, ierr, _ = _run(_op(s, l_kinetic_only=True, n_dfpt_maxiter=400), dvg, 1e-12)
    assert (ierr == 0).all()
    assert _rel(dng, ref) < 1e-10
