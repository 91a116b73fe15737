"""The PDEP Davidson's dense steps as CUDA graphs (davidson_diago.f90:273-347).

With graphs on (the default) each iteration runs two graph launches around the
operator call: the reordering of the unconverged Ritz pairs, update_with_vr and
do_mgs before it; build_hr, diagox, the convergence test and the copy of the
state to the host after it.  A repeated solve replays the cached graphs and
must reproduce the first solve bit for bit; with graphs off the same kernels run
eagerly (the operator's PCG loop then also runs eagerly, with its own split-K
shapes, so the two agree to rounding: eigenvalues within 1e-10, identical
iteration counts and convergence flags)."""
import numpy as np
import pytest

from oracle import west_oracle as O
from west_b200.system import randomized_basis

pytestmark = pytest.mark.gpu


def _solve(op, dvg0, nvec, times, maxiter=100):
    return op.davidson(dvg0, nvec, n_pdep_times=times, n_pdep_maxiter=maxiter, tr2_dfpt=1e-12, trev_pdep=1e-6,
                       trev_pdep_rel=1e-1)


# (2, 2): the basis refresh of :390-414; (32, 4): a basis of 128, whose diagox is
# the block Jacobi with its sweep loop in a conditional WHILE node of the graph
@pytest.mark.parametrize("nvec,times", [(4, 4), (2, 2), (32, 4)])
def test_davidson_graphs_replay_and_eager(small, nvec, times):
    from west_b200.wstat import ResponseOperator
    s = small
    dvg0 = randomized_basis(s, nvec)
    op = ResponseOperator(s, verbose=False)
    ev1, conv1, vec1, info1 = _solve(op, dvg0, nvec, times)
    ev2, conv2, vec2, info2 = _solve(op, dvg0, nvec, times)      # cached graphs
    assert info1["dav_iter"] == info2["dav_iter"]
    assert (ev1 == ev2).all() and (conv1 == conv2).all() and (vec1 == vec2).all()
    op_e = ResponseOperator(s, verbose=False)
    op_e.set_graphs(False)
    ev3, conv3, vec3, info3 = _solve(op_e, dvg0, nvec, times)
    assert info3["dav_iter"] == info1["dav_iter"]
    assert (conv3 == conv1).all()
    assert np.abs((ev3 - ev1) / ev1).max() < 1e-10
    ov = O.glbrak_gamma(vec1, vec3)
    assert np.allclose(np.abs(np.diag(ov)), 1.0, atol=1e-8)


def test_davidson_graphs_after_diagox_grows_the_scratch(small):
    """wb_diagox on a larger matrix reallocates the eigensolver scratch the
    Davidson's cached graphs point into; the next solve must capture anew and
    reproduce the first one bit for bit."""
    import torch
    from west_b200.wstat import ResponseOperator, diagox
    s = small
    dvg0 = randomized_basis(s, 32)
    op = ResponseOperator(s, verbose=False)
    ev1, conv1, vec1, info1 = _solve(op, dvg0, 32, 4)             # basis 128: block Jacobi in the graph
    rng = np.random.default_rng(3)
    x = rng.standard_normal((200, 200))
    hr = torch.from_numpy(np.ascontiguousarray((x + x.T) / 2)).cuda()
    ew, _ = diagox(op, hr, 200, 8)
    assert np.allclose(ew, np.linalg.eigvalsh((x + x.T) / 2)[:8], rtol=0, atol=1e-11 * np.abs(ew).max())
    ev2, conv2, vec2, info2 = _solve(op, dvg0, 32, 4)
    assert info1["dav_iter"] == info2["dav_iter"]
    assert (ev1 == ev2).all() and (conv1 == conv2).all() and (vec1 == vec2).all()
