"""PDEP Davidson on the GPU (wb_davidson through the C ABI) against the oracle's
restatement of davidson_diago_gamma.  Bar: PDEP eigenvalues within 1e-6
relative, same convergence flags and iteration count."""
import numpy as np
import pytest

from oracle import west_oracle as O
from west_b200.system import build_system, randomized_basis

pytestmark = pytest.mark.gpu

TOL_EV = 1e-6


def _run(s, nvec, times, maxiter=100, tr2=1e-12, trev=1e-6, trev_rel=1e-1):
    from west_b200.wstat import ResponseOperator
    dvg0 = randomized_basis(s, nvec)
    op = ResponseOperator(s, verbose=False)
    ev, conv, vec, info = op.davidson(dvg0, nvec, n_pdep_times=times, n_pdep_maxiter=maxiter, tr2_dfpt=tr2,
                                      trev_pdep=trev, trev_pdep_rel=trev_rel)
    rev, rconv, rvec, rit = O.davidson_diago_gamma(s, dvg0, nvec, nvec * times, tr2_dfpt=tr2, trev_pdep=trev,
                                                    trev_pdep_rel=trev_rel, n_pdep_maxiter=maxiter)
    return ev, conv, vec, info, rev, rconv, rvec, rit


def test_davidson_small_matches_oracle(small):
    ev, conv, vec, info, rev, rconv, rvec, rit = _run(small, 4, 4)
    assert info["converged"] == 1 and rconv.all()
    assert info["dav_iter"] == rit
    assert np.abs((ev - rev) / rev).max() < TOL_EV
    assert (ev < 0).all()
    # eigenvectors: Gamma-orthonormal and the same up to sign
    ov = O.glbrak_gamma(vec, rvec)
    assert np.allclose(np.abs(np.diag(ov)), 1.0, atol=1e-5)
    assert np.allclose(O.glbrak_gamma(vec, vec), np.eye(4), atol=1e-10)


def test_davidson_refresh_path(tiny):
    """n_pdep_basis = 2 n_pdep_eigen forces the basis refresh of davidson_diago.f90:390-414."""
    ev, conv, vec, info, rev, rconv, rvec, rit = _run(tiny, 2, 2)
    assert info["dav_iter"] == rit
    assert (conv == rconv).all()
    assert np.abs((ev - rev) / rev).max() < TOL_EV


def test_davidson_maxiter_exit(small):
    ev, conv, vec, info, rev, rconv, rvec, rit = _run(small, 4, 4, maxiter=1)
    assert info["dav_iter"] == rit == 1
    assert (conv == rconv).all()
    assert np.abs((ev - rev) / rev).max() < TOL_EV


def test_davidson_block_jacobi_basis(small):
    """n_pdep_basis = 128 > 112: the subspace eigensolver is the block Jacobi
    over many CTAs (wb_diagox above the one-CTA size)."""
    ev, conv, vec, info, rev, rconv, rvec, rit = _run(small, 32, 4)
    assert info["converged"] == 1 and rconv.all()
    assert info["dav_iter"] == rit
    assert np.abs((ev - rev) / rev).max() < TOL_EV


def test_davidson_rejects_small_basis(small):
    from west_b200.lib import WestB200Error
    from west_b200.wstat import ResponseOperator
    op = ResponseOperator(small, verbose=False)
    with pytest.raises(WestB200Error, match="n_pdep_basis"):
        op.davidson(randomized_basis(small, 4), 4, n_pdep_times=1)


_C1 = {}


def _c1_oracle():
    if not _C1:
        s = build_system("c1", "cuda")
        dvg0 = randomized_basis(s, 16)
        rev, rconv, _, rit = O.davidson_diago_gamma(s, dvg0, 16, 64, tr2_dfpt=1e-10, trev_pdep=1e-6,
                                                     trev_pdep_rel=1e-1)
        _C1.update(s=s, dvg0=dvg0, rev=rev, rconv=rconv, rit=rit)
    return _C1


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_davidson_c1_configuration(precision):
    """L = 15 bohr, 20 Ry, 48^3, 4 atoms, 8 bands; n_pdep_eigen 16, n_pdep_times 4,
    PCG 1e-10, Davidson tolerance 1e-6; both forms against the FP64 oracle."""
    from west_b200.wstat import ResponseOperator
    c = _c1_oracle()
    op = ResponseOperator(c["s"], verbose=False)
    op.set_precision(precision)
    ev, conv, vec, info = op.davidson(c["dvg0"], 16, n_pdep_times=4, tr2_dfpt=1e-10, trev_pdep=1e-6,
                                      trev_pdep_rel=1e-1)
    assert info["converged"] == 1 and c["rconv"].all()
    assert np.abs((ev - c["rev"]) / c["rev"]).max() < TOL_EV


def test_davidson_108cube_reduced_both_forms():
    """The 108^3 box (radix 12 x 9 transforms, one-pass plane kernel) in a
    reduced system (3 bands, npw 36,763): 8 eigenpairs x 4, tight thresholds
    (tr2_dfpt 1e-14, trev_pdep 1e-9), FP64 and mixed against the oracle's
    Davidson at 1e-6."""
    import math
    from west_b200.system import SystemSpec
    from west_b200.wstat import ResponseOperator
    L = 8.0 + 108 / 6.0
    spec = SystemSpec(L=L, ecutwfc=(26 * 2.0 * math.pi / L) ** 2 * (1.0 + 1e-9), nr=108, natoms=2, nbnd_occ=3,
                      proj="sp", seed=208)
    s = build_system(spec, "cuda")
    dvg0 = randomized_basis(s, 8)
    kw = dict(tr2_dfpt=1e-14, trev_pdep=1e-9, trev_pdep_rel=1e-1)
    rev, rconv, _, rit = O.davidson_diago_gamma(s, dvg0, 8, 32, **kw)
    assert rconv.all()
    for precision in ("fp64", "mixed"):
        op = ResponseOperator(s, verbose=False)
        op.set_precision(precision)
        ev, conv, _, info = op.davidson(dvg0, 8, n_pdep_times=4, **kw)
        assert info["converged"] == 1, precision
        assert np.abs((ev - rev) / rev).max() < TOL_EV, (precision, np.abs((ev - rev) / rev).max())
