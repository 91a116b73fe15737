"""Boxes without a compiled edge run the runtime-size transforms: non-cubic
boxes (QE picks nr1, nr2, nr3 separately for orthorhombic cells) and the
2, 3, 5, 7-smooth edges outside the compiled list (45, 50, 54, 75, 90, 120,
128, 144 here: radices 2, 3, 4, 5, 8 in up to five stages).  Each case is a
small synthetic system (2 atoms, 3 bands) whose sphere reaches about a quarter
of every edge, checked against the oracle like the compiled edges: 5 fixed PCG
steps and a converged solve (tr2 1e-14) in FP64 (1e-10), the converged solve
in the mixed form (1e-7), identical ierr."""
import math

import numpy as np
import pytest

from oracle import west_oracle as O
from west_b200.system import SystemSpec, build_system, perturbations

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _gpu(s, dvg, tr2, precision="fp64", **kw):
    from west_b200.wstat import ResponseOperator
    op = ResponseOperator(s, verbose=False, **kw)
    op.set_precision(precision)
    dng = np.zeros_like(dvg, order="F")
    ierr = op.apply_operator(dvg.shape[1], dvg, dng, tr2, 1)
    st = op.stats()
    op.close()
    return dng, ierr, st


def _spec(L, nr, seed):
    """The largest cutoff whose sphere stays below a quarter of every edge."""
    q = min((n // 4 - 1) * 2.0 * math.pi / l for l, n in zip(L, nr))
    return SystemSpec(L=tuple(L), ecutwfc=q * q * (1.0 + 1e-9), nr=tuple(nr), natoms=2, nbnd_occ=3, proj="sp",
                      seed=seed)


def _check(L, nr, seed):
    s = build_system(_spec(L, nr, seed), "cuda")
    assert s.nrs == tuple(nr)
    dvg = perturbations(s, 2, seed=seed)
    fixed, ferr = O.apply_operator(s, dvg, 0.0, maxiter=5)
    conv, cerr = O.apply_operator(s, dvg, 1e-14, maxiter=400)
    assert (cerr == 0).all()
    got, ierr, st = _gpu(s, dvg, 0.0, n_dfpt_maxiter=5)
    assert (ierr == ferr).all() and (ierr == s.nbnd_occ).all()
    assert _rel(got, fixed) < 1e-10, ("fixed", _rel(got, fixed))
    got, ierr, _ = _gpu(s, dvg, 1e-14, n_dfpt_maxiter=400)
    assert (ierr == 0).all()
    assert _rel(got, conv) < 1e-10, ("fp64", _rel(got, conv))
    got, ierr, st = _gpu(s, dvg, 1e-14, "mixed", n_dfpt_maxiter=400)
    assert (ierr == 0).all() and st["refinements"] >= 1
    assert _rel(got, conv) < 1e-7, ("mixed", _rel(got, conv))


@pytest.mark.parametrize("L,nr", [((10.0, 12.0, 14.0), (32, 36, 45)),
                                  ((15.0, 11.0, 13.0), (54, 40, 50)),
                                  ((9.0, 9.0, 18.0), (30, 30, 60)),
                                  ((12.0, 16.0, 10.0), (42, 56, 35))])
def test_noncubic_box(L, nr):
    _check(L, nr, seed=sum(nr))


@pytest.mark.parametrize("n", [45, 50, 54, 75, 90, 120, 128, 144])
def test_uncompiled_cubic_edge(n):
    L = 8.0 + n / 6.0
    _check((L, L, L), (n, n, n), seed=n)


def test_edge_with_large_prime_rejected():
    from west_b200.lib import WestB200Error
    from west_b200.system import build_system as bs
    from west_b200.wstat import ResponseOperator
    s = bs(_spec((10.0, 10.0, 10.0), (22, 22, 22), 1))
    with pytest.raises(WestB200Error, match="prime factor above 7"):
        ResponseOperator(s, verbose=False)
