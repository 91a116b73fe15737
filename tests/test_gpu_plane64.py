"""64^3 box (the c2 cell: L = 20 bohr, 25 Ry, 32 bands): the only box size of
the test systems that runs the fused local-potential plane kernel with the
grouped-row plane layout, the block-per-half-warp column mapping and the
bank-ordered stick pairs.  dng of two perturbations against the oracle in
both forms (bars as in the other parity tests: 1e-10 FP64, 1e-7 mixed)."""
import numpy as np
import pytest

from oracle import west_oracle as O
from west_b200.system import build_system, perturbations

pytestmark = pytest.mark.gpu

TR2 = 1e-16  # tight, so neither side stops one iteration apart on the threshold
_CACHE = {}


def _case():
    if not _CACHE:
        s = build_system("c2", "cuda")
        dvg = perturbations(s, 2)
        ref, ierr = O.apply_operator(s, dvg, TR2)
        assert (ierr == 0).all()
        _CACHE.update(s=s, dvg=dvg, ref=ref)
    return _CACHE["s"], _CACHE["dvg"], _CACHE["ref"]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_c2_fused_plane_matches_oracle(precision):
    from west_b200.wstat import ResponseOperator
    s, dvg, ref = _case()
    assert s.nr == 64
    op = ResponseOperator(s, verbose=False)
    op.set_precision(precision)
    dng = np.zeros_like(dvg, order="F")
    op.apply_operator(dvg.shape[1], dvg, dng, TR2, 1)
    tuned = op.tuning()
    assert tuned["plane_fused_fp64" if precision == "fp64" else "plane_fused_mixed"]
    rel = np.linalg.norm(dng - ref) / np.linalg.norm(ref)
    assert rel < (1e-10 if precision == "fp64" else 1e-7), rel
