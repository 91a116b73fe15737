"""Davidson restart hand-off in WEST's file layout (Wstat/davidson_restart.f90):
the files written at the reference's checkpoints hold a consistent state, a run
interrupted at n_pdep_maxiter and resumed from them ends where the uninterrupted
run ends, and the files are cleared on convergence."""
import json
import os

import numpy as np
import pytest

from oracle import west_oracle as O
from west_b200.system import randomized_basis

pytestmark = pytest.mark.gpu

NVEC, TIMES = 4, 4
KW = dict(n_pdep_times=TIMES, tr2_dfpt=1e-12, trev_pdep=1e-6, trev_pdep_rel=1e-1)


def _op(s):
    from west_b200.wstat import ResponseOperator
    return ResponseOperator(s, verbose=False)


def test_restart_files_hold_the_davidson_state(small, tmp_path):
    from west_b200.pdep import read_davidson_restart
    d = str(tmp_path / "wstat_restart")
    ev, conv, vec, info = _op(small).davidson(randomized_basis(small, NVEC), NVEC, n_pdep_maxiter=2,
                                              restart_dir=d, n_steps_write_restart=1, **KW)
    assert info["dav_iter"] == 2
    r = read_davidson_restart(d)
    # the last iteration (kter = n_pdep_maxiter) exits before its checkpoint (:384-392)
    assert r["dav_iter"] == 1
    nb = r["nbase"]
    assert NVEC < nb <= NVEC * TIMES and r["dvg"].shape == (small.npw, nb) == r["dng"].shape
    assert r["conv"].shape == (NVEC,) and r["ew"].shape == (NVEC * TIMES,)
    # the basis is Gamma-orthonormal and hr is its bra-ket with dng (build_hr fills
    # hr(1:nbase+notcnv, new columns): the upper triangle and the diagonal)
    assert np.allclose(O.glbrak_gamma(r["dvg"], r["dvg"]), np.eye(nb), atol=1e-10)
    hr = r["hr"][:nb, :nb]
    ref = O.glbrak_gamma(r["dvg"], r["dng"])
    up = np.triu_indices(nb)
    assert np.abs(hr[up] - ref[up]).max() < 1e-10 * np.abs(ref).max()
    # vr holds the eigenvectors of hr for the ew of the same step
    hs = np.triu(hr) + np.triu(hr, 1).T
    vr = r["vr"][:nb, :NVEC]
    assert np.abs(hs @ vr - vr * r["ew"][:NVEC]).max() < 1e-9 * np.abs(r["ew"]).max()
    assert np.allclose(r["ev"], r["ew"][:NVEC])


def test_restart_resumes_to_the_uninterrupted_result(small, tmp_path):
    d = str(tmp_path / "wstat_restart")
    dvg0 = randomized_basis(small, NVEC)
    ev_a, conv_a, vec_a, info_a = _op(small).davidson(dvg0, NVEC, n_pdep_maxiter=100, **KW)
    assert info_a["converged"] == 1 and info_a["dav_iter"] > 3
    _op(small).davidson(dvg0, NVEC, n_pdep_maxiter=3, restart_dir=d, n_steps_write_restart=1, **KW)
    assert os.path.exists(os.path.join(d, "summary.json"))
    ev_c, conv_c, vec_c, info_c = _op(small).davidson(None, NVEC, n_pdep_maxiter=100, restart_dir=d,
                                                      n_steps_write_restart=1, restart=True, **KW)
    assert info_c["converged"] == 1
    assert info_c["dav_iter"] == info_a["dav_iter"]          # dav_iter continues from the checkpoint
    assert np.abs((ev_c - ev_a) / ev_a).max() < 1e-9
    assert np.allclose(np.abs(np.diag(O.glbrak_gamma(vec_c, vec_a))), 1.0, atol=1e-6)
    # davidson_restart_clear on convergence
    assert not os.path.exists(os.path.join(d, "summary.json"))
    assert not os.path.exists(os.path.join(d, "V000001.dat"))


def test_restart_from_the_starting_step(small, tmp_path):
    """A checkpoint at dav_iter = -1 (after the lite-solver application) resumes
    with the extra starting step (davidson_diago.f90:204-247)."""
    d = str(tmp_path / "wstat_restart")
    dvg0 = randomized_basis(small, NVEC)
    ev_a, _, _, info_a = _op(small).davidson(dvg0, NVEC, n_pdep_maxiter=100, **KW)
    _op(small).davidson(dvg0, NVEC, n_pdep_maxiter=1, restart_dir=d, n_steps_write_restart=1, **KW)
    # rewrite the summary as the dav_iter = -1 checkpoint of the first NVEC files
    sf = os.path.join(d, "summary.json")
    s = json.load(open(sf))
    s.update(dav_iter=-1, notcnv=NVEC, nbase=NVEC, conv=[False] * NVEC, ev=[0.0] * NVEC,
             ew=[0.0] * (NVEC * TIMES))
    json.dump(s, open(sf, "w"))
    ev_c, conv_c, _, info_c = _op(small).davidson(None, NVEC, n_pdep_maxiter=100, restart_dir=d, restart=True, **KW)
    assert info_c["converged"] == 1
    # the extra starting step applied the operator once before the iterations
    assert info_c["apply_calls"] == info_c["dav_iter"] + 1
    # another starting basis, another trajectory: the eigenvalues agree to the
    # Davidson's own accuracy at this trev_pdep, not to rounding
    assert np.abs((ev_c - ev_a) / ev_a).max() < 1e-3


def test_restart_needs_a_directory(small):
    from west_b200.lib import WestB200Error
    with pytest.raises(WestB200Error, match="restart_dir"):
        _op(small).davidson(randomized_basis(small, NVEC), NVEC, n_pdep_maxiter=2, n_steps_write_restart=1, **KW)
