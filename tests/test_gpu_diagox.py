"""wb_diagox (diagox_dsy, Wstat/wstat_tools.f90:48) against LAPACK (numpy eigh)
through the C ABI: the one-CTA Jacobi (nbase <= 112) and the block Jacobi over
many CTAs (nbase > 112, up to the 1024 of the large-cell basis).

Bars, with eps the FP64 unit roundoff: eigenvalues within 8 n eps of the
largest |eigenvalue| (the backward-error scale of any dense symmetric
eigensolver, LAPACK's included; a sweep of block rotations accumulates a few
ulps of the norm per round), eigenvectors orthonormal to 1e-12 and residuals
||A v - l v|| below 16 n eps ||A||.  The matrices mimic a PDEP
subspace: negative spectrum decaying over four decades with a few exactly
degenerate pairs; only the upper triangle is meaningful (the lower one holds
noise, which DSYEV 'U' ignores too)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _matrix(n, seed):
    rng = np.random.default_rng(seed)
    lam = -np.exp(-np.linspace(0.0, 9.0, n))
    lam[5] = lam[4]
    lam[n // 2 + 1] = lam[n // 2]
    q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    a = (q * lam) @ q.T
    a = 0.5 * (a + a.T)
    noisy = a.copy()
    il = np.tril_indices(n, -1)
    noisy[il] = rng.standard_normal(il[0].size)
    return a, noisy


@pytest.mark.parametrize("n,nvec,ldh", [(40, 10, 40), (112, 28, 120), (113, 30, 113), (200, 50, 256),
                                        (512, 128, 512), (1024, 256, 1024)])
def test_diagox_matches_lapack(n, nvec, ldh):
    import torch
    from west_b200.system import build_system
    from west_b200.wstat import ResponseOperator, diagox

    a, noisy = _matrix(n, n)
    op = ResponseOperator(build_system("tiny"), verbose=False)
    h = np.zeros((n, ldh))                 # column-major [ldh, n] as row-major [n, ldh]
    h[:, :n] = noisy.T
    hr = torch.from_numpy(h).cuda()
    ew, vr = diagox(op, hr, n, nvec)
    w, _ = np.linalg.eigh(a)
    eps = np.finfo(np.float64).eps / 2
    scale = np.abs(w).max()
    assert np.abs(ew - w[:nvec]).max() < 8 * n * eps * scale
    v = vr.cpu().numpy().T                 # [n, nvec]
    assert np.abs(v.T @ v - np.eye(nvec)).max() < 1e-12
    assert np.linalg.norm(a @ v - v * ew, axis=0).max() < 16 * n * eps * np.linalg.norm(a)


def test_diagox_rejects_bad_sizes():
    import torch
    from west_b200.lib import WestB200Error
    from west_b200.system import build_system
    from west_b200.wstat import ResponseOperator, diagox

    op = ResponseOperator(build_system("tiny"), verbose=False)
    hr = torch.zeros((8, 8), dtype=torch.float64, device="cuda")
    with pytest.raises(WestB200Error, match="nvec"):
        diagox(op, hr, 8, 9)
