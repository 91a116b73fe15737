"""The iterative ground-state solver (matrix-free block LOBPCG on the Gamma half
sphere, used for cells whose dense real basis is too large) against the dense
eigensolver on the same synthetic Hamiltonian.  CPU only."""
import numpy as np
import pytest

import west_b200.system as S


def _sysd(name):
    sp = S.SPECS[name]
    rng = np.random.default_rng(sp.seed)
    mill, tpiba2 = S.gamma_half_sphere(sp.L, sp.ecutwfc, sp.nr)
    tau = rng.uniform(0.0, sp.L, size=(sp.natoms, 3))
    vkb = S._kb_projectors(mill, sp.L, tau, sp.proj, sp.sigma_p)
    return sp, dict(nr=sp.nr, mill=mill, vrs=S._local_potential(sp.L, sp.nr, tau, sp.Z, sp.sigma), vkb=vkb,
                    deeq=np.eye(vkb.shape[1]) * sp.dion, g2kin=(mill.astype(np.float64) ** 2).sum(1) * tpiba2)


def _gdot(a, b):
    return 2 * (a.conj().T @ b).real - np.outer(a[0].conj(), b[0]).real


@pytest.mark.parametrize("name", ["tiny", "small"])
def test_iterative_matches_dense(name):
    sp, sysd = _sysd(name)
    nb = sp.nbnd_occ + sp.nbnd_extra
    w1, e1 = S._ground_state(sysd, nb)
    w2, e2 = S._ground_state_iterative(sysd, nb)
    assert np.abs(w1 - w2).max() < 1e-10
    no = sp.nbnd_occ
    sv = np.linalg.svd(_gdot(e1[:, :no], e2[:, :no]))[1]      # occupied subspaces coincide
    assert np.abs(sv - 1).max() < 1e-10
    assert np.abs(_gdot(e2, e2) - np.eye(nb)).max() < 1e-12
    assert np.abs(e2[0].imag).max() == 0.0


def test_matrix_free_h_matches_dense(tiny):
    """H psi of the matrix-free operator equals the dense Hamiltonian's action."""
    import torch
    sp, sysd = _sysd("tiny")
    H = S._GammaH(sysd, "cpu")
    Hd = S._dense_gamma_hamiltonian(sysd).numpy()
    npw = sysd["mill"].shape[0]
    rng = np.random.default_rng(3)
    x = rng.standard_normal(2 * npw - 1)
    psi = np.empty(npw, dtype=np.complex128)            # real basis -> half-sphere coefficients
    psi[0] = x[0]
    psi[1:] = (x[1:npw] + 1j * x[npw:]) / np.sqrt(2.0)
    hpsi = H(torch.as_tensor(psi[:, None]))[:, 0].numpy()
    y = Hd @ x
    ref = np.empty(npw, dtype=np.complex128)
    ref[0] = y[0]
    ref[1:] = (y[1:npw] + 1j * y[npw:]) / np.sqrt(2.0)
    assert np.abs(hpsi - ref).max() < 1e-11 * np.abs(ref).max()
