"""Known-answer and regression tests of the CPU oracle (no GPU)."""
import json
import math
import os

import numpy as np
import pytest

from oracle import west_oracle as O
from west_b200.system import (_dense_gamma_hamiltonian, build_system, gamma_half_sphere, perturbations, SPECS)

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _pins():
    return json.load(open(os.path.join(GOLDEN, "reference_pins.json")))


def test_half_sphere_count_matches_reference_log():
    """test001 (cubic L=20 bohr, 25 Ry) records npw.sum = 8440 and a 64^3 box."""
    p = _pins()
    mill, _ = gamma_half_sphere(p["cell_alat_bohr"], p["ecutwfc_ry"], p["fft_s"][0])
    assert len(mill) == p["npw_sum"] == 8440
    assert (mill[0] == 0).all()
    assert p["gamma_only"]


def test_named_workload_sizes():
    assert len(gamma_half_sphere(15.0, 20.0, 48)[0]) == 2521
    assert len(gamma_half_sphere(30.0, 30.0, 108)[0]) == 37387
    assert len(gamma_half_sphere(25.0, 25.0, 80)[0]) == 16494


def test_plane_wave_invfft(tiny):
    """single_invfft_gamma of a unit coefficient at G gives 2 cos(G r)."""
    s = tiny
    ig = 5
    a = np.zeros(s.npw, complex); a[ig] = 1.0
    box = O.single_invfft_gamma(s, a)[0].reshape(s.nr, s.nr, s.nr)
    n = np.arange(s.nr)
    mz, my, mx = s.mill[ig][2], s.mill[ig][1], s.mill[ig][0]
    ph = 2 * math.pi * (mx * n[None, None, :] + my * n[None, :, None] + mz * n[:, None, None]) / s.nr
    np.testing.assert_allclose(box.real, 2 * np.cos(ph), atol=1e-12)
    np.testing.assert_allclose(box.imag, 0.0, atol=1e-12)
    # forward of the real function returns the coefficient (QE: fwfft carries 1/N^3)
    back = O.single_fwfft_gamma(s, box.ravel())[0]
    np.testing.assert_allclose(back, a, atol=1e-14)


def test_gamma_pack_unpack_roundtrip(small):
    s = small
    rng = np.random.default_rng(3)
    a1 = rng.standard_normal(s.npw) + 1j * rng.standard_normal(s.npw)
    a2 = rng.standard_normal(s.npw) + 1j * rng.standard_normal(s.npw)
    a1[0] = a1[0].real; a2[0] = a2[0].real
    b1, b2 = O.double_fwfft_gamma(s, O.double_invfft_gamma(s, a1, a2))
    np.testing.assert_allclose(b1[0], a1, atol=1e-13)
    np.testing.assert_allclose(b2[0], a2, atol=1e-13)


@pytest.mark.parametrize("name", ["tiny", "small"])
def test_hpsi_reproduces_ground_state(name):
    """The FFT-based h_psi and the dense diagonalisation agree: H evc = et evc."""
    s = build_system(name)
    r = O.h_psi(s, s.evc) - s.evc * s.et[None, : s.nbnd_occ]
    assert np.abs(r).max() < 1e-12
    np.testing.assert_allclose(O.glbrak_gamma(s.evc, s.evc), np.eye(s.nbnd_occ), atol=1e-12)


def _to_real(c):
    return np.concatenate([c[:1].real, math.sqrt(2) * c[1:].real, math.sqrt(2) * c[1:].imag])


def _from_real(x, npw):
    c = np.empty(npw, complex)
    c[0] = x[0]
    c[1:] = (x[1:npw] + 1j * x[npw:]) / math.sqrt(2)
    return c


def test_pcg_matches_dense_direct_solve(small):
    """linsolve_sternheimer at tight tr2 equals a direct solve of H - e_v + alpha Pv."""
    s = small
    H = _dense_gamma_hamiltonian(dict(nr=s.nr, mill=s.mill, vrs=s.vrs, vkb=s.vkb, deeq=s.deeq,
                                      g2kin=s.g2kin)).numpy()
    H = 0.5 * (H + H.T)
    U = np.stack([_to_real(s.evc[:, v]) for v in range(s.nbnd_occ)], 1)
    rng = np.random.default_rng(5)
    b = rng.standard_normal((s.npw, s.nbnd_occ)) + 1j * rng.standard_normal((s.npw, s.nbnd_occ))
    b[0] = b[0].real
    b = O.apply_alpha_pc(s, b, -1.0)
    eprec = O.set_eprec(s)
    x0 = O.precondition_m_wfcts(s, b, eprec)
    x, ierr = O.linsolve_sternheimer(s, b, x0, s.et[: s.nbnd_occ], eprec, 1e-24, 500, s.alpha_pv)
    assert ierr == 0
    for v in range(s.nbnd_occ):
        A = H - s.et[v] * np.eye(H.shape[0]) + s.alpha_pv * U @ U.T
        y = np.linalg.solve(A, _to_real(b[:, v]))
        np.testing.assert_allclose(x[:, v], _from_real(y, s.npw), atol=1e-9 * np.abs(y).max())


def test_kinetic_only_operator_is_k_psi(tiny):
    s = tiny
    rng = np.random.default_rng(1)
    psi = rng.standard_normal((s.npw, 2)) + 1j * rng.standard_normal((s.npw, 2))
    e = np.array([0.1, -0.2])
    got = O.apply_sternheimerop(s, psi, e, s.alpha_pv, kinetic_only=True)
    want = s.g2kin[:, None] * psi
    want[0] = want[0].real
    want = want - e[None, :] * psi + s.alpha_pv * (s.evc @ O.glbrak_gamma(s.evc, psi))
    np.testing.assert_allclose(got, want, atol=1e-13)


def test_response_matrix_symmetric_negative(tiny):
    s = tiny
    dvg = perturbations(s, 4)
    dng, ierr = O.apply_operator(s, dvg, 1e-20, maxiter=400)
    assert (ierr == 0).all()
    hr = O.glbrak_gamma(dvg, dng)
    assert np.abs(hr - hr.T).max() < 1e-8 * np.abs(hr).max()
    assert np.linalg.eigvalsh(0.5 * (hr + hr.T)).max() < 0


def test_lite_solver_is_preconditioned_rhs(tiny):
    s = tiny
    dvg = perturbations(s, 2)
    dng, ierr = O.apply_operator(s, dvg, -1.0)
    assert (ierr == 0).all()
    aux = dvg * s.sqvc[:, None]
    want = np.zeros_like(dng)
    eprec = O.set_eprec(s)
    for p in range(2):
        dv = O.single_invfft_gamma(s, aux[:, p])[0]
        dvpsi = O.apply_alpha_pc(s, O.dvpsi_rhs(s, dv), -1.0)
        dpsi = O.precondition_m_wfcts(s, dvpsi, eprec)
        drho = O.drho_gamma(s, dpsi)
        want[:, p] = 2 * s.wk * O.single_fwfft_gamma(s, drho.astype(complex))[0] / s.omega
    want[0] = 0
    np.testing.assert_allclose(dng, want * s.sqvc[:, None], atol=1e-12 * np.abs(want).max())


def test_oracle_regression_fixture():
    """The oracle reproduces its committed outputs on the committed inputs."""
    g = np.load(os.path.join(GOLDEN, "oracle_tiny.npz"))
    s = build_system("tiny")
    np.testing.assert_allclose(np.abs(s.evc), np.abs(g["evc"]), atol=1e-10)
    s.evc = g["evc"]; s.et = g["et"]
    for tag, tr2, maxit in (("lite", -1.0, 250), ("tr2_1e-12", 1e-12, 250), ("fixed5", 0.0, 5)):
        dng, ierr = O.apply_operator(s, g["dvg"], tr2, maxiter=maxit)
        ref = g["dng_" + tag]
        assert np.abs(dng - ref).max() <= 1e-10 * np.abs(ref).max()
        assert (ierr == g["ierr_" + tag]).all()


def test_davidson_first_threshold_matches_reference_log():
    """davidson_diago.f90:229: the second starting apply uses min(1e-4, 1e8 tr2_dfpt)."""
    p = _pins()
    assert min(1e-4, 1e8 * p["tr2_dfpt"]) == p["davitr_dfpt_tr2"][0]
    assert all(t == p["tr2_dfpt"] for t in p["davitr_dfpt_tr2"][1:])


def _sum_over_states_dng(s, dvg):
    """dng from the independent-particle response written as a sum over all
    eigenpairs of the dense Gamma Hamiltonian:
    drho(r) = sum_{i<j} (f_i - f_j) / (e_i - e_j) psi_i(r) psi_j(r) <psi_j|dV|psi_i>,
    f = the occupations of the occupied bands and 0 above; then the prefactors
    of dfpt_module.f90:485-487 and apply_operator.f90:49-67."""
    import math
    from west_b200.system import _dense_gamma_hamiltonian
    H = _dense_gamma_hamiltonian(dict(nr=s.nr, mill=s.mill, vrs=s.vrs, vkb=s.vkb, deeq=s.deeq,
                                      g2kin=s.g2kin)).numpy()
    w, v = np.linalg.eigh(0.5 * (H + H.T))
    npw = s.npw
    psi = np.empty((npw, w.size), dtype=np.complex128)
    psi[0] = v[0]
    psi[1:] = (v[1:npw] + 1j * v[npw:]) / math.sqrt(2.0)
    f = np.zeros(w.size)
    f[: s.nbnd_occ] = s.occupation
    psir = np.stack([O.single_invfft_gamma(s, psi[:, k])[0].real for k in range(w.size)])
    dng = np.zeros_like(dvg)
    for p in range(dvg.shape[1]):
        dv = O.single_invfft_gamma(s, dvg[:, p] * s.sqvc)[0].real
        M = np.stack([O.single_fwfft_gamma(s, (psir[i] * dv).astype(np.complex128))[0] for i in range(w.size)], 1)
        M = O.glbrak_gamma(psi, M)                       # M[j, i] = <psi_j|dV|psi_i>
        drho = np.zeros(s.nnr)
        for i in range(w.size):
            for j in range(i + 1, w.size):
                if f[i] != f[j]:
                    drho += (f[i] - f[j]) / (w[i] - w[j]) * psir[i] * psir[j] * M[j, i]
        g = O.single_fwfft_gamma(s, drho.astype(np.complex128))[0]
        dng[:, p] = 2.0 * s.wk * g / s.omega * s.sqvc
    dng[0] = 0.0
    return dng


@pytest.mark.parametrize("frac", [(), (0.5,)])
def test_dfpt_matches_sum_over_states(frac):
    """The Sternheimer route (integer occupations, and l_frac_occ with the
    correction of dfpt_module.f90:328-401) against the sum over all states."""
    import dataclasses
    from west_b200.system import SPECS, build_system, perturbations
    s = build_system(dataclasses.replace(SPECS["tiny"], frac_occ=frac))
    if frac:
        assert O.nbnd_occ_full(s) == s.nbnd_occ - 1
    dvg = perturbations(s, 2)
    got, ierr = O.apply_operator(s, dvg, 1e-26, maxiter=400)
    ref = _sum_over_states_dng(s, dvg)
    assert (ierr == 0).all()
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-9
