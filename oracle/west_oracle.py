"""CPU restatement (NumPy/SciPy, FP64) of WEST's Wstat response path.

TEST INFRASTRUCTURE ONLY.  This module is the checker: tests, the smoke check
and the CPU-baseline leg of the benchmark import it.  The product path
(``west_b200``) never imports, links or calls anything here.

What it restates, function by function, with the reference file:line each one
follows (paths inside the WEST 6.2.0 tree):

* ``apply_operator``            Wstat/apply_operator.f90:14-69
* ``dfpt``                      DFPT_kernel/dfpt_module.f90:22-533 (Gamma branches,
                                fractional occupations :328-401)
* ``linsolve_sternheimer``      DFPT_kernel/linsolve_sternheimer_m_wfcts.f90:14-382
* ``apply_sternheimerop``       DFPT_kernel/apply_sternheimerop_to_m_wfcs.f90:14-84
* ``precondition_m_wfcts``      DFPT_kernel/precondition_m_wfcts.f90:14-53
* ``apply_alpha_pc/pv``         Hamiltonian_kernel/apply_alpha_pc_to_m_wfcs.f90:48-72,
                                Hamiltonian_kernel/apply_alpha_pv_to_m_wfcs.f90:48-72
* ``glbrak_gamma``              Hamiltonian_kernel/glbrak.f90:14-43
* ``k_psi``                     Hamiltonian_kernel/k_psi.f90:14-85
* ``double/single_*fft_gamma``  FFT_kernel/fft_at_gamma.f90:30-203
* ``set_eprec``                 Tools/set_eprec.f90:14-60
* ``get_alpha_pv``              Tools/get_alpha_pv.f90:14-67

The Hamiltonian itself (``h_psi``) is Quantum ESPRESSO code that is not part
of the WEST tree (pinned by WEST's CI at qe-7.4.1).  ``h_psi`` below restates
QE's published Gamma-only algorithm: ``hpsi = g2kin*psi`` (h_psi_), the local
potential applied to band pairs through one complex FFT each
(vloc_psi_gamma), the Kleinman-Bylander term through the real-pair GEMMs of
calbec (``2 Re<beta|psi> - G0``) and add_vuspsi (``vkb (D becp)``), and the
Gamma fix ``Im hpsi(G=0) = 0``.  QE's FFT convention is kept: ``invfft`` is
the unscaled sum over exp(+iGr) and ``fwfft`` carries 1/N^3.

Parity status: parity unpinned at the QE boundary.  The reference ships no
golden vectors for apply_operator, h_psi or the FFTs; its only pins are
end-to-end PDEP eigenvalues of real molecules that need pw.x and downloaded
pseudopotentials, which are absent here, and the Fortran sources cannot be
compiled here (no Fortran compiler, no QE).  This restatement is therefore
checked by known-answer tests (FFT of plane waves, the Gamma pack/unpack
identity, the kinetic-only closed form, a dense direct solve, the plane-wave
count recorded in test-suite/test001/ref/wstat.json) and by committed
regression fixtures under tests/golden/.
"""
from __future__ import annotations

import os

import numpy as np

try:
    import scipy.fft as _sfft
except Exception:  # pragma: no cover
    _sfft = None

_WORKERS = int(os.environ.get("WEST_ORACLE_WORKERS", len(os.sched_getaffinity(0))))


# ----------------------------------------------------------------------------
# FFTs in QE's convention on an nr^3 box stored x fastest.
# ----------------------------------------------------------------------------
def _edges(nr):
    return tuple(int(x) for x in nr) if isinstance(nr, (tuple, list)) else (int(nr),) * 3


def _boxes(a, nr):
    n1, n2, n3 = _edges(nr)
    return a.reshape(a.shape[:-1] + (n3, n2, n1))


def invfft(box, nr):
    """QE invfft 'Wave': f(r) = sum_G f(G) exp(+iGr), unscaled.  box [..., nnr],
    nr the box edge or (nr1, nr2, nr3), x fastest."""
    x = _boxes(box, nr)
    if _sfft is not None:
        y = _sfft.ifftn(x, axes=(-3, -2, -1), norm="forward", workers=_WORKERS)
    else:
        y = np.fft.ifftn(x, axes=(-3, -2, -1)) * x.shape[-1] * x.shape[-2] * x.shape[-3]
    return y.reshape(box.shape)


def fwfft(box, nr):
    """QE fwfft 'Wave': f(G) = (1/N) sum_r f(r) exp(-iGr), N = nr1 nr2 nr3.  box [..., nnr]."""
    x = _boxes(box, nr)
    if _sfft is not None:
        y = _sfft.fftn(x, axes=(-3, -2, -1), norm="forward", workers=_WORKERS)
    else:
        y = np.fft.fftn(x, axes=(-3, -2, -1)) / (x.shape[-1] * x.shape[-2] * x.shape[-3])
    return y.reshape(box.shape)


# FFT_kernel/fft_at_gamma.f90 -------------------------------------------------
def double_invfft_gamma(s, a1, a2):
    """fft_at_gamma.f90:30-68.  a1, a2: [npw] or [k, npw] -> box [.., nnr]."""
    a1 = np.atleast_2d(a1); a2 = np.atleast_2d(a2)
    b = np.zeros((a1.shape[0], s.nnr), dtype=np.complex128)
    b[:, s.nl] = a1 + 1j * a2                              # :60
    b[:, s.nlm] = np.conj(a1 - 1j * a2)                    # :61 (wins at G=0)
    return invfft(b, s.nrs)


def double_fwfft_gamma(s, a):
    """fft_at_gamma.f90:72-118.  a: box [k, nnr] -> (b1, b2) each [k, npw]."""
    a = fwfft(np.atleast_2d(a), s.nrs)
    ap = a[:, s.nl]; am = a[:, s.nlm]
    fp = (ap + am) * 0.5                                   # :106
    fm = (ap - am) * 0.5                                   # :107
    b1 = fp.real + 1j * fm.imag                            # :108
    b2 = fp.imag - 1j * fm.real                            # :109
    return b1, b2


def single_invfft_gamma(s, a1):
    """fft_at_gamma.f90:122-158."""
    a1 = np.atleast_2d(a1)
    b = np.zeros((a1.shape[0], s.nnr), dtype=np.complex128)
    b[:, s.nl] = a1                                        # :152
    b[:, s.nlm] = np.conj(a1)                              # :153
    return invfft(b, s.nrs)


def single_fwfft_gamma(s, a):
    """fft_at_gamma.f90:162-203."""
    a = fwfft(np.atleast_2d(a), s.nrs)
    return a[:, s.nl]                                      # :194


# ----------------------------------------------------------------------------
# Bra-kets and projectors
# ----------------------------------------------------------------------------
def glbrak_gamma(a, b):
    """glbrak.f90:39-40: c = 2 a^T b over the real pairs minus the G=0 row
    (DGEMM alpha=2 then DGER -1 on the first real row).  a [npw, na], b [npw, nb]."""
    c = 2.0 * (a.real.T @ b.real + a.imag.T @ b.imag)
    c -= np.outer(a[0].real, b[0].real)
    return c


def apply_alpha_pc(s, f, alpha):
    """apply_alpha_pc_to_m_wfcs.f90:58-72 (Gamma): f <- alpha f - alpha evc (evc^T f)."""
    ps = glbrak_gamma(s.evc, f)
    return alpha * f - alpha * (s.evc @ ps)


def apply_alpha_pv(s, f, g, alpha):
    """apply_alpha_pv_to_m_wfcs.f90:58-72 (Gamma): g <- g + alpha evc (evc^T f)."""
    ps = glbrak_gamma(s.evc, f)
    return g + alpha * (s.evc @ ps)


def set_eprec(s, wfc=None):
    """set_eprec.f90:40-53: eprec_v = 1.35 sum_{G in half sphere} |psi_v(G)|^2 g2kin(G)."""
    wfc = s.evc if wfc is None else wfc
    return 1.35 * ((np.abs(wfc) ** 2) * s.g2kin[:, None]).sum(0)


def get_alpha_pv(et, nbnd_occ):
    """get_alpha_pv.f90:36-63: max(2 (e_max,occ - e_min), 0.01)."""
    return max(2.0 * (np.max(et[:nbnd_occ]) - np.min(et)), 0.01)


def precondition_m_wfcts(s, f, eprec):
    """precondition_m_wfcts.f90:35-51: pf = f / max(1, g2kin / eprec)."""
    return f / np.maximum(1.0, s.g2kin[:, None] / eprec[None, :])


# ----------------------------------------------------------------------------
# Hamiltonian (QE h_psi_, Gamma-only) and the Sternheimer operator
# ----------------------------------------------------------------------------
def vloc_psi_gamma(s, psi):
    """QE vloc_psi_gamma: bands in pairs through one complex FFT."""
    npw, m = psi.shape
    out = np.zeros_like(psi)
    npair = m // 2
    if npair:
        a1 = psi[:, 0:2 * npair:2].T; a2 = psi[:, 1:2 * npair:2].T
        for c0 in range(0, npair, 16):
            c1 = min(npair, c0 + 16)
            box = double_invfft_gamma(s, a1[c0:c1], a2[c0:c1])
            box *= s.vrs[None, :]
            b1, b2 = double_fwfft_gamma(s, box)
            out[:, 2 * c0:2 * c1:2] = b1.T
            out[:, 2 * c0 + 1:2 * c1:2] = b2.T
    if m % 2:
        box = single_invfft_gamma(s, psi[:, m - 1])
        box *= s.vrs[None, :]
        out[:, m - 1] = fwfft(box, s.nrs)[0, s.nl]
    return out


def h_psi(s, psi):
    """QE h_psi_ at Gamma: kinetic + vloc_psi_gamma + calbec/add_vuspsi, then
    Im hpsi(G=0) = 0."""
    hpsi = s.g2kin[:, None] * psi
    hpsi = hpsi + vloc_psi_gamma(s, psi)
    if s.nkb:
        becp = glbrak_gamma(s.vkb, psi)                    # calbec, Gamma real-pair form
        hpsi = hpsi + s.vkb @ (s.deeq @ becp)             # add_vuspsi
    hpsi[0] = hpsi[0].real
    return hpsi


def k_psi(s, psi):
    """k_psi.f90:51-77: kinetic-only Hamiltonian with Im hpsi(G=0) = 0."""
    hpsi = s.g2kin[:, None] * psi
    hpsi[0] = hpsi[0].real
    return hpsi


def apply_sternheimerop(s, psi, e, alpha, kinetic_only=False):
    """apply_sternheimerop_to_m_wfcs.f90:48-76: (H - e_v + alpha P_v) psi."""
    hpsi = k_psi(s, psi) if kinetic_only else h_psi(s, psi)
    hpsi = hpsi - e[None, :] * psi                         # :65-74
    return apply_alpha_pv(s, psi, hpsi, alpha)             # :76


def _gamma_dot_cols(a, b):
    """Column-wise Gamma dot 2 sum Re(a* b) - Re a0 Re b0
    (linsolve_sternheimer_m_wfcts.f90:164-180)."""
    t = (a.real * b.real + a.imag * b.imag).sum(0)
    return 2.0 * t - a[0].real * b[0].real


def linsolve_sternheimer(s, b, x, e, eprec, tr2, maxiter, alpha, kinetic_only=False,
                         trace=None):
    """linsolve_sternheimer_m_wfcts.f90:14-345: masked preconditioned CG for
    (H - e_v + alpha P_v) x_v = b_v, all m columns at once.

    The compaction of active bands follows map_lbnd2ibnd (:356-382): active
    bands are kept in increasing band order, so the operator sees them in the
    same pairs the reference forms.  Returns (x, ierr) with ierr = number of
    bands still unconverged (:332).  ``trace`` (a list) receives the active
    count at each iteration when given.
    """
    b = b.copy(); x = x.copy()
    npw, m = b.shape
    is_conv = np.zeros(m, dtype=bool)
    rho = np.zeros(m); rhoold = np.zeros(m)
    g = apply_sternheimerop(s, x, e, alpha, kinetic_only)   # :127
    g = g - b                                                 # :130-138
    h = np.zeros_like(g)
    l2i = np.flatnonzero(~is_conv)                             # :142
    not_conv = l2i.size
    prec = np.maximum(1.0, s.g2kin[:, None] / eprec[None, :])
    for it in range(1, maxiter + 1):                          # :146
        h[:, l2i] = g[:, l2i] / prec[:, l2i]                  # :150-160
        rho[l2i] = _gamma_dot_cols(h[:, l2i], g[:, l2i])      # :162-181, :210-218
        is_conv[l2i] = rho[l2i] < tr2
        l2i = np.flatnonzero(~is_conv)                         # :220
        not_conv = l2i.size
        if trace is not None:
            trace.append(not_conv)
        if not_conv == 0:                                     # :222
            break
        if it != 1:                                           # :226-240
            h[:, l2i] = -h[:, l2i] + (rho[l2i] / rhoold[l2i])[None, :] * b[:, l2i]
        else:
            h[:, l2i] = -h[:, l2i]
        t = apply_sternheimerop(s, h[:, l2i], e[l2i], alpha, kinetic_only)  # :251
        a = _gamma_dot_cols(h[:, l2i], g[:, l2i])              # :253-277
        c = _gamma_dot_cols(h[:, l2i], t)
        r = (a / c)[None, :]
        x[:, l2i] = x[:, l2i] - r * h[:, l2i]                  # :313-322
        g[:, l2i] = g[:, l2i] - r * t
        b[:, l2i] = h[:, l2i]
        rhoold[l2i] = rho[l2i]                                 # :324-329
    return x, not_conv


# ----------------------------------------------------------------------------
# dfpt and apply_operator
# ----------------------------------------------------------------------------
def dvpsi_rhs(s, aux_r):
    """dfpt_module.f90:241-278: dvpsi_v = P_G[psi_v(r) * Re dv(r)], bands in pairs."""
    nb = s.nbnd_occ
    dvpsi = np.zeros((s.npw, nb), dtype=np.complex128)
    dv = aux_r.real
    npair = nb // 2
    if npair:
        box = double_invfft_gamma(s, s.evc[:, 0:2 * npair:2].T, s.evc[:, 1:2 * npair:2].T)
        box *= dv[None, :]
        b1, b2 = double_fwfft_gamma(s, box)
        dvpsi[:, 0:2 * npair:2] = b1.T
        dvpsi[:, 1:2 * npair:2] = b2.T
    if nb % 2:
        box = single_invfft_gamma(s, s.evc[:, nb - 1])
        box = (box.real * dv[None, :]).astype(np.complex128)
        dvpsi[:, nb - 1] = single_fwfft_gamma(s, box)[0]
    return dvpsi


def drho_gamma(s, dpsi):
    """dfpt_module.f90:403-423: drho(r) = sum_v occ_v Re psi_v(r) Im(...) with
    psic = invfft(evc_v + i dpsi_v)."""
    box = double_invfft_gamma(s, s.evc.T, dpsi.T)
    return (s.occupation[:, None] * box.real * box.imag).sum(0)


DOCC_THR = 0.001   # westcom docc_thr (Modules/westcom.f90:417)
DE_THR = 0.001     # westcom de_thr (Modules/westcom.f90:418)


def nbnd_occ_full(s):
    """Tools/set_nbndocc.f90:58-69: the highest band whose occupation exceeds
    1 - docc_thr (all bands up to nbnd_occ count as fully occupied when the
    occupations are integer)."""
    full = np.flatnonzero(np.asarray(s.occupation) > 1.0 - DOCC_THR)
    return int(full.max()) + 1 if full.size else 0


def frac_coefficients(s, dvpsi):
    """dfpt_module.f90:328-337 and :363-393 (Gamma): psi_dvpsi(j, i) =
    <psi_j|dV psi_i> for the fractionally occupied bands j > nbnd_occ_full,
    zeroed for j <= i and for |occ_i - occ_j| < docc_thr, else scaled by
    (occ_i - occ_j) / occ_i / (e_i - e_j); degenerate pairs are an error as in
    the reference (errore)."""
    nb, nfull = s.nbnd_occ, nbnd_occ_full(s)
    if nfull >= nb:
        return None
    ps = glbrak_gamma(s.evc[:, nfull:nb], dvpsi)           # [nfrac, nbnd]
    occ, et = np.asarray(s.occupation), s.et
    for i in range(nb):
        for jf in range(nb - nfull):
            j = nfull + jf
            if j <= i:
                ps[jf, i] = 0.0
                continue
            docc = occ[i] - occ[j]
            if abs(docc) < DOCC_THR:
                ps[jf, i] = 0.0
                continue
            de = et[i] - et[j]
            if abs(de) < DE_THR:
                raise ValueError("dfpt: fractional occupation degenerate orbitals")
            ps[jf, i] *= docc / occ[i] / de
    return ps


def dfpt(s, dvg, tr2, maxiter=250, kinetic_only=False, eprec=None, trace=None):
    """dfpt_module.f90:22-533 at Gamma, one k-point, no band groups, integer or
    fractional occupations (l_frac_occ).  dvg [npw, m] -> (dng [npw, m], ierr [m])."""
    npw, m = dvg.shape
    l_dost = tr2 >= 0.0                                     # :130
    eprec = set_eprec(s) if eprec is None else eprec        # :211
    et = s.et[: s.nbnd_occ]
    nfull = nbnd_occ_full(s)
    dng = np.zeros((npw, m), dtype=np.complex128)
    ierrs = np.zeros(m, dtype=np.int64)
    for ipert in range(m):                                  # :227
        aux_r = single_invfft_gamma(s, dvg[:, ipert])[0]    # :235
        dvpsi = dvpsi_rhs(s, aux_r)                         # :241-278
        psi_dvpsi = frac_coefficients(s, dvpsi)             # :328-337, :363-393
        dvpsi = apply_alpha_pc(s, dvpsi, -1.0)              # :346
        dpsi = precondition_m_wfcts(s, dvpsi, eprec)        # :348
        if l_dost:                                          # :350-361
            tr = [] if trace is not None else None
            dpsi, ierr = linsolve_sternheimer(s, dvpsi, dpsi, et, eprec, tr2, maxiter,
                                              s.alpha_pv, kinetic_only, trace=tr)
            ierrs[ipert] = ierr
            if trace is not None:
                trace.append(tr)
        if psi_dvpsi is not None:                           # :397-398 (DGEMM)
            dpsi = dpsi + s.evc[:, nfull:s.nbnd_occ] @ psi_dvpsi
        aux_r = drho_gamma(s, dpsi)                          # :403-423
        aux_g = single_fwfft_gamma(s, aux_r.astype(np.complex128))[0]   # :478
        dng[:, ipert] += 2.0 * s.wk * aux_g / s.omega       # :485-487
    dng[0, :] = 0.0                                         # :502-503
    return dng, ierrs


def apply_operator(s, dvg, tr2, maxiter=250, kinetic_only=False, trace=None):
    """apply_operator.f90:44-67: dng = sqvc * chi0(sqvc * dvg)."""
    aux_g = dvg * s.sqvc[:, None]                           # :49-53
    dng, ierr = dfpt(s, aux_g, tr2, maxiter, kinetic_only, trace=trace)  # :58
    return dng * s.sqvc[:, None], ierr                      # :63-67


# ----------------------------------------------------------------------------
# PDEP Davidson (Wstat/davidson_diago.f90, Wstat/wstat_tools.f90), one image
# ----------------------------------------------------------------------------
def do_mgs(amat, start, end):
    """davidson_diago.f90:909-1117: modified Gram-Schmidt of columns [start, end)
    against [0, start) and among themselves, Gamma dot products; in place."""
    for k in range(end):
        if k >= start:                                                   # :1003-1031
            a = amat[:, k]
            anorm = 2.0 * (a.real ** 2 + a.imag ** 2).sum() - a[0].real ** 2
            amat[:, k] = a * (1.0 / np.sqrt(anorm))
        vec = amat[:, k].copy()                                          # :1035
        j0 = max(k + 1, start)
        if j0 >= end:
            continue
        blk = amat[:, j0:end]
        zb = 2.0 * (vec.real[:, None] * blk.real + vec.imag[:, None] * blk.imag).sum(0) \
            - vec[0].real * blk[0].real                                  # :1056-1085
        amat[:, j0:end] = blk - np.outer(vec, zb)                         # :1094 (ZGERU)


def build_hr(dvg, dng, col_start, col_end, hr, g_e):
    """wstat_tools.f90:345-468 (build_hr_real): hr(i, j) = <dvg_i|dng_j>_Gamma for
    i < g_e and j in [col_start, col_end)."""
    hr[:g_e, col_start:col_end] = glbrak_gamma(dvg[:, :g_e], dng[:, col_start:col_end])


def diagox(nbase, nvec, hr):
    """wstat_tools.f90:208-273 + linear_algebra_kernel.f90:84-200 (DSYEV 'U'):
    lowest nvec eigenpairs of the upper triangle of hr[:nbase, :nbase]."""
    a = np.triu(hr[:nbase, :nbase])
    a = a + np.triu(a, 1).T
    w, v = np.linalg.eigh(a)
    return w[:nvec], v[:, :nvec]


def davidson_diago_gamma(s, dvg0, nvec, nvecx, tr2_dfpt=1e-16, trev_pdep=1e-3, trev_pdep_rel=1e-1,
                         n_pdep_maxiter=100, n_dfpt_maxiter=250, apply=None, log=None):
    """davidson_diago.f90:31-437 on one image from the starting vectors dvg0
    (the output of do_randomize, davidson_diago.f90:171).  ``apply(dvg, tr2)``
    defaults to this module's apply_operator.  Returns (ev, conv, dvg[:, :nvec],
    dav_iter)."""
    if apply is None:
        def apply(v, tr2):
            return apply_operator(s, v, tr2, maxiter=n_dfpt_maxiter)[0]
    npw = dvg0.shape[0]
    dvg = np.zeros((npw, nvecx), complex)
    dng = np.zeros((npw, nvecx), complex)
    hr = np.zeros((nvecx, nvecx))
    vr = np.zeros((nvecx, nvecx))
    ew = np.zeros(nvecx)
    ev = np.zeros(nvec)
    conv = np.zeros(nvec, bool)
    nbase = nvec
    notcnv = nvec
    dvg[:, :nvec] = dvg0[:, :nvec]
    do_mgs(dvg, 0, nvec)                                                   # :175
    dng[:, :nvec] = apply(dvg[:, :nvec], -1.0)                             # :195-196
    dvg[:] = dng                                                           # :208
    do_mgs(dvg, 0, nvec)                                                   # :209
    tr2 = min(1e-4, 1e8 * tr2_dfpt)                                        # :229
    dng[:, :nvec] = apply(dvg[:, :nvec], tr2)
    build_hr(dvg, dng, 0, nvec, hr, nvec)                                  # :236
    w, v = diagox(nbase, nvec, hr)                                         # :240
    ew[:nvec] = w
    vr[:nbase, :nvec] = v
    ev[:] = ew[:nvec]
    if log is not None:
        log.append(dict(dav_iter=-1, ev=ev.copy(), notcnv=notcnv, dfpt_tr2=tr2, diago_dim=nbase))
    dav_iter = 0
    for kter in range(1, n_pdep_maxiter + 1):                               # :259
        dav_iter += 1
        ishift = np.zeros(nvecx, int)
        np_ = 0
        for n in range(nvec):                                              # :273-296
            if not conv[n]:
                ishift[nbase + np_] = n
                ew[nbase + np_] = ev[n]
                np_ += 1
        for j in range(nbase, nbase + notcnv):                             # :300, redistribute_vr_distr
            vr[:, j] = vr[:, ishift[j]]
        # update_with_vr_distr_real (wstat_tools.f90:945-1092)
        coef = vr[:nbase, nbase:nbase + notcnv]
        hg = dvg[:, :nbase] @ coef
        hg2 = dng[:, :nbase] @ coef
        dvg[:, nbase:nbase + notcnv] = -ew[nbase:nbase + notcnv][None, :] * hg + hg2
        do_mgs(dvg, nbase, nbase + notcnv)                                 # :306
        dng[:, nbase:nbase + notcnv] = apply(dvg[:, nbase:nbase + notcnv], tr2_dfpt)   # :324
        build_hr(dvg, dng, nbase, nbase + notcnv, hr, nbase + notcnv)     # :331
        nbase += notcnv
        w, v = diagox(nbase, nvec, hr)                                     # :340
        ew[:nvec] = w
        vr[:, :] = 0.0
        vr[:nbase, :nvec] = v
        conv = (np.abs((ew[:nvec] - ev) / ev) < trev_pdep_rel) & (np.abs(ew[:nvec] - ev) < trev_pdep)  # :346
        notcnv = int((~conv).sum())
        ev[:] = ew[:nvec]
        if log is not None:
            log.append(dict(dav_iter=dav_iter, ev=ev.copy(), notcnv=notcnv, dfpt_tr2=tr2_dfpt, diago_dim=nbase))
        if notcnv == 0 or nbase + notcnv > nvecx or kter == n_pdep_maxiter:   # :362
            if notcnv == 0:
                dvg[:, :nvec] = dvg[:, :nbase] @ vr[:nbase, :nvec]         # refresh_with_vr_distr
                break
            if kter == n_pdep_maxiter:
                break
            dvg[:, :nvec] = dvg[:, :nbase] @ vr[:nbase, :nvec]             # :397-398
            dng[:, :nvec] = dng[:, :nbase] @ vr[:nbase, :nvec]
            nbase = nvec
            hr[:, :] = 0.0
            vr[:, :] = 0.0
            for i in range(nbase):                                         # :404-409
                hr[i, i] = ev[i]
                vr[i, i] = 1.0
    return ev.copy(), conv.copy(), dvg[:, :nvec].copy(), dav_iter
