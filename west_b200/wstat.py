"""Python host interface mirroring WEST's Wstat response operator.

``ResponseOperator.apply_operator(m, dvg, dng, tr2, iq)`` has the argument
meaning of ``SUBROUTINE apply_operator(m, dvg, dng, tr2, iq)``
(Wstat/apply_operator.f90:14): ``dvg`` and ``dng`` are ``[npwqx, m]``
complex128 arrays (Fortran order), ``dng`` is overwritten, ``tr2 < 0``
selects the lite solver, and ``iq`` must be 1 (Gamma).  Unconverged bands are
reported the way dfpt does (a WARNING line per perturbation,
DFPT_kernel/dfpt_module.f90:358-359) and returned as the ``ierr`` array;
setup errors raise, where WEST calls ``errore``.

Device arrays are accepted as torch CUDA tensors (complex128, Fortran column
layout expressed as a ``[m, npwqx]`` row-major tensor), which skips the host
copies.
"""
from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

from . import lib as _lib
from .system import GammaSystem


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


class ResponseOperator:
    """B200 implementation of apply_operator for one Gamma-point ground state."""

    def __init__(self, system: GammaSystem, n_dfpt_maxiter: int = 250, l_kinetic_only: bool = False,
                 device: int = 0, verbose: bool = True):
        self._lib = _lib.load()
        self.system = system
        self.verbose = verbose
        s = system
        self._keep = keep = dict(
            nl=np.ascontiguousarray(s.nl + 1, dtype=np.int32),
            nlm=np.ascontiguousarray(s.nlm + 1, dtype=np.int32),
            g2kin=np.ascontiguousarray(s.g2kin, dtype=np.float64),
            vrs=np.ascontiguousarray(s.vrs, dtype=np.float64),
            evc=np.asfortranarray(s.evc, dtype=np.complex128),
            et=np.ascontiguousarray(s.et[: s.nbnd_occ], dtype=np.float64),
            occ=np.ascontiguousarray(s.occupation, dtype=np.float64),
            vkb=np.asfortranarray(s.vkb, dtype=np.complex128),
            deeq=np.asfortranarray(s.deeq, dtype=np.float64),
            sqvc=np.ascontiguousarray(s.sqvc, dtype=np.float64),
        )
        ws = _lib.WbSystem()
        ws.npw = ws.npwx = s.npw
        ws.nr1, ws.nr2, ws.nr3 = s.nrs
        ws.nbnd_occ = s.nbnd_occ
        ws.nkb = s.nkb
        ws.n_dfpt_maxiter = n_dfpt_maxiter
        ws.l_kinetic_only = int(bool(l_kinetic_only))
        ws.gstart = 2
        ws.nl = _ptr(keep["nl"]); ws.nlm = _ptr(keep["nlm"])
        ws.g2kin = _ptr(keep["g2kin"]); ws.vrs = _ptr(keep["vrs"])
        ws.evc = _ptr(keep["evc"]); ws.et = _ptr(keep["et"]); ws.occupation = _ptr(keep["occ"])
        ws.vkb = _ptr(keep["vkb"]); ws.deeq = _ptr(keep["deeq"]); ws.sqvc = _ptr(keep["sqvc"])
        ws.alpha_pv = s.alpha_pv
        ws.omega = s.omega
        ws.wk = s.wk
        ctx = ctypes.c_void_p()
        _lib.check(self._lib.wb_ctx_create(ctypes.byref(ctx), ctypes.byref(ws), device))
        self._ctx = ctx
        self.npwqx = s.npw

    def close(self):
        if getattr(self, "_ctx", None) is not None and self._ctx.value:
            self._lib.wb_ctx_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_precision(self, mode: str):
        code = {"fp64": _lib.WB_PRECISION_FP64, "mixed": _lib.WB_PRECISION_MIXED}[mode]
        _lib.check(self._lib.wb_set_precision(self._ctx, code))

    def set_batch(self, max_perturbations: int):
        _lib.check(self._lib.wb_set_batch(self._ctx, int(max_perturbations)))

    def set_profiling(self, stages="all"):
        """Time the named pipeline stages (west_b200.lib.STAGES) with CUDA events;
        "all", or None / [] to switch off."""
        if stages == "all":
            mask = (1 << _lib.NSTAGES) - 1
        else:
            mask = 0
            for name in stages or ():
                mask |= 1 << _lib.STAGES.index(name)
        _lib.check(self._lib.wb_set_profiling(self._ctx, mask))

    def set_graphs(self, enable: bool = True):
        """Run each batch's PCG loop from one CUDA graph launch and each Davidson
        iteration's dense steps from two cached graphs (default), or both eagerly."""
        _lib.check(self._lib.wb_set_graphs(self._ctx, int(bool(enable))))

    def set_autotune(self, enable: bool = True):
        """Tune launch shapes on the first batch of each form (default) or keep the built-in ones."""
        _lib.check(self._lib.wb_set_autotune(self._ctx, int(bool(enable))))

    def set_davidson_apply(self, fn):
        """Operator hook of davidson() (wb_davidson_set_apply): a lib.WB_APPLY_FN, or
        None for the library's own apply_operator.  See distribute.ShardedDavidsonApply."""
        self._dav_hook = fn
        _lib.check(self._lib.wb_davidson_set_apply(self._ctx, fn if fn is not None else _lib.WB_APPLY_FN(), None))

    def tuning(self) -> dict:
        """Launch shapes the autotuner chose (wb_get_tuning)."""
        t = _lib.WbTuning()
        _lib.check(self._lib.wb_get_tuning(self._ctx, ctypes.byref(t)))
        return {k: getattr(t, k) for k, _ in t._fields_}

    def stats(self) -> dict:
        st = _lib.WbStats()
        _lib.check(self._lib.wb_get_stats(self._ctx, ctypes.byref(st)))
        out = {k: getattr(st, k) for k, _ in st._fields_ if not k.startswith("stage_")}
        out["stages"] = {name: {"ms": st.stage_ms[i], "launches": st.stage_launches[i],
                                "items": st.stage_items[i]} for i, name in enumerate(_lib.STAGES)}
        return out

    def apply_operator(self, m, dvg, dng, tr2, iq=1):
        """dng <- sqvc chi0 sqvc dvg for m columns; returns ierr[m]."""
        ierr = np.zeros(max(m, 1), dtype=np.int32)
        if _is_torch_cuda(dvg):
            ld_in = int(dvg.shape[1]); ld_out = int(dng.shape[1])
            rc = self._lib.wb_apply_operator_device(self._ctx, m, dvg.data_ptr(), ld_in, dng.data_ptr(), ld_out,
                                                    float(tr2), int(iq), _ptr(ierr))
        else:
            if not (isinstance(dng, np.ndarray) and dng.dtype == np.complex128 and dng.flags.f_contiguous):
                raise TypeError("dng must be a Fortran-ordered complex128 array")
            dvg_f = np.asfortranarray(dvg, dtype=np.complex128)
            if dvg_f.ndim != 2 or dvg_f.shape[1] < m or dng.shape[1] < m:
                raise ValueError("dvg/dng must be [npwqx, >= m]")
            rc = self._lib.wb_apply_operator(self._ctx, m, _ptr(dvg_f), dvg_f.shape[0], _ptr(dng), dng.shape[0],
                                             float(tr2), int(iq), _ptr(ierr))
        _lib.check(rc)
        ierr = ierr[:m]
        if self.verbose:
            for ipert in np.flatnonzero(ierr):
                sys.stdout.write(f"       ** WARNING : PERT {ipert + 1:8d} iks {1:8d} not converged, "
                                 f"ierr = {ierr[ipert]:8d}\n")
        return ierr


    def davidson(self, dvg0, n_pdep_eigen, n_pdep_times=4, n_pdep_maxiter=100, tr2_dfpt=1e-16,
                 trev_pdep=1e-3, trev_pdep_rel=1e-1, restart_dir=None, n_steps_write_restart=0,
                 restart=False):
        """PDEP Davidson (davidson_diago_gamma, Wstat/davidson_diago.f90:31) from the
        starting basis dvg0 [npwqx, >= n_pdep_eigen] (do_randomize's output).
        With restart_dir, writes WEST's restart files every n_steps_write_restart
        iterations (davidson_restart.f90) and, with restart=True (wstat_calculation
        'R'), resumes from them (dvg0 may then be None).
        Returns (ev, conv, pdep eigenvectors [npwqx, n_pdep_eigen], info dict)."""
        nvec = int(n_pdep_eigen)
        rdir = None if restart_dir is None else os.fsencode(restart_dir)
        prm = _lib.WbDavidsonParams(nvec, nvec * int(n_pdep_times), int(n_pdep_maxiter), float(tr2_dfpt),
                                    float(trev_pdep), float(trev_pdep_rel), int(n_steps_write_restart),
                                    int(bool(restart)), rdir)
        if dvg0 is None:
            d0, ld0, npwx = None, 0, int(self.system.npw)
        else:
            d0 = np.asfortranarray(dvg0[:, :nvec], dtype=np.complex128)
            ld0, npwx = d0.shape[0], d0.shape[0]
        ev = np.zeros(nvec)
        conv = np.zeros(nvec, dtype=np.int32)
        vec = np.zeros((npwx, nvec), dtype=np.complex128, order="F")
        info = _lib.WbDavidsonInfo()
        _lib.check(self._lib.wb_davidson(self._ctx, ctypes.byref(prm), None if d0 is None else _ptr(d0), ld0,
                                         _ptr(ev), _ptr(conv), _ptr(vec), vec.shape[0], ctypes.byref(info)))
        if self.verbose and not info.converged:
            sys.stdout.write(f"     WARNING : {info.notcnv:5d} eigenvalues not converged in chidiago\n")
        return ev, conv.astype(bool), vec, {k: getattr(info, k) for k, _ in info._fields_}


def diagox(op, hr, nbase, nvec):
    """diagox_dsy (Wstat/wstat_tools.f90:48) through wb_diagox: the nvec lowest
    eigenpairs of the symmetric hr[:nbase, :nbase] (upper triangle read).  hr is
    a float64 CUDA tensor holding the column-major [ldh, nbase] array as a
    row-major [nbase, ldh] tensor.  Returns (ew numpy [nvec], vr CUDA tensor
    [nvec, ldv]: row k is eigenvector k)."""
    import torch
    ldh = int(hr.shape[1])
    vr = torch.zeros((nvec, nbase), dtype=torch.float64, device=hr.device)
    ew = np.zeros(nvec)
    _lib.check(op._lib.wb_diagox(op._ctx, int(nbase), int(nvec), hr.data_ptr(), ldh, _ptr(ew), vr.data_ptr(), nbase))
    return ew, vr


def apply_operator_multi(ops, dvgs, dngs, tr2, iq=1):
    """Several ground states in one call (wb_apply_operator_multi): ops[i] maps
    dvgs[i] [npwqx_i, m_i] to dngs[i]; the systems run concurrently on one GPU.
    All arrays are host numpy (Fortran complex128) or all torch CUDA tensors
    ([m_i, npwqx_i]).  Returns the list of ierr arrays."""
    n = len(ops)
    if not (len(dvgs) == len(dngs) == n):
        raise ValueError("ops, dvgs and dngs must have the same length")
    lib = ops[0]._lib
    on_device = n > 0 and _is_torch_cuda(dvgs[0])
    keep, ierrs = [], []
    ms, lds_in, lds_out, pin, pout = [], [], [], [], []
    for op, dvg, dng in zip(ops, dvgs, dngs):
        if on_device:
            m = int(dvg.shape[0])
            ms.append(m); lds_in.append(int(dvg.shape[1])); lds_out.append(int(dng.shape[1]))
            pin.append(dvg.data_ptr()); pout.append(dng.data_ptr())
        else:
            if not (isinstance(dng, np.ndarray) and dng.dtype == np.complex128 and dng.flags.f_contiguous):
                raise TypeError("dng must be a Fortran-ordered complex128 array")
            d = np.asfortranarray(dvg, dtype=np.complex128)
            keep.append(d)
            ms.append(int(d.shape[1])); lds_in.append(d.shape[0]); lds_out.append(dng.shape[0])
            pin.append(_ptr(d)); pout.append(_ptr(dng))
        ierrs.append(np.zeros(max(ms[-1], 1), dtype=np.int32))
    P = ctypes.c_void_p * max(n, 1)
    I = ctypes.c_int * max(n, 1)
    ctxs = P(*[op._ctx.value for op in ops])
    perr = P(*[_ptr(e) for e in ierrs])
    rc = lib.wb_apply_operator_multi(n, ctxs, I(*ms), P(*pin), I(*lds_in), P(*pout), I(*lds_out), float(tr2), int(iq),
                                     perr, int(on_device))
    _lib.check(rc)
    return [e[:m] for e, m in zip(ierrs, ms)]


def _is_torch_cuda(x) -> bool:
    return type(x).__module__.startswith("torch") and getattr(x, "is_cuda", False)
