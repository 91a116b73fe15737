"""PDEP database files in WEST's format (wstat.save/summary.json and
Q<iq>E<j>.dat), through wb_pdep_db_write / wb_pdep_db_read."""
from __future__ import annotations

import math
import os

import numpy as np

from . import lib as _lib


def cubic_cell(L: float) -> np.ndarray:
    """a1, a2, a3 (bohr) and b1, b2, b3 (bohr^-1, with the 2 pi) of a cubic cell."""
    a = np.eye(3) * L
    b = np.eye(3) * (2.0 * math.pi / L)
    return np.ascontiguousarray(np.concatenate([a, b]).ravel())


def pdep_db_write(save_dir: str, ev, pdep, cell, iq: int = 1, q_cryst=(0.0, 0.0, 0.0)):
    lib = _lib.load()
    os.makedirs(save_dir, exist_ok=True)
    ev = np.ascontiguousarray(ev, dtype=np.float64)
    pdep = np.asfortranarray(pdep, dtype=np.complex128)
    cell = np.ascontiguousarray(cell, dtype=np.float64)
    q = np.ascontiguousarray(q_cryst, dtype=np.float64)
    _lib.check(lib.wb_pdep_db_write(save_dir.encode(), iq, q.ctypes.data, cell.ctypes.data, ev.size,
                                    ev.ctypes.data, pdep.ctypes.data, pdep.shape[0], pdep.shape[0]))


def pdep_db_read(save_dir: str, nglob: int, npw: int, iq: int = 1):
    lib = _lib.load()
    ev = np.zeros(nglob)
    pdep = np.zeros((npw, nglob), dtype=np.complex128, order="F")
    _lib.check(lib.wb_pdep_db_read(save_dir.encode(), iq, nglob, ev.ctypes.data, pdep.ctypes.data, npw, npw))
    return ev, pdep


def read_pdep_vector(fname: str) -> np.ndarray:
    """One file of the pdep format (IO_kernel/pdep_io.f90:35-156): 32 int32 header
    (version 210405, little-endian flag, npw) then npw complex128 coefficients."""
    raw = open(fname, "rb").read()
    hd = np.frombuffer(raw[:128], dtype="<i4")
    if hd[0] != 210405:
        raise ValueError(f"{fname}: unknown header version {hd[0]}")
    npw = int(hd[2])
    return np.frombuffer(raw[128:128 + 16 * npw], dtype="<c16").copy()


def read_davidson_restart(restart_dir: str) -> dict:
    """WEST's Davidson restart files (Wstat/davidson_restart.f90:33-411) as arrays:
    dav_iter, notcnv, nbase, conv, ev, ew from summary.json; hr and vr from
    hr_vr.dat (Fortran unformatted sequential, n_pdep_basis^2 doubles each,
    column-major); dvg and dng [npw, nbase] from V<j>.dat / N<j>.dat."""
    import json
    with open(os.path.join(restart_dir, "summary.json")) as f:
        s = json.load(f)
    nvecx = len(s["ew"])
    raw = open(os.path.join(restart_dir, "hr_vr.dat"), "rb").read()
    mats, off = [], 0
    for _ in range(2):
        n = int(np.frombuffer(raw[off:off + 4], dtype="<i4")[0])
        if n != 8 * nvecx * nvecx:
            raise ValueError("hr_vr.dat record is not n_pdep_basis^2 doubles")
        mats.append(np.frombuffer(raw[off + 4:off + 4 + n], dtype="<f8").reshape(nvecx, nvecx).T.copy())
        if int(np.frombuffer(raw[off + 4 + n:off + 8 + n], dtype="<i4")[0]) != n:
            raise ValueError("hr_vr.dat record markers differ")
        off += n + 8
    nbase = int(s["nbase"])
    dvg = np.stack([read_pdep_vector(os.path.join(restart_dir, f"V{j:06d}.dat")) for j in range(1, nbase + 1)], 1)
    dng = np.stack([read_pdep_vector(os.path.join(restart_dir, f"N{j:06d}.dat")) for j in range(1, nbase + 1)], 1)
    return {"dav_iter": int(s["dav_iter"]), "notcnv": int(s["notcnv"]), "nbase": nbase,
            "conv": np.array(s["conv"], dtype=bool), "ev": np.array(s["ev"]), "ew": np.array(s["ew"]),
            "hr": mats[0], "vr": mats[1], "dvg": dvg, "dng": dng}
