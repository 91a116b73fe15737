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
