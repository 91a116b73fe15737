"""Perturbation distribution over GPUs, as WEST distributes it over images.

WEST's Davidson hands each image the perturbation columns of a cyclic
``idistribute`` (Para_kernel/class_idistribute.f90: nloc/nlocx :76-111,
cyclic g2l :183-186, l2g) and each image calls ``apply_operator`` on its own
columns with no communication inside the call (davidson_diago.f90:97-98,
:186-196).  One process per GPU plays the role of one image here.
"""
from __future__ import annotations

import numpy as np


class PertDistribution:
    """Cyclic distribution of ``nglob`` columns over ``nlevel`` ranks (0-based)."""

    def __init__(self, nglob: int, nlevel: int, rank: int):
        if nlevel < 1 or not 0 <= rank < nlevel:
            raise ValueError("need 0 <= rank < nlevel")
        self.nglob, self.nlevel, self.rank = nglob, nlevel, rank
        self.nloc = nglob // nlevel + (1 if rank < nglob % nlevel else 0)      # :79-88
        self.nlocx = nglob // nlevel + (1 if nglob % nlevel else 0)

    def l2g(self, iloc: int, rank: int | None = None) -> int:
        """Global column of local column iloc."""
        r = self.rank if rank is None else rank
        return self.nlevel * iloc + r

    def g2l(self, iglob: int):
        """(local column, owning rank) of global column iglob (:183-186)."""
        return iglob // self.nlevel, iglob % self.nlevel

    def local_columns(self, rank: int | None = None) -> np.ndarray:
        r = self.rank if rank is None else rank
        n = self.nglob // self.nlevel + (1 if r < self.nglob % self.nlevel else 0)
        return self.nlevel * np.arange(n) + r


def apply_operator_sharded(apply, dvg, tr2, dist: PertDistribution):
    """Apply ``apply(dvg_local, tr2) -> (dng_local, ierr_local)`` to this rank's
    columns of ``dvg`` [npw, nglob]; returns (dng_local, ierr_local, columns)."""
    cols = dist.local_columns()
    dng, ierr = apply(np.asfortranarray(dvg[:, cols]), tr2)
    return dng, ierr, cols
