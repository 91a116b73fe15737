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


def batch_owner_rows(col0: int, m: int, nranks: int, rank: int) -> list:
    """Rows (0-based within the batch) of the basis columns col0 .. col0+m-1 that
    rank owns under the cyclic rule of pert%l2g (global column j -> rank j % nranks)."""
    return [i for i in range(m) if (col0 + i) % nranks == rank]


def gather_batch(local, col0: int, m: int, nranks: int, rank: int, group=None):
    """All-gather of a sharded batch: local [nloc, n] holds this rank's rows of the
    m-row batch (batch_owner_rows order); returns the whole batch [m, n] on every
    rank.  One all_gather_into_tensor (NCCL on GPUs, gloo on CPU) over rows padded
    to ceil(m / nranks)."""
    import torch
    import torch.distributed as dist
    maxloc = (m + nranks - 1) // nranks
    n = local.shape[1]
    cplx = local.is_complex()
    send = torch.zeros((maxloc, n), dtype=local.dtype, device=local.device)
    send[: local.shape[0]] = local
    if cplx:  # exchanged as real pairs
        send = torch.view_as_real(send)
    if local.is_cuda and dist.get_backend(group) == "nccl":
        recv = torch.empty((nranks * maxloc,) + tuple(send.shape[1:]), dtype=send.dtype, device=send.device)
        dist.all_gather_into_tensor(recv, send, group=group)
    else:  # gloo: through host memory
        host = send.cpu()
        parts = [torch.empty_like(host) for _ in range(nranks)]
        dist.all_gather(parts, host, group=group)
        recv = torch.cat(parts, 0).to(send.device)
    if cplx:
        recv = torch.view_as_complex(recv)
    out = torch.empty((m, n), dtype=local.dtype, device=local.device)
    for q in range(nranks):
        rows = batch_owner_rows(col0, m, nranks, q)
        if rows:
            out[rows] = recv[q * maxloc: q * maxloc + len(rows)]
    return out


class _CudaBuffer:
    """A device pointer seen as a [rows, ld] complex128 array (CUDA array interface)."""

    def __init__(self, ptr: int, rows: int, ld: int):
        self.__cuda_array_interface__ = {"shape": (rows, ld), "typestr": "<c16", "data": (ptr, False),
                                         "strides": None, "version": 3}


class ShardedDavidsonApply:
    """Operator hook of the PDEP Davidson for several GPUs (wb_davidson_set_apply):
    every rank runs the same Davidson on the same starting basis; for each batch of
    new basis vectors a rank applies the operator to the columns it owns (WEST's
    cyclic pert distribution) and one all-gather of the dng rows gives every rank
    the whole batch, so the small dense steps (build_hr, diagox, MGS, updates) run
    redundantly and identically everywhere.  The autotuner is switched off so all
    ranks use the same launch shapes (identical rounding keeps the ranks' bases,
    convergence flags and batch sizes in lock step); a (col0, m) check before each
    exchange turns a divergence into an error instead of a mismatched collective."""

    def __init__(self, op, group=None):
        import torch.distributed as dist
        from . import lib as _lib
        self.op, self.group = op, group
        self.rank = dist.get_rank(group)
        self.nranks = dist.get_world_size(group)
        self.calls = 0
        self.error = None
        op.set_autotune(False)
        self._fn = _lib.WB_APPLY_FN(self._hook)          # keep the ctypes thunk alive

    def _hook(self, user, col0, m, dvg_ptr, dng_ptr, ld, tr2):
        try:
            self.apply(col0, m, dvg_ptr, dng_ptr, ld, tr2)
            return 0
        except Exception as e:  # reported by wb_davidson as a failed call (WB_ERR_ARG)
            self.error = e
            return -1

    def apply(self, col0, m, dvg_ptr, dng_ptr, ld, tr2):
        import torch
        import torch.distributed as dist
        x = torch.as_tensor(_CudaBuffer(dvg_ptr, m, ld), device="cuda")
        y = torch.as_tensor(_CudaBuffer(dng_ptr, m, ld), device="cuda")
        dev = "cuda" if dist.get_backend(self.group) == "nccl" else "cpu"
        chk = torch.tensor([col0, m, -col0, -m], dtype=torch.int64, device=dev)
        dist.all_reduce(chk, op=dist.ReduceOp.MAX, group=self.group)
        if int(chk[0]) != col0 or int(chk[1]) != m or -int(chk[2]) != col0 or -int(chk[3]) != m:
            raise RuntimeError(f"ranks diverged: batch ({col0}, {m}) on rank {self.rank}")
        rows = batch_owner_rows(col0, m, self.nranks, self.rank)
        local = torch.zeros((len(rows), ld), dtype=torch.complex128, device="cuda")
        if rows:
            xl = x[rows].contiguous()
            self.op.apply_operator(len(rows), xl, local, tr2)
        y.copy_(gather_batch(local, col0, m, self.nranks, self.rank, self.group))
        torch.cuda.synchronize()
        self.calls += 1

    def install(self):
        self.op.set_davidson_apply(self._fn)
        return self

    def remove(self):
        self.op.set_davidson_apply(None)
