"""The perturbation-sharded Davidson apply (wb_davidson_set_apply +
distribute.ShardedDavidsonApply) on one GPU: an NCCL process group of one rank
runs the same exchange as a multi-GPU job, and the Davidson through the hook
gives the built-in path's eigenvalues.  The split and the all-gather of a batch
over two ranks are tested with gloo on CPU (tests/test_distribute.py)."""
import datetime
import socket

import numpy as np
import pytest

from west_b200.system import randomized_basis

pytestmark = pytest.mark.gpu

KW = dict(n_pdep_times=4, n_pdep_maxiter=100, tr2_dfpt=1e-12, trev_pdep=1e-6, trev_pdep_rel=1e-1)


@pytest.fixture
def nccl_group():
    import torch.distributed as dist
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    yield
    dist.destroy_process_group()


def test_sharded_hook_matches_builtin_apply(small, nccl_group):
    from west_b200.distribute import ShardedDavidsonApply
    from west_b200.wstat import ResponseOperator
    dvg0 = randomized_basis(small, 4)
    a = ResponseOperator(small, verbose=False)
    a.set_autotune(False)
    ev_a, conv_a, vec_a, info_a = a.davidson(dvg0, 4, **KW)
    b = ResponseOperator(small, verbose=False)
    hook = ShardedDavidsonApply(b).install()
    ev_b, conv_b, vec_b, info_b = b.davidson(dvg0, 4, **KW)
    hook.remove()
    assert hook.calls == info_b["apply_calls"] == info_a["apply_calls"]
    assert info_b["dav_iter"] == info_a["dav_iter"] and (conv_a == conv_b).all()
    assert np.abs((ev_b - ev_a) / ev_a).max() < 1e-12


def test_failing_hook_is_reported(small):
    from west_b200.lib import WB_APPLY_FN, WestB200Error
    from west_b200.wstat import ResponseOperator
    op = ResponseOperator(small, verbose=False)
    fn = WB_APPLY_FN(lambda user, col0, m, x, y, ld, tr2: -1)
    op.set_davidson_apply(fn)
    with pytest.raises(WestB200Error, match="hook"):
        op.davidson(randomized_basis(small, 4), 4, **KW)
    op.set_davidson_apply(None)
    ev, conv, vec, info = op.davidson(randomized_basis(small, 4), 4, **KW)
    assert info["converged"] == 1
