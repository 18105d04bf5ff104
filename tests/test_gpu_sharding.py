"""The occupied-pair stage of tc3a2a4b2b5 split over ranks, on one GPU.

Each "rank" is its own context on the same device; the ranks run one after
the other (nothing waits on another rank), and their partial buffers are
summed with torch in place of the NCCL all_reduce that tc_b200.sharding
issues on several GPUs.  After tcg_qp_finish every rank's apply must equal the
unsharded apply."""
import numpy as np
import pytest

from tc_b200 import abi, synth
from tc_b200.context import Context
from tc_b200.sharding import device_view

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-12), ("mixed", 2e-5)])
@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("case", ["BITC", "TC-tr"])
def test_split_stage_equals_whole(case, world, prec, tol):
    import torch
    if case == "BITC":
        s = synth.small("BITC", nk=2, nbands=3, nocc=2, seed=21)
    else:
        s = synth.small("TC", tr=True, nr=(16, 16, 16), ecut=1.5, nbands=2, nocc=1, seed=22)
    mask = abi.TERMS_TC
    with Context(s, prec) as ref_ctx:
        ref_ctx.set_state()
        r2, r3 = ref_ctx.apply(mask)
    dev = torch.device("cuda", 0)
    ctxs = [Context(s, prec) for _ in range(world)]
    try:
        views = []
        for r, ctx in enumerate(ctxs):
            ctx.set_state()
            ptr, nbytes = ctx.qp_partial(r, world)
            views.append(device_view(ptr, nbytes, dev))
        torch.cuda.synchronize()
        total = torch.stack(views).sum(0)
        for v in views:
            v.copy_(total)
        torch.cuda.synchronize()
        for ctx in ctxs:
            ctx.qp_finish()
            g2, g3 = ctx.apply(mask)
            assert rel(g2, r2) < tol
            assert rel(g3, r3) < tol
    finally:
        for ctx in ctxs:
            ctx.close()


def test_apply_between_partial_and_finish_is_refused():
    from tc_b200 import TCError
    s = synth.small("TC", nk=2, seed=23)
    with Context(s, "fp64") as ctx:
        ctx.set_state()
        ctx.qp_partial(0, 2)
        with pytest.raises(TCError) as e:
            ctx.apply(abi.TERMS_TC)
        assert e.value.code == abi.TCG_ERR_STATE
        with pytest.raises(TCError):
            ctx.qp_partial(2, 2)           # rank outside [0, nranks)
