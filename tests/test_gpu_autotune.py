"""The kernel-form autotuner (tc_b200.autotune) on a small 36^3 BITC system:
it times the candidates, leaves the context on the fastest, and the apply
with the chosen forms -- and with every candidate it timed -- still matches
the oracle."""
import numpy as np
import pytest

from tc_b200 import abi, synth
from tc_b200.autotune import autotune
from tc_b200.context import Context
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


def test_autotune_small_36():
    import torch
    s = synth.small("BITC", nr=(36, 36, 36), nk=2, ecut=4.0, nbands=3, nocc=2, seed=9)
    r2, r3 = O.apply(s, abi.TERMS_TC)
    psi = torch.from_numpy(s.psi.view(np.float64)).cuda()
    h2 = torch.zeros_like(psi)
    h3 = torch.zeros_like(psi)
    knobs = (("fuse", (1, 0)), ("xy", (0, 1, 3)), ("z", (0, 2, 4)), ("min_targets", (0, 8)))
    with Context(s, "mixed") as ctx:
        ctx.set_state()
        default = ctx.forms()
        best, trials = autotune(ctx, abi.TERMS_TC, psi.data_ptr(), h2.data_ptr(), h3.data_ptr(), knobs=knobs)
        assert ctx.forms() == best
        assert trials[0][0] == default and all(ms > 0 for _, ms in trials)
        assert len(trials) >= 5
        for forms, _ in trials[:6]:
            ctx.set_forms(**forms)
            g2, g3 = ctx.apply(abi.TERMS_TC)
            assert rel(g2, r2) < 2e-5, forms
            assert rel(g3, r3) < 2e-5, forms


def test_forms_round_trip_and_rejection():
    from tc_b200 import TCError
    s = synth.small("TC", nr=(12, 12, 12), nk=1, ecut=2.0, nbands=2, nocc=1)
    with Context(s, "mixed") as ctx:
        f = ctx.forms()
        ctx.set_forms(xy=1, z=2, prefetch=0)
        assert ctx.forms() == dict(f, xy=1, z=2, prefetch=0)
        with pytest.raises(TCError) as e:
            ctx.set_forms(xy=3)          # six threads per line exist for 36^3 only
        assert e.value.code == abi.TCG_ERR_UNSUPPORTED
        with pytest.raises(TCError):
            ctx.set_forms(z=9)
