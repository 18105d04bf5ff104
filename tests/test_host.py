"""Host-side logic: the reference-shaped nested containers of the
calc_hamiltonian mirror, band packing and ownership flags."""
import numpy as np
import pytest

from tc_b200 import synth
from tc_b200 import calc_hamiltonian as CH


class FakeCtx:
    """records what the mirror passes to Context.apply"""
    def __init__(self, system):
        self.system = system
        self.calls = []

    def apply(self, mask, psi=None, nb_apply=None, h2=None, h3=None):
        self.calls.append((mask, psi.copy(), nb_apply.copy()))
        h2 = h2 + 1.0 * psi
        h3 = h3 + 2.0 * psi
        return h2, h3


def test_nested_roundtrip_and_accumulate():
    s = synth.small("TC")
    phi = CH.nested(s, s.psi)
    assert len(phi) == s.nspin and len(phi[0]) == s.nk_irr and len(phi[0][0]) == int(s.nb_apply[0][0])
    H2 = CH.nested(s, np.ones_like(s.psi))
    ctx = FakeCtx(s)
    CH.tc2x(ctx, phi, H2)
    mask, psi, nb = ctx.calls[0]
    assert np.array_equal(psi, s.psi)
    assert np.array_equal(nb, s.nb_apply)
    # H2 += 1 * psi on top of the previous content (accumulate semantics)
    assert np.allclose(H2[0][1][2][0], 1.0 + s.band_view(s.psi, 0, 1, 2))
    H3 = CH.nested(s, np.zeros_like(s.psi))
    CH.tc3a1(ctx, phi, H3)
    assert np.allclose(H3[0][0][0][0], 2.0 * s.band_view(s.psi, 0, 0, 0))


def test_wrong_band_length_rejected():
    from tc_b200 import TCError
    s = synth.small("HF")
    phi = CH.nested(s, s.psi)
    phi[0][1][0][0] = phi[0][1][0][0][:-1]
    with pytest.raises(TCError):
        CH.hf2x(FakeCtx(s), phi, CH.nested(s, np.zeros_like(s.psi)))


def test_psi_offsets_cover_packed_array():
    s = synth.small("BITC", nspin=2)
    off, total = s.psi_offsets()
    assert total == s.psi.size
    assert off[(1, 0)] == s.psi.size // 2
