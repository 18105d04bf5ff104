"""The applied operator is the gradient of the energy functional (oracle, CPU).

TotalEnergy (total_energy.cpp:101-168) defines
    E = sum_{k, isym, i} f_i [e2_i / 2 + e3_i / 3] / N_k,   e_n = <chi_i | H_n phi_i>,
with H_n built from the same occupied orbitals and their density
n = sum f chi* phi (bloch_states_scfloop_filling_density.cpp:256-360).  E is a
polynomial in conj(chi) of degree 2 (two-body) and 3 (three-body); if H2 and
H3 are the mean-field derivatives of E2 and E3, Euler's theorem gives
    dE / d conj(chi_i)(G) = f_i / N_k (H2 + H3) phi_i (G).
This holds for tc2x, tc2h, hf2x and hf2h alone, for tc3a1 + tc3b1 together
and for tc3a2a4b2b5 + tc3a3b3b4b6 together (the reference splits each
three-body derivative over two routines), so a wrong factor or sign in any
term breaks it.  Checked by
central finite differences (h = 1e-5) of the oracle's energy, with the
density recomputed from the perturbed orbitals: E depends on chi only through
conj(chi), so d/dRe chi = dE/d conj(chi) and d/dIm chi = -i dE/d conj(chi).
"""
import copy

import numpy as np
import pytest

from tc_b200 import abi, synth
from oracle import oracle as O

H = 1e-5
GROUPS = {"tc2x": ["tc2x"], "tc2h": ["tc2h"], "tc3a1+tc3b1": ["tc3a1", "tc3b1"],
          "tc3a2a4b2b5+tc3a3b3b4b6": ["tc3a2a4b2b5", "tc3a3b3b4b6"], "hf2x": ["hf2x"], "hf2h": ["hf2h"]}
NAMES = dict(abi.TERM_NAMES, **abi.TERM_NAMES_EXTRA)


def energy(s, mask):
    """E2 + E3 of the occupied orbitals: H applied to the occupied right
    orbitals (psi rebuilt from the current orbitals), density recomputed"""
    s.nb_apply = np.array(s.nocc, dtype=np.int32)
    s.psi = np.concatenate([s.orb(0, k, b) for k in range(s.nk_irr) for b in range(int(s.nocc[0][k]))])
    s.density = O.density(s)
    h2, h3 = O.apply(s, mask)
    e2, e3 = s.energy_terms(h2, h3)
    return e2 + e3, h2, h3


def left_offset(s, k, b, g):
    """offset of coefficient g of band b at k in phik_left / phik"""
    off, _ = s._band_offsets(np.full((s.nspin, s.nk_irr), int(s.nbands[0])))
    return off[(0, k)] + b * int(s.npw[k]) + g


def perturbed(s, field, off, d):
    t = copy.copy(s)
    arr = getattr(s, field).copy()
    arr[off] += d
    setattr(t, field, arr)
    return t


@pytest.mark.parametrize("group", list(GROUPS))
def test_operator_is_energy_gradient(group):
    method = "HF" if group.startswith("hf") else "BITC"
    s = synth.small(method, nk=2, nr=(12, 12, 12), ecut=2.0, nbands=2, nocc=2, seed=7)
    mask = 0
    for t in GROUPS[group]:
        mask |= NAMES[t]
    field = "phik_left" if method == "BITC" else "phik"
    _, h2, h3 = energy(s, mask)
    rng = np.random.default_rng(3)
    for k, b in ((0, 0), (1, 1)):
        for g in rng.choice(int(s.npw[k]), size=3, replace=False):
            pred = s.fill(0, k, b) / s.num_kpoints * (s.band_view(h2, 0, k, b)[g] + s.band_view(h3, 0, k, b)[g])
            off = left_offset(s, k, b, g)
            if method == "HF":
                # chi = phi: E depends on both conj(phi) and phi; d/dRe phi = 2 Re-part rule
                ep, _, _ = energy(perturbed(s, field, off, H), mask)
                em, _, _ = energy(perturbed(s, field, off, -H), mask)
                fd = (ep - em) / (2 * H)
                assert abs(fd - 2 * pred.real) <= 1e-6 * max(1.0, abs(pred))
                continue
            ep, _, _ = energy(perturbed(s, field, off, H), mask)
            em, _, _ = energy(perturbed(s, field, off, -H), mask)
            fd_re = (ep - em) / (2 * H)
            ep, _, _ = energy(perturbed(s, field, off, 1j * H), mask)
            em, _, _ = energy(perturbed(s, field, off, -1j * H), mask)
            fd_im = (ep - em) / (2 * H)
            scale = max(1e-3, abs(pred))
            assert abs(fd_re - pred) <= 1e-6 * scale, (group, k, b, g, fd_re, pred)
            assert abs(1j * fd_im - pred) <= 1e-6 * scale, (group, k, b, g, fd_im, pred)
