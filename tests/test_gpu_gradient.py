"""The backward pass on the GPU (tcg_energy_grad) against central finite
differences (h = 1e-5) of the GPU's own FP64 energy.

- Orbitals: dE / d conj(chi_i)(G) for a BITC system of 8 irreducible k-points,
  all terms, with the density recomputed (tcg_density) from the perturbed
  orbitals.  E depends on chi only through conj(chi): d/dRe = dE/d conj(chi),
  d/dIm = -i dE/d conj(chi).
- Jastrow tables (Gamma only): the tc2x parts dE2/du(G) and dE2/dV_2body(G),
  contracted with the derivatives of the RPA forms u(G), V_2body(G) with
  respect to A and F (complex-step derivatives of the formulas of
  jastrow_functions.cpp:6-97), against finite differences of E2 in A and F.
"""
import copy

import numpy as np
import pytest

from tc_b200 import abi, synth
from tc_b200.context import Context

pytestmark = pytest.mark.gpu
H = 1e-5


def energy(s, mask):
    with Context(s, "fp64") as ctx:
        s.density = ctx.density()
        ctx.set_state()
        e2, e3, _, _ = ctx.energy_grad(mask)
    return e2 + e3


def test_orbital_gradient_fd():
    import torch
    s = synth.small("BITC", nk=2, nr=(12, 12, 12), ecut=2.0, nbands=2, nocc=2, seed=51)
    mask = abi.TERMS_TC
    with Context(s, "fp64") as ctx:
        s.density = ctx.density()
        ctx.set_state()
        buf = torch.zeros(s.phik_left.size * 2, dtype=torch.float64, device="cuda")
        ctx.energy_grad(mask, dchi_ptr=buf.data_ptr())
        torch.cuda.synchronize()
        grad = buf.cpu().numpy().view(np.complex128)
    off, _ = s._band_offsets(np.full((s.nspin, s.nk_irr), int(s.nbands[0])))
    rng = np.random.default_rng(5)
    for k, b in ((0, 0), (3, 1), (7, 0)):
        for g in rng.choice(int(s.npw[k]), size=2, replace=False):
            o = off[(0, k)] + b * int(s.npw[k]) + g
            vals = []
            for d in (H, -H, 1j * H, -1j * H):
                t = copy.copy(s)
                t.phik_left = s.phik_left.copy()
                t.phik_left[o] += d
                vals.append(energy(t, mask))
            fd_re = (vals[0] - vals[1]) / (2 * H)
            fd_im = (vals[2] - vals[3]) / (2 * H)
            scale = max(1e-3, abs(grad[o]))
            assert abs(fd_re - grad[o]) <= 1e-6 * scale, (k, b, g, fd_re, grad[o])
            assert abs(1j * fd_im - grad[o]) <= 1e-6 * scale, (k, b, g, fd_im, grad[o])


def _rpa_tables(s, A, F):
    """u(G), V_2body(G) of one channel on the FFT grid (G of a Gamma-only system)"""
    n = np.array(s.nr)
    x = np.arange(s.N)
    w = np.stack([x % n[0], (x // n[0]) % n[1], x // (n[0] * n[1])], 1)
    m = np.where(w > n // 2, w - n, w)
    G = m @ np.asarray(s.recip)
    G2 = np.sum(G * G, axis=1).astype(complex)
    G1 = np.sqrt(G2)
    z = G2 < 1e-12
    Gs2 = np.where(z, 1.0, G2)
    Gs1 = np.where(z, 1.0, G1)
    u = np.where(z, -4 * np.pi * A * F * F, 4 * np.pi * A / (Gs2 * (Gs2 * F * F + 1)))
    F2G2 = F * F * Gs2
    v2 = (4 * np.pi / Gs2 - 4 * np.pi * A / (1 + F2G2) + (np.pi * A * A / (F * F) / Gs1)
          * (np.pi * F2G2 + (4 + 2 * F2G2) * np.arctan(F * Gs1 / 2) - (4 + 4 * F2G2) * np.arctan(F * Gs1)))
    v2 = np.where(z, -2 * np.pi * A * A / F, v2)
    return u, v2


def test_jastrow_table_gradient_fd():
    A0, F0 = 0.6, 1.1
    base = synth.small("BITC", nk=1, nr=(16, 16, 16), ecut=3.0, nbands=3, nocc=3, seed=52, A=A0, F=F0)
    mask = abi.TERM_TC2X
    with Context(base, "fp64") as ctx:
        ctx.set_state()
        _, _, du, dv = ctx.energy_grad(mask, tables=True)
    h = 1e-7
    for which in ("A", "F"):
        ua, va = _rpa_tables(base, A0 + (1j * h if which == "A" else 0), F0 + (1j * h if which == "F" else 0))
        du_dp, dv_dp = ua.imag / h, va.imag / h
        pred = np.sum(du[0] * du_dp) + np.sum(dv[0] * dv_dp)
        vals = []
        for d in (H, -H):
            s = copy.copy(base)
            Aa = np.full((2, 2), A0 + (d if which == "A" else 0.0))
            Fa = np.full((2, 2), F0 + (d if which == "F" else 0.0))
            s.jastrow_A, s.jastrow_F = Aa, Fa
            with Context(s, "fp64") as ctx:
                ctx.set_state()
                e2, _, _, _ = ctx.energy_grad(mask)
            vals.append(e2)
        fd = (vals[0] - vals[1]) / (2 * H)
        print(f"d E2 / d {which}: adjoint {pred:.10e}, finite difference {fd:.10e}")
        assert abs(fd - pred) <= 1e-6 * max(abs(pred), 1e-6)


def test_c4_gradients_fd():
    """The adjoint at the homogeneous-electron-gas configuration C4 in full
    (simple cubic, 54 electrons at r_s = 2, Gamma only, 27 occupied + 27 trial
    bands, grid 40^3, TC++'s default RPA Jastrow): dE/d conj(chi) of all
    terms along a seeded random direction of every occupied left orbital,
    and the tc2x Jastrow-table gradient contracted with d u / d A, d V_2body /
    d A, against central finite differences (h = 1e-5) of the FP64 energy."""
    import torch
    s = synth.heg_config()
    mask = abi.TERMS_TC
    with Context(s, "fp64") as ctx:
        s.density = ctx.density()
        ctx.set_state()
        buf = torch.zeros(s.phik_left.size * 2, dtype=torch.float64, device="cuda")
        ctx.energy_grad(mask, dchi_ptr=buf.data_ptr())
        torch.cuda.synchronize()
        grad = buf.cpu().numpy().view(np.complex128)
    rng = np.random.default_rng(11)
    delta = rng.standard_normal(grad.shape) + 1j * rng.standard_normal(grad.shape)
    nb, no, npw = int(s.nbands[0]), int(s.nocc[0][0]), int(s.npw[0])
    delta.reshape(nb, npw)[no:] = 0.0                  # occupied orbitals only
    vals = []
    for d in (H, -H):
        t = copy.copy(s)
        t.phik_left = s.phik_left + d * delta
        vals.append(energy(t, mask))
    fd = (vals[0] - vals[1]) / (2 * H)
    pred = np.sum(grad * np.conj(delta))
    print(f"C4 d E / d h along a random direction: adjoint {pred:.10e}, finite difference {fd:.10e}")
    assert abs(fd - pred) <= 1e-6 * abs(pred)

    A0, F0 = s.jastrow_A[0, 0], s.jastrow_F[0, 0]
    with Context(s, "fp64") as ctx:
        ctx.set_state()
        _, _, du, dv = ctx.energy_grad(abi.TERM_TC2X, tables=True)
    h = 1e-7
    ua, va = _rpa_tables(s, A0 + 1j * h, F0)
    pred = np.sum(du[0] * ua.imag / h) + np.sum(dv[0] * va.imag / h)
    vals = []
    for d in (H, -H):
        t = copy.copy(s)
        t.jastrow_A = s.jastrow_A + d                  # tc2x reads the same-spin channel only
        with Context(t, "fp64") as ctx:
            ctx.set_state()
            e2, _, _, _ = ctx.energy_grad(abi.TERM_TC2X)
        vals.append(e2)
    fd = (vals[0] - vals[1]) / (2 * H)
    print(f"C4 d E2 / d A: adjoint {pred:.10e}, finite difference {fd:.10e}")
    assert abs(fd - pred) <= 1e-6 * max(abs(pred), 1e-6)
