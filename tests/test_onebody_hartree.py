"""Oracle restatements of the Hartree-type and one-body terms against an
independent numpy restatement (numpy FFTs, vectorised):
  hf2h     calc_hamiltonian_hf2h.cpp:7-85     V_H = 4 pi n(G) / G^2, G != 0
  kinetic  calc_hamiltonian_kinetic.cpp:6-52  1/2 |k+G|^2
  pseudo   calc_hamiltonian_pseudo.cpp:6-180  D_ij <beta_j|phi> beta_i (per atom, m)
                                              + V_loc(r) phi(r)
(tc2h is pinned by the energy-gradient identity in tests/test_gradient.py.)"""
import numpy as np

from tc_b200 import abi, synth
from oracle import oracle as O


def rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


def to_r(s, coef, gi):
    n0, n1, n2 = s.nr
    g = np.zeros(s.N, dtype=np.complex128)
    g[gi] = coef
    return (np.fft.ifftn(g.reshape(n2, n1, n0)) * s.N).ravel()


def to_g(s, r):
    n0, n1, n2 = s.nr
    return (np.fft.fftn(r.reshape(n2, n1, n0)) / s.N).ravel()


def gvecs(s):
    n = np.array(s.nr)
    x = np.arange(s.N)
    w = np.stack([x % n[0], (x // n[0]) % n[1], x // (n[0] * n[1])], 1)
    m = np.where(w > n // 2, w - n, w)
    return m @ np.asarray(s.recip)


def test_kinetic_and_pseudo_vs_numpy():
    s = synth.small("TC", nk=2, seed=41)
    pp = synth.pseudo(s, seed=42)
    h1 = O.apply_h1(s, abi.TERMS_H1, pp)
    G = gvecs(s)
    ref = np.zeros_like(s.psi)
    ncomp = sum(2 * l + 1 for l in pp.lbeta[0])
    koff = 0
    for k in range(s.nk_irr):
        gi, _ = s.gidx(0, int(s.kall_off[k]))
        npw = int(s.npw[k])
        kc = np.asarray(s.kvec[int(s.kall_off[k])]) @ np.asarray(s.recip)
        proj = pp.projector[koff:koff + ncomp * npw].reshape(ncomp, npw)
        koff += ncomp * npw
        for b in range(int(s.nb_apply[0][k])):
            psi = s.band_view(s.psi, 0, k, b)
            out = s.band_view(ref, 0, k, b)
            out += 0.5 * np.sum((kc + G[gi]) ** 2, axis=1) * psi
            for ia, R in enumerate(pp.atom_pos):
                ph = np.exp(1j * G[gi] @ R)
                comps, c0 = [], 0
                for l in pp.lbeta[0]:
                    comps.append(list(range(c0, c0 + 2 * l + 1)))
                    c0 += 2 * l + 1
                D = pp.dij[0]
                for jp, cj in enumerate(comps):
                    for m, c in enumerate(cj):
                        coeff = np.sum(ph * proj[c] * psi)
                        for ip, ci in enumerate(comps):
                            if abs(D[ip, jp]) > 1e-8:
                                out += D[ip, jp] * coeff * np.conj(ph * proj[ci[m]])
            out += to_g(s, pp.vloc * to_r(s, psi, gi))[gi]
    assert rel(h1, ref) < 1e-12


def test_hf2h_vs_numpy():
    s = synth.small("HF", nk=2, seed=43)
    h2, _ = O.apply(s, abi.TERM_HF2H)
    G = gvecs(s)
    nG = to_g(s, s.density[0] + s.density[1])
    g2 = np.sum(G ** 2, axis=1)
    VG = np.where(g2 > 0, 4 * np.pi * nG / np.where(g2 > 0, g2, 1.0), 0.0)
    VG[0] = 0.0
    Vr = (np.fft.ifftn(VG.reshape(s.nr[2], s.nr[1], s.nr[0])) * s.N).ravel()
    f = 1.0 / (s.num_kpoints * s.omega)
    ref = np.zeros_like(s.psi)
    for k in range(s.nk_irr):
        gi, _ = s.gidx(0, int(s.kall_off[k]))
        for b in range(int(s.nb_apply[0][k])):
            out = s.band_view(ref, 0, k, b)
            out += f * to_g(s, Vr * to_r(s, s.band_view(s.psi, 0, k, b), gi))[gi]
    assert rel(h2, ref) < 1e-12
