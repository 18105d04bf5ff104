"""Host-side mirror of TC++'s calc_hamiltonian namespace for the operator
terms (src/include/calc_hamiltonian.hpp:54-130): same routine names, the
same nested containers phi[ispin][ik][jband][ispinor] / HXphi[...] with
accumulate ("+=") semantics, computed by the CUDA library.

Differences: the physics objects (CrystalStructure, Kpoints, PlaneWaveBasis,
BlochStates, Potentials, Method) are carried by one Context built from a
TCSystem, and errors raise TCError instead of calling MPI_Abort
(error_messages.cpp:60-64).  Only the first spinor component is used (TC++
asserts !spin.is_spinor() in these routines, e.g. calc_hamiltonian_hf2x.cpp:19).
"""
import numpy as np

from . import abi
from ._lib import TCError


def _flatten(ctx, phi):
    s = ctx.system
    nb = np.array([[len(phi[isp][ik]) for ik in range(s.nk_irr)] for isp in range(s.nspin)], dtype=np.int32)
    parts = []
    for isp in range(s.nspin):
        for ik in range(s.nk_irr):
            for b in phi[isp][ik]:
                v = np.asarray(b[0], dtype=np.complex128)
                if v.shape != (int(s.npw[ik]),):
                    raise TCError(abi.TCG_ERR_ARG, f"band at spin {isp}, k {ik} has {v.shape} coefficients, "
                                                   f"expected {int(s.npw[ik])}")
                parts.append(v)
    flat = np.concatenate(parts) if parts else np.zeros(0, dtype=np.complex128)
    return nb, flat


def _scatter_back(ctx, nb, flat, HX):
    s = ctx.system
    o = 0
    for isp in range(s.nspin):
        for ik in range(s.nk_irr):
            n = int(s.npw[ik])
            for j in range(int(nb[isp][ik])):
                HX[isp][ik][j][0][...] = flat[o:o + n]
                o += n


def _run(ctx, mask, phi, HX, which):
    nb, psi = _flatten(ctx, phi)
    _, cur = _flatten(ctx, HX)
    h2 = cur.copy() if which == 2 else np.zeros_like(psi)
    h3 = cur.copy() if which == 3 else np.zeros_like(psi)
    h2, h3 = ctx.apply(mask, psi=psi, nb_apply=nb, h2=h2, h3=h3)
    _scatter_back(ctx, nb, h2 if which == 2 else h3, HX)


def hf2x(ctx, phi, H2phi):
    """calc_hamiltonian::hf2x (calc_hamiltonian_hf2x.cpp:8)."""
    _run(ctx, abi.TERM_HF2X, phi, H2phi, 2)


def tc2x(ctx, phi, H2phi):
    """calc_hamiltonian::tc2x (calc_hamiltonian_tc2x.cpp:11)."""
    _run(ctx, abi.TERM_TC2X, phi, H2phi, 2)


def tc3a1(ctx, phi, H3phi):
    """calc_hamiltonian::tc3a1 (calc_hamiltonian_tc3a1.cpp:8)."""
    _run(ctx, abi.TERM_TC3A1, phi, H3phi, 3)


def tc3b1(ctx, phi, H3phi):
    """calc_hamiltonian::tc3b1 (calc_hamiltonian_tc3b1.cpp:8)."""
    _run(ctx, abi.TERM_TC3B1, phi, H3phi, 3)


def tc3a2a4b2b5(ctx, phi, H3phi):
    """calc_hamiltonian::tc3a2a4b2b5 (calc_hamiltonian_tc3a2a4b2b5.cpp:11)."""
    _run(ctx, abi.TERM_TC3A2A4B2B5, phi, H3phi, 3)


def tc3a3b3b4b6(ctx, phi, H3phi):
    """calc_hamiltonian::tc3a3b3b4b6 (calc_hamiltonian_tc3a3b3b4b6.cpp:11)."""
    _run(ctx, abi.TERM_TC3A3B3B4B6, phi, H3phi, 3)


def nested(system, flat, nb=None):
    """Packed [spin][k][band][npw] array -> nested phi[ispin][ik][jband][0]."""
    nb = system.nb_apply if nb is None else nb
    out, o = [], 0
    for isp in range(system.nspin):
        ks = []
        for ik in range(system.nk_irr):
            n = int(system.npw[ik])
            bands = []
            for j in range(int(nb[isp][ik])):
                bands.append([np.array(flat[o:o + n])])
                o += n
            ks.append(bands)
        out.append(ks)
    return out
