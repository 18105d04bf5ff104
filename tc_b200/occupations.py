"""Band occupations of an SCF iteration as TC++ sets them
(BlochStates::set_filling, bloch_states_scfloop_filling_density.cpp:8-200,
with Kpoints::return_band_filling, kpoints.cpp:349-387).

  fixed     the round(nelec / 2) lowest bands of every k with non-zero weight
            hold spin_factor electrons (2 unpolarised, 1 per spin channel)
  gaussian  f = spin_factor (1 - erf((e - E_F) / width)) / 2, with E_F found by
            60 bisection steps in [-1e5, 1e5] Ha on the electron count
            sum_{s,k,b} f w_k / spin_factor (w_k: the k-point weights of the
            QE run, summing to spin_factor)

Eigenvalues are given per spin and irreducible k in the order TC++ holds
them (sorted by the real part after each Davidson call); only their real
parts enter.
"""
import math

import numpy as np


def fermi_filling(eig, kweight, nelec, nspin, smearing="fixed", width=0.01):
    """(filling [nspin][nk][nb], fermi_energy) for eigenvalues eig
    [nspin][nk][nb] (real or complex), weights kweight [nk]."""
    e = np.real(np.asarray(eig))
    ns, nk, nb = e.shape
    spin_factor = 2.0 if nspin == 1 else 1.0
    w = np.asarray(kweight, dtype=np.float64)
    f = np.zeros((ns, nk, nb))
    if smearing == "fixed":
        nocc = int(round(nelec / 2.0))
        if abs(nocc - nelec / 2.0) > 1e-5:
            raise ValueError("fixed occupations need an even electron count")
        if nocc > nb:
            raise ValueError("fewer bands than occupied states")
        ef = -1e5
        for s in range(ns):
            for k in range(nk):
                if w[k] < 1e-8:
                    continue
                f[s, k, :nocc] = spin_factor
                ef = max(ef, float(e[s, k, :nocc].max()))
        return f, ef
    if smearing != "gaussian":
        raise ValueError(f"unknown smearing mode {smearing}")
    erf = np.vectorize(math.erf, otypes=[np.float64])
    lo, hi = -1e5, 1e5
    ef = 0.0
    for _ in range(60):
        ef = (hi + lo) / 2.0
        f = spin_factor * 0.5 * (1.0 - erf((e - ef) / width))
        f[:, w < 1e-8, :] = 0.0
        n = float(np.sum(f * (w[None, :, None] / spin_factor)))
        if n > nelec:
            hi = ef
        else:
            lo = ef
    # the occupations of the last midpoint (set_filling keeps them)
    if abs(float(np.sum(f * (w[None, :, None] / spin_factor))) - nelec) > 1e-8:
        raise ValueError("the Fermi level was not found (more bands or another smearing needed)")
    return f, ef


def occupied_counts(filling):
    """num_occupied_bands: bands with f > 1e-8, per spin and k."""
    return np.sum(np.asarray(filling) > 1e-8, axis=2).astype(np.int32)
