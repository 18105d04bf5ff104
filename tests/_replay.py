"""Golden replay of the reference's own test runs (test/example1 HF,
test/example2 TC, test/example3 BITC: fcc Si from Quantum ESPRESSO files):
the first SCF iteration of TC++ restated in numpy around an H-apply callable,
so that the energies TC++ printed for it can be reproduced from the oracle's
(or the library's) H phi.

Restated steps:
  io_qe_files_read.cpp:135-141, read_casl  Jastrow: F from parameters.casl, A by the cusp condition
  bloch_states_scfloop_filling_density.cpp:8-70   fixed occupations: nelec/2 lowest bands, f = 2
  diagonalization.cpp:176-236                      iteration 1: filling, density, one block_davidson
  diagonalization_davidson.cpp:6-600               block Davidson, num_refresh_david = 1,
                                                   max_num_blocks_david = 2, biortho_david = false
  diagonalization_utils.cpp:7-28                   Gram_Schmidt (drop below norm 1e-8)
  diagonalization_utils.cpp:82-119                 sort_eigen (swap sort on the real part)
  diagonalization_utils.cpp:165-211                make_a_new_trial_vector (Payne preconditioner,
                                                   eigenvalue of the previous iteration)
  total_energy.cpp:101-168                         E_n = sum_k sum_isym sum_b f e_n / N_k
                                                   (conj for time-reversed partners; 1/2, 1/3)
"""
import json
import os

import numpy as np

from tc_b200 import abi
from tc_b200.qe import QEData, system_from_qe
from tc_b200.upf import UPF, pseudo_from_upf, species_and_positions

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

H2_TERMS = {"HF": abi.TERM_HF2H | abi.TERM_HF2X, "TC": abi.TERM_TC2H | abi.TERM_TC2X,
            "BITC": abi.TERM_TC2H | abi.TERM_TC2X}
H3_TERMS = {"HF": 0, "TC": abi.TERMS_TC & ~abi.TERM_TC2X, "BITC": abi.TERMS_TC & ~abi.TERM_TC2X}


def examples():
    with open(os.path.join(GOLDEN, "si_examples.json")) as f:
        return json.load(f)


def si_system(example):
    """(TCSystem of the first SCF iteration, Pseudo, QE eigenvalues
    [nspin][nk][nb], golden record) of one of the replayed runs."""
    rec = examples()[example]
    method = rec["calc_method"]
    q = QEData.load_npz(os.path.join(GOLDEN, rec["qe"]))
    A = F = None
    if "F" in rec:
        F = np.array(rec["F"], dtype=np.float64)
        A = np.array([[F[0, 0] ** 2 / 2, F[0, 1] ** 2], [F[1, 0] ** 2, F[1, 1] ** 2 / 2]])
    s = system_from_qe(q, method=method, A=A, F=F, smearing=rec["smearing"], smearing_width=rec["smearing_width"])
    upf = UPF.from_arrays(np.load(os.path.join(GOLDEN, "si_upf.npz")))
    sp, pos, _ = species_and_positions(q)
    pp = pseudo_from_upf(s, [upf], sp, pos)
    return s, pp, s.meta["eig"], rec


def kg2(system, k):
    """|k+G|^2 at the isym-0 plane waves of irreducible k (Cartesian)."""
    a0 = int(system.kall_off[k])
    gi, _ = system.gidx(0, a0)
    n = np.array(system.nr)
    w = np.stack([gi % n[0], (gi // n[0]) % n[1], gi // (n[0] * n[1])], 1)
    m = np.where(w > n // 2, w - n, w)
    kg = (np.asarray(system.kvec[a0])[None, :] + m) @ np.asarray(system.recip)
    return np.einsum("ij,ij->i", kg, kg)


def precondition(kG2, phi, h, e):
    """make_a_new_trial_vector: -K (H phi - e phi), normalised (zero below 1e-8)."""
    p2 = np.abs(phi) ** 2
    kin = float(kG2 @ p2) / float(np.sum(p2))
    x = kG2 / kin
    c = (27 + x * (18 + x * (12 + x * 8))) / (27 + x * (18 + x * (12 + x * (8 + x * 16))))
    out = -c * (h - e * phi)
    nrm = np.linalg.norm(out)
    return np.zeros_like(out) if nrm < 1e-8 else out / nrm


def gram_schmidt(basis, t, tol=1e-8):
    t = t.copy()
    for v in basis:
        t -= np.vdot(v, t) * v
    nrm = np.linalg.norm(t)
    return None if nrm < tol else t / nrm


def sort_eigen(w, X):
    w = w.copy()
    X = X.copy()
    n = len(w)
    for i in range(n):
        for j in range(i + 1, n):
            if w[i].real > w[j].real:
                w[[i, j]] = w[[j, i]]
                X[:, [i, j]] = X[:, [j, i]]
    return w, X


def davidson(system, apply, eig_ref, max_blocks=2):
    """One Diagonalization::block_davidson call (num_refresh_david 1, not
    bi-orthogonal) for every spin channel.  apply(psi_flat, nb_apply[nspin][nk])
    -> (h1, h2, h3) flat, packed like psi.  eig_ref [nspin][nk][nb]: the
    previous eigenvalues.  Returns eigenvalues [nspin][nk][nb] and energies
    e[n][nspin][nk][nb] (n = 1-, 2-, 3-body: diag(L^H H_n,sub X),
    L = (X^-1)^H for BITC); the new orbitals stay in davidson.last_orbitals."""
    bitc = system.method == "BITC"
    ns, nk = system.nspin, system.nk_irr
    nb = int(system.nbands[0])
    V = {}
    for sp in range(ns):
        for k in range(nk):
            rows = [system.orb(sp, k, b).copy() for b in range(nb)]
            if bitc:                                             # :64-71
                out = []
                for r in rows:
                    g = gram_schmidt(out, r)
                    assert g is not None
                    out.append(g)
                rows = out
            V[sp, k] = rows
    HV = {key: [[], [], []] for key in V}
    nfix = {key: 0 for key in V}
    keys = [(sp, k) for sp in range(ns) for k in range(nk)]

    def run_block():
        blocks = {key: V[key][nfix[key]:] for key in keys}
        nba = np.array([[len(blocks[sp, k]) for k in range(nk)] for sp in range(ns)], dtype=np.int32)
        psi = np.concatenate([np.concatenate(blocks[key]) for key in keys])
        hs = apply(psi, nba)
        off = 0
        out = {}
        for key in keys:
            npw = len(V[key][0])
            per = []
            for i in range(len(blocks[key])):
                sl = slice(off, off + npw)
                per.append(tuple(None if h is None else h[sl].copy() for h in hs))
                off += npw
            out[key] = per
        return blocks, out

    for _ in range(max_blocks - 1):                                  # :207-400
        blocks, hs = run_block()
        for key in keys:
            kG2 = kg2(system, key[1])
            old = len(V[key])
            for i, phi in enumerate(blocks[key]):
                h1, h2, h3 = hs[key][i]
                for n, h in enumerate((h1, h2, h3)):
                    HV[key][n].append(h)
                htot = sum(h for h in (h1, h2, h3) if h is not None)
                t = precondition(kG2, phi, htot, eig_ref[key[0]][key[1]][i])
                g = gram_schmidt(V[key], t)
                if g is not None:
                    V[key].append(g)
            nfix[key] = old
    blocks, hs = run_block()                                          # :405-430
    for key in keys:
        for i in range(len(blocks[key])):
            for n in range(3):
                HV[key][n].append(hs[key][i][n])
    eig = np.zeros((ns, nk, nb), dtype=np.complex128)
    en = np.zeros((3, ns, nk, nb), dtype=np.complex128)
    right, left = {}, {}
    for key in keys:                                                  # :431-600
        sp, k = key
        Vm = np.array(V[key])
        Hn = [None if HV[key][n][0] is None else Vm.conj() @ np.array(HV[key][n]).T for n in range(3)]
        H = sum(h for h in Hn if h is not None)
        w, X = np.linalg.eig(H)
        w, X = sort_eigen(w, X)
        L = np.linalg.inv(X).conj().T if bitc else X
        eig[sp, k] = w[:nb]
        for n in range(3):
            if Hn[n] is not None:
                en[n, sp, k] = np.einsum("ai,ab,bi->i", L[:, :nb].conj(), Hn[n], X[:, :nb])
        R = X[:, :nb].T @ Vm                                          # V X
        if bitc:                                                      # BITC final loop: V X, V (X^-1)^H
            right[key] = R
            left[key] = L[:, :nb].T @ Vm
        else:                                                         # Gram-Schmidt of V X
            out = []
            for r in R:
                g = gram_schmidt(out, r)
                assert g is not None
                out.append(g)
            right[key] = np.array(out)
    davidson.last_orbitals = ([right[key] for key in keys], [left[key] for key in keys] if bitc else None)
    return eig, en


def occupations(system, eig):
    """set_filling with the run's smearing on eigenvalues [nspin][nk][nb]."""
    from tc_b200.occupations import fermi_filling
    mode, width = system.meta["smearing"]
    f, _ = fermi_filling(eig, system.meta["kweight"], system.meta["nelec"], system.nspin, mode, width)
    return f


def scf_update(system, eig, mixing_beta=0.7):
    """Next SCF iteration's system from the last davidson() call: new
    orbitals, occupations of the new eigenvalues, density of the new orbitals
    (numpy restatement of set_density) mixed with the previous one,
    (1 - beta) n_old + beta n_new (bloch_states_scfloop_filling_density.cpp:340-345)."""
    import dataclasses
    from tc_b200 import synth
    from tc_b200.occupations import occupied_counts
    right, left = davidson.last_orbitals
    f = occupations(system, eig)
    s = dataclasses.replace(system, phik=np.concatenate([r.ravel() for r in right]),
                            phik_left=None if left is None else np.concatenate([l.ravel() for l in left]),
                            filling=f.ravel(), nocc=occupied_counts(f), meta=dict(system.meta))
    s.density = (1.0 - mixing_beta) * system.density + mixing_beta * synth.density_numpy(s)
    return s


def total_energy(system, eig, en):
    """(E_1, E_2, E_3) with the occupations of the new eigenvalues
    (calc_total_energy runs after set_filling of the next iteration)."""
    f = occupations(system, eig)
    E = np.zeros(3, dtype=np.complex128)
    w = np.array([1.0, 0.5, 1.0 / 3.0])
    for sp in range(system.nspin):
        for k in range(system.nk_irr):
            if system.meta["kweight"][k] < 1e-8:
                continue
            a0 = int(system.kall_off[k])
            for isym in range(int(system.nsym_k[k])):
                tr = bool(system.time_rev[a0 + isym])
                e = np.conj(en[:, sp, k]) if tr else en[:, sp, k]
                E += (e * f[sp, k][None, :]).sum(axis=1) * w
    return E / system.num_kpoints


def oracle_apply(system, pseudo):
    from oracle import oracle
    m2 = H2_TERMS[system.method]
    m3 = H3_TERMS[system.method]

    def apply(psi, nba):
        h1 = oracle.apply_h1(system, abi.TERMS_H1, pseudo=pseudo, psi=psi, nb_apply=nba)
        h2, h3 = oracle.apply(system, m2 | m3, psi=psi, nb_apply=nba)
        return h1, h2, (h3 if m3 else None)
    return apply
