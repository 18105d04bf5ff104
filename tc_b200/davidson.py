"""Block Davidson of TC++ on the device (Diagonalization::block_davidson,
diagonalization_davidson.cpp:6-689), one call per SCF iteration, with the
defaults TC++ runs with: num_refresh_david = 1, max_num_blocks_david = 2,
biortho_david = false.

Per irreducible k the basis V (orthonormal) lives on the device; H phi of each
block comes from the library's operator application (one-body terms through
tcg_apply_h1, two- and three-body terms through tcg_apply, all bands of all
k-points of a block in one call); new trial vectors from tcg_davidson_expand
(preconditioned residuals, Gram-Schmidt, drop of vanishing vectors); the
Rayleigh-Ritz step from tcg_subspace_ritz (ZGEMM, FP64 non-Hermitian
eigensolve, sort by the real part, left vectors for BITC); the Ritz vectors
of HF / TC re-orthonormalised by tcg_gram_schmidt (:534-547).

scf_update then does what the SCF loop does between two Davidson calls
(diagonalization.cpp:176-197): the new orbitals and eigenvalues, fixed
occupations (bloch_states_scfloop_filling_density.cpp:37-70) and the mixed
density (tcg_density), and total_energy the energy functional
(total_energy.cpp:101-168).
"""
import dataclasses

import numpy as np

from . import abi
from .context import davidson_expand, gram_schmidt, subspace_ritz

#: two- and three-body terms of calc_hamiltonian::all per calc_method
#: (calc_hamiltonian_all.cpp:80-158)
H2_TERMS = {"HF": abi.TERM_HF2H | abi.TERM_HF2X, "TC": abi.TERM_TC2H | abi.TERM_TC2X,
            "BITC": abi.TERM_TC2H | abi.TERM_TC2X}
H3_TERMS = {"HF": 0, "TC": abi.TERMS_TC & ~abi.TERM_TC2X, "BITC": abi.TERMS_TC & ~abi.TERM_TC2X}


def kg2(system, k):
    """|k+G|^2 at the plane waves of irreducible k (isym 0), Cartesian."""
    a0 = int(system.kall_off[k])
    gi, _ = system.gidx(0, a0)
    n = np.array(system.nr)
    w = np.stack([gi % n[0], (gi // n[0]) % n[1], gi // (n[0] * n[1])], 1)
    m = np.where(w > n // 2, w - n, w)
    kg = (np.asarray(system.kvec[a0])[None, :] + m) @ np.asarray(system.recip)
    return np.einsum("ij,ij->i", kg, kg)


@dataclasses.dataclass
class DavidsonResult:
    eigenvalues: np.ndarray        # [nk_irr][nbands] complex, sorted by the real part
    energies: np.ndarray           # [3][nk_irr][nbands] complex: 1-, 2-, 3-body e_n of each band
    phik: list                     # per k: [nbands][npw] complex128 (host), new right orbitals
    phik_left: list                # per k (BITC): new left orbitals, else None
    basis_size: list               # per k: subspace dimension of the Rayleigh-Ritz step


def block_davidson(ctx, system, eig_ref, max_blocks=2, h1_terms=abi.TERMS_H1):
    """One block-Davidson call for spin 0 of `system` (the context's state:
    occupied orbitals, fillings and density stay fixed during the call).
    eig_ref: [nk_irr][nbands] eigenvalues of the previous iteration, used by
    the preconditioner.  Needs torch with CUDA for the device basis."""
    import torch
    if system.nspin != 1:
        raise ValueError("block_davidson drives one spin channel (nspin = 1)")
    dev = torch.device("cuda", torch.cuda.current_device())
    method = system.method
    bitc = method == "BITC"
    m2, m3 = H2_TERMS[method], H3_TERMS[method]
    nk, nb = system.nk_irr, int(system.nbands[0])
    cap = nb * max_blocks
    V, HV, kG2 = [], [[], [], []], []
    for k in range(nk):
        npw = int(system.npw[k])
        Vk = torch.zeros((cap, npw), dtype=torch.complex128, device=dev)
        Vk[:nb] = torch.from_numpy(np.stack([system.orb(0, k, b) for b in range(nb)])).to(dev)
        if bitc:                                    # orthonormal basis for BITC (:64-71)
            gram_schmidt(Vk[:nb])
        V.append(Vk)
        for n in range(3):
            HV[n].append(torch.zeros((cap, npw), dtype=torch.complex128, device=dev) if (n < 2 or m3) else None)
        kG2.append(torch.from_numpy(kg2(system, k)).to(dev))
    nbasis = [nb] * nk
    nfix = [0] * nk

    def apply_block():
        nba = np.array([[nbasis[k] - nfix[k] for k in range(nk)]], dtype=np.int32)
        psi = np.ascontiguousarray(np.concatenate([V[k][nfix[k]:nbasis[k]].cpu().numpy().ravel()
                                                   for k in range(nk)]))
        h1 = ctx.apply_h1(h1_terms, psi=psi, nb_apply=nba)
        h2, h3 = ctx.apply(m2 | m3, psi=psi, nb_apply=nba)
        off = 0
        for k in range(nk):
            npw = int(system.npw[k])
            cnt = nbasis[k] - nfix[k]
            sl = slice(off, off + cnt * npw)
            for n, h in enumerate((h1, h2, h3)):
                if HV[n][k] is not None:
                    HV[n][k][nfix[k]:nbasis[k]] = torch.from_numpy(h[sl].reshape(cnt, npw)).to(dev)
            off += cnt * npw

    for _ in range(max_blocks - 1):                  # grow the subspace (:207-400)
        apply_block()
        for k in range(nk):
            old = nbasis[k]
            h = [None if HV[n][k] is None else HV[n][k][nfix[k]:old] for n in range(3)]
            nbasis[k] = davidson_expand(V[k], old, V[k][nfix[k]:old], h, kG2[k],
                                        np.asarray(eig_ref[k])[:old - nfix[k]])
            nfix[k] = old
    apply_block()                                    # H on the last block (:402-430)
    eig = np.zeros((nk, nb), dtype=np.complex128)
    en = np.zeros((3, nk, nb), dtype=np.complex128)
    phik, phil = [], []
    for k in range(nk):                              # Rayleigh-Ritz (:431-600)
        n = nbasis[k]
        w, e, Vo, Vl = subspace_ritz(V[k][:n], [None if HV[i][k] is None else HV[i][k][:n] for i in range(3)],
                                     nb, biortho=bitc, left=bitc)
        if not bitc:
            Vo = Vo.contiguous()
            gram_schmidt(Vo)
        eig[k] = w[:nb]
        en[:, k] = e
        phik.append(Vo.cpu().numpy())
        phil.append(None if Vl is None else Vl.cpu().numpy())
    return DavidsonResult(eigenvalues=eig, energies=en, phik=phik, phik_left=phil if bitc else None,
                          basis_size=list(nbasis))


def fixed_filling(system, nelec):
    """Fixed occupations (bloch_states_scfloop_filling_density.cpp:37-70):
    the round(nelec / 2) lowest bands of every k get 2 (unpolarised)."""
    nocc = int(round(nelec / 2.0))
    nb = int(system.nbands[0])
    if nocc > nb:
        raise ValueError("fewer bands than occupied states")
    f = np.zeros((system.nk_irr, nb))
    f[:, :nocc] = 2.0
    return f, nocc


def total_energy(system, res, nelec):
    """(E_1, E_2, E_3) of a Davidson result with fixed occupations
    (TotalEnergy::calc_total_energy, total_energy.cpp:101-168)."""
    f, _ = fixed_filling(system, nelec)
    w = np.array([1.0, 0.5, 1.0 / 3.0])
    E = np.zeros(3, dtype=np.complex128)
    for k in range(system.nk_irr):
        a0 = int(system.kall_off[k])
        for isym in range(int(system.nsym_k[k])):
            tr = bool(system.time_rev[a0 + isym])
            e = np.conj(res.energies[:, k]) if tr else res.energies[:, k]
            E += (e * f[k][None, :]).sum(axis=1) * w
    return E / system.num_kpoints


def scf_update(ctx, system, res, nelec, mixing_beta=0.7):
    """The TCSystem of the next SCF iteration: new orbitals (left ones for
    BITC), fixed occupations and the density of the new orbitals computed on
    the device, mixed with the previous density as (1 - beta) n_old + beta
    n_new (BlochStates::reset_phik, set_filling, set_density with density
    mixing, bloch_states_scfloop_filling_density.cpp:255-345); returns
    (system, eigenvalues for the next preconditioner)."""
    f, nocc = fixed_filling(system, nelec)
    flat = np.concatenate([np.ascontiguousarray(p).ravel() for p in res.phik])
    left = None if res.phik_left is None else np.concatenate([np.ascontiguousarray(p).ravel()
                                                              for p in res.phik_left])
    s = dataclasses.replace(system, phik=flat, phik_left=left, filling=f.ravel().copy(),
                            nocc=np.full((1, system.nk_irr), nocc, dtype=np.int32), meta=dict(system.meta))
    s.density = (1.0 - mixing_beta) * system.density + mixing_beta * ctx.density(s)
    return s, res.eigenvalues.copy()
