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
(diagonalization.cpp:176-197): the new orbitals and eigenvalues, the
occupations (fixed or Gaussian smearing, tc_b200.occupations) and the mixed
density (tcg_density), and total_energy the energy functional
(total_energy.cpp:101-168).  Spin-polarised systems run every channel.
"""
import dataclasses

import numpy as np

from . import abi
from .context import davidson_expand, gram_schmidt, subspace_ritz
from .occupations import fermi_filling, occupied_counts

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
    eigenvalues: np.ndarray        # [nspin][nk_irr][nbands] complex, sorted by the real part
    energies: np.ndarray           # [3][nspin][nk_irr][nbands] complex: 1-, 2-, 3-body e_n of each band
    phik: list                     # per (spin, k): [nbands][npw] complex128 (host), new right orbitals
    phik_left: list                # per (spin, k) (BITC): new left orbitals, else None
    basis_size: list               # per (spin, k): subspace dimension of the Rayleigh-Ritz step


def block_davidson(ctx, system, eig_ref, max_blocks=2, h1_terms=abi.TERMS_H1):
    """One block-Davidson call for every spin channel of `system` (the
    context's state: occupied orbitals, fillings and density stay fixed during
    the call).  eig_ref: [nspin][nk_irr][nbands] eigenvalues of the previous
    iteration, used by the preconditioner.  Needs torch with CUDA for the
    device basis."""
    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    method = system.method
    bitc = method == "BITC"
    m2, m3 = H2_TERMS[method], H3_TERMS[method]
    ns, nk, nb = system.nspin, system.nk_irr, int(system.nbands[0])
    if any(int(x) != nb for x in system.nbands):
        raise ValueError("block_davidson needs the same band count in both spin channels")
    keys = [(sp, k) for sp in range(ns) for k in range(nk)]
    cap = nb * max_blocks
    V, HV, kG2 = {}, {}, {}
    for sp, k in keys:
        npw = int(system.npw[k])
        Vk = torch.zeros((cap, npw), dtype=torch.complex128, device=dev)
        Vk[:nb] = torch.from_numpy(np.stack([system.orb(sp, k, b) for b in range(nb)])).to(dev)
        if bitc:                                    # orthonormal basis for BITC (:64-71)
            gram_schmidt(Vk[:nb])
        V[sp, k] = Vk
        HV[sp, k] = [torch.zeros((cap, npw), dtype=torch.complex128, device=dev) if (n < 2 or m3) else None
                     for n in range(3)]
        if sp == 0:
            kG2[k] = torch.from_numpy(kg2(system, k)).to(dev)
    nbasis = {key: nb for key in keys}
    nfix = {key: 0 for key in keys}

    def apply_block():
        nba = np.array([[nbasis[sp, k] - nfix[sp, k] for k in range(nk)] for sp in range(ns)], dtype=np.int32)
        psi = np.ascontiguousarray(np.concatenate([V[key][nfix[key]:nbasis[key]].cpu().numpy().ravel()
                                                   for key in keys]))
        h1 = ctx.apply_h1(h1_terms, psi=psi, nb_apply=nba)
        h2, h3 = ctx.apply(m2 | m3, psi=psi, nb_apply=nba)
        off = 0
        for key in keys:
            npw = int(system.npw[key[1]])
            cnt = nbasis[key] - nfix[key]
            sl = slice(off, off + cnt * npw)
            for n, h in enumerate((h1, h2, h3)):
                if HV[key][n] is not None:
                    HV[key][n][nfix[key]:nbasis[key]] = torch.from_numpy(h[sl].reshape(cnt, npw)).to(dev)
            off += cnt * npw

    for _ in range(max_blocks - 1):                  # grow the subspace (:207-400)
        apply_block()
        for key in keys:
            old = nbasis[key]
            h = [None if HV[key][n] is None else HV[key][n][nfix[key]:old] for n in range(3)]
            nbasis[key] = davidson_expand(V[key], old, V[key][nfix[key]:old], h, kG2[key[1]],
                                          np.asarray(eig_ref[key[0]][key[1]])[:old - nfix[key]])
            nfix[key] = old
    apply_block()                                    # H on the last block (:402-430)
    eig = np.zeros((ns, nk, nb), dtype=np.complex128)
    en = np.zeros((3, ns, nk, nb), dtype=np.complex128)
    phik, phil = [], []
    for key in keys:                                 # Rayleigh-Ritz (:431-600)
        n = nbasis[key]
        w, e, Vo, Vl = subspace_ritz(V[key][:n], [None if HV[key][i] is None else HV[key][i][:n] for i in range(3)],
                                     nb, biortho=bitc, left=bitc)
        if not bitc:
            Vo = Vo.contiguous()
            gram_schmidt(Vo)
        eig[key] = w[:nb]
        en[(slice(None),) + key] = e
        phik.append(Vo.cpu().numpy())
        phil.append(None if Vl is None else Vl.cpu().numpy())
    return DavidsonResult(eigenvalues=eig, energies=en, phik=phik, phik_left=phil if bitc else None,
                          basis_size=[nbasis[key] for key in keys])


def occupations(system, eigenvalues):
    """set_filling on eigenvalues [nspin][nk][nb] with the system's k-point
    weights, electron count and smearing (system.meta: "kweight", "nelec",
    "smearing" = (mode, width); tc_b200.qe.system_from_qe sets them)."""
    mode, width = system.meta.get("smearing", ("fixed", 0.01))
    kw = system.meta.get("kweight")
    if kw is None:
        kw = np.asarray(system.nsym_k, dtype=np.float64) * (2.0 if system.nspin == 1 else 1.0) / system.num_kpoints
    nelec = system.meta.get("nelec")
    if nelec is None:
        raise ValueError("system.meta['nelec'] is needed for the occupations")
    f, _ = fermi_filling(eigenvalues, kw, nelec, system.nspin, mode, width)
    return f


def total_energy(system, res):
    """(E_1, E_2, E_3) of a Davidson result with the occupations of its
    eigenvalues (TotalEnergy::calc_total_energy, total_energy.cpp:101-168)."""
    f = occupations(system, res.eigenvalues)
    w = np.array([1.0, 0.5, 1.0 / 3.0])
    E = np.zeros(3, dtype=np.complex128)
    for sp in range(system.nspin):
        for k in range(system.nk_irr):
            a0 = int(system.kall_off[k])
            for isym in range(int(system.nsym_k[k])):
                tr = bool(system.time_rev[a0 + isym])
                e = np.conj(res.energies[:, sp, k]) if tr else res.energies[:, sp, k]
                E += (e * f[sp, k][None, :]).sum(axis=1) * w
    return E / system.num_kpoints


def scf_update(ctx, system, res, mixing_beta=0.7):
    """The TCSystem of the next SCF iteration: new orbitals (left ones for
    BITC), the occupations of the new eigenvalues and the density of the new
    orbitals computed on the device, mixed with the previous density as
    (1 - beta) n_old + beta n_new (BlochStates::reset_phik, set_filling,
    set_density with density mixing, bloch_states_scfloop_filling_density.cpp:
    8-345); returns (system, eigenvalues for the next preconditioner)."""
    f = occupations(system, res.eigenvalues)
    flat = np.concatenate([np.ascontiguousarray(p).ravel() for p in res.phik])
    left = None if res.phik_left is None else np.concatenate([np.ascontiguousarray(p).ravel()
                                                              for p in res.phik_left])
    s = dataclasses.replace(system, phik=flat, phik_left=left, filling=f.ravel().copy(),
                            nocc=occupied_counts(f), meta=dict(system.meta))
    s.density = (1.0 - mixing_beta) * system.density + mixing_beta * ctx.density(s)
    return s, res.eigenvalues.copy()
