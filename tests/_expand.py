"""Expand a symmetry-reduced TCSystem into the equivalent system with every
k-point of the full Brillouin zone listed as irreducible (nsym_k = 1), the
rotated / time-reversed orbitals written out explicitly.  Used to check the
symmetry machinery (Gindex_at_k[isym], phase, time reversal and the rotation
of intermediates in tc3a2a4b2b5) against a direct evaluation."""
import numpy as np

from tc_b200.system import TCSystem


def expand(s):
    ik_of_all = np.repeat(np.arange(s.nk_irr), s.nsym_k)
    nka = s.nk_all
    npw = s.npw[ik_of_all].astype(np.int32)
    gidx, phase, phik, left, fill, nocc, psi, nb = [], [], [], [], [], [], [], []
    for sp in range(s.nspin):
        for a in range(nka):
            gi, ph = s.gidx(sp, a)
            gidx.append(gi.copy())
            phase.append(np.ones(len(gi), dtype=np.complex128))
    for sp in range(s.nspin):
        for a in range(nka):
            k = ik_of_all[a]
            gi, ph = s.gidx(sp, a)
            tr = bool(s.time_rev[a])
            tf = (lambda c: np.conj(c) * ph) if tr else (lambda c: c * ph)
            for b in range(int(s.nbands[sp])):
                phik.append(tf(s.orb(sp, k, b)))
                if s.phik_left is not None:
                    left.append(tf(s.orb(sp, k, b, left=True)))
                fill.append(s.fill(sp, k, b))
            nocc.append(int(s.nocc[sp][k]))
            n_ap = int(s.nb_apply[sp][k])
            nb.append(n_ap)
            for b in range(n_ap):
                psi.append(tf(s.band_view(s.psi, sp, k, b)))
    e = TCSystem(
        nr=s.nr, recip=s.recip, lattice=s.lattice, omega=s.omega, method=s.method, nspin=s.nspin,
        nsym_k=np.ones(nka, dtype=np.int32), kvec=s.kvec.copy(), time_rev=np.zeros(nka, dtype=np.uint8),
        rot_index=np.zeros(nka, dtype=np.int32), rotation=np.eye(3, dtype=np.int32)[None],
        translation=np.zeros((1, 3)), num_kpoints=s.num_kpoints, npw=npw,
        gindex=np.concatenate(gidx).astype(np.int32), phase=np.concatenate(phase),
        jastrow_A=s.jastrow_A, jastrow_F=s.jastrow_F, includes_div_correction=s.includes_div_correction,
        alpha_Vaux=s.alpha_Vaux, sum_Vaux=None,
        nbands=s.nbands.copy(), nocc=np.array(nocc, dtype=np.int32).reshape(s.nspin, nka),
        filling=np.array(fill), phik=np.concatenate(phik),
        phik_left=np.concatenate(left) if left else None, density=s.density.copy(), name=s.name + "-expanded",
    )
    # sum_of_Vaux depends on k only through the mesh: the partner of k has the
    # same value (the q-sum runs over the whole mesh)
    e.sum_Vaux = np.array([s.sum_Vaux[ik_of_all[a]] for a in range(nka)])
    e.nb_apply = np.array(nb, dtype=np.int32).reshape(s.nspin, nka)
    e.psi = np.concatenate(psi)
    e.meta["first_of_irr"] = np.concatenate([[0], np.cumsum(s.nsym_k)[:-1]])
    return e
