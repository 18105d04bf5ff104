"""Quantum ESPRESSO inputs as TC++ reads them: data-file-schema.xml and the
text wave-function files wfc{ik}.dat_nonbin, assembled into a TCSystem with the
symmetry-expanded k-set, Gindex maps and phase factors TC++ builds from them.

Follows, for the quantities this library consumes:
  io_qe_files_read_xml.cpp:78-98      lattice a_i, reciprocal b_i = (2 pi / alat) b_i^norm
  io_qe_files_read_xml.cpp:158-186    symmetry operations (rotation, fractional translation),
                                      only entries with <equivalent_atoms>
  symmetry.cpp:20-33, :124            U = inverse of the QE rotation; time reversal unless noinv
  io_qe_files_read_xml.cpp:204-241    irreducible k: Cartesian (2 pi / alat) -> crystal
  kpoints.cpp:34-91                   equivalent k-points k' = U^T k (+ time-reversed -k'),
                                      first match wins, irreducible-major order
  io_qe_files_read_wfc.f90:117-136    wfc*.dat_nonbin: header, b vectors, Miller indices,
                                      coefficients (band-major), scale factor
  plane_wave_basis.cpp:7-37           Miller index wrapped into (-(n+1)/2, n/2]
  plane_wave_basis.cpp:116-142        Gindex[isym] = wrap(+-U^T G), phase = exp(2 pi i t . (+-U^T G))
"""
import os
import xml.etree.ElementTree as ET

import numpy as np

from .system import TCSystem


def _floats(text):
    return np.array([float(x) for x in text.split()], dtype=np.float64)


class QEData:
    """Raw contents of a QE save directory (xml + text wave functions)."""

    def __init__(self, save_dir):
        self.dir = save_dir
        root = ET.parse(os.path.join(save_dir, "data-file-schema.xml")).getroot()
        out = root.find("output")
        ast = out.find("atomic_structure")
        self.alat = float(ast.attrib["alat"])
        cell = ast.find("cell")
        self.lattice = np.array([_floats(cell.find(a).text) for a in ("a1", "a2", "a3")])
        bs = out.find("basis_set")
        rl = bs.find("reciprocal_lattice")
        self.recip_norm = np.array([_floats(rl.find(b).text) for b in ("b1", "b2", "b3")])
        self.recip = (2.0 * np.pi / self.alat) * self.recip_norm
        fg = bs.find("fft_grid").attrib
        self.nr = (int(fg["nr1"]), int(fg["nr2"]), int(fg["nr3"]))
        self.gamma_only = bs.find("gamma_only").text.strip() == "true"
        self.atoms = [(a.attrib["name"], _floats(a.text)) for a in ast.find("atomic_positions")]
        self.pseudo_files = {sp.attrib["name"]: sp.find("pseudo_file").text.strip()
                             for sp in out.find("atomic_species").findall("species")}
        rots, trans = [], []
        for sym in out.find("symmetries").findall("symmetry"):
            if sym.find("equivalent_atoms") is None:
                continue
            r = np.rint(_floats(sym.find("rotation").text)).astype(np.int64).reshape(3, 3)
            rots.append(r)
            trans.append(_floats(sym.find("fractional_translation").text))
        self.rotation_qe = np.array(rots)
        self.translation = np.array(trans)
        flags = root.find("input").find("symmetry_flags")
        self.noinv = flags.find("noinv").text.strip() == "true"
        mag = out.find("magnetization")
        self.lsda = mag.find("lsda").text.strip() == "true"
        if mag.find("noncolin").text.strip() == "true":
            raise ValueError("non-collinear QE runs are outside this library's scope")
        band = out.find("band_structure")
        if self.lsda:
            self.nbnd_s = [int(band.find("nbnd_up").text), int(band.find("nbnd_dw").text)]
        else:
            self.nbnd_s = [int(band.find("nbnd").text)]
        self.nbnd = self.nbnd_s[0]
        self.nelec = float(band.find("nelec").text)
        self.kcart, self.kweight, self.npw_k, self.eig, self.occ = [], [], [], [], []
        for ks in band.findall("ks_energies"):
            kp = ks.find("k_point")
            self.kcart.append(_floats(kp.text))
            self.kweight.append(float(kp.attrib["weight"]))
            self.npw_k.append(int(ks.find("npw").text))
            self.eig.append(_floats(ks.find("eigenvalues").text))
            self.occ.append(_floats(ks.find("occupations").text))
        self.kcart = np.array(self.kcart)
        # Cartesian (2 pi / alat) -> crystal: k_cart = B_norm^T k_crys
        self.kcrys = np.linalg.solve(self.recip_norm.T, self.kcart.T).T

    # compact copy of the fields above plus every k-point's Miller indices and
    # coefficients, for inputs that travel without the QE directory
    _FIELDS = ("alat", "lattice", "recip_norm", "recip", "nr", "gamma_only", "rotation_qe", "translation", "noinv",
               "lsda", "nbnd", "nelec", "kcart", "kweight", "npw_k", "kcrys")

    @property
    def nspin(self):
        return 2 if self.lsda else 1

    def eig_spin(self, ik, s):
        """Eigenvalues (Ha) of spin s at irreducible k: QE lists the up bands, then the down bands."""
        o = sum(self.nbnd_s[:s])
        return self.eig[ik][o:o + self.nbnd_s[s]]

    def save_npz(self, path):
        d = {f: np.asarray(getattr(self, f)) for f in self._FIELDS}
        d["nbnd_s"] = np.array(self.nbnd_s)
        d["atom_names"] = np.array([n for n, _ in self.atoms])
        d["atom_pos"] = np.array([p for _, p in self.atoms])
        for ik in range(len(self.kweight)):
            d[f"eig_{ik}"], d[f"occ_{ik}"] = self.eig[ik], self.occ[ik]
            for sp in range(self.nspin):
                m, c = self.read_wfc(ik, sp)
                tag = "" if sp == 0 else "dw_"
                d[f"mill_{tag}{ik}"], d[f"evc_{tag}{ik}"] = m, c
        np.savez_compressed(path, **d)

    @classmethod
    def load_npz(cls, path):
        z = np.load(path)
        q = cls.__new__(cls)
        q.dir = None
        for f in cls._FIELDS:
            v = z[f]
            setattr(q, f, v.item() if v.ndim == 0 else v)
        q.nr = tuple(int(x) for x in q.nr)
        nk = len(q.kweight)
        q.kweight = [float(w) for w in q.kweight]
        q.eig = [z[f"eig_{ik}"] for ik in range(nk)]
        q.occ = [z[f"occ_{ik}"] for ik in range(nk)]
        q.atoms = [(str(n), p) for n, p in zip(z["atom_names"], z["atom_pos"])] if "atom_names" in z else []
        q.pseudo_files = {}
        q.nbnd_s = [int(x) for x in z["nbnd_s"]] if "nbnd_s" in z else [int(q.nbnd)]
        q._wfc = [[(z[f"mill_{tag}{ik}"], z[f"evc_{tag}{ik}"]) for ik in range(nk)]
                  for tag in ([""] if not q.lsda else ["", "dw_"])]
        return q

    def read_wfc(self, ik, spin=0):
        """(miller [npw][3] int, coefficients [nbnd][npw] complex) of wfc{ik+1}.dat_nonbin
        (wfcup / wfcdw for spin-polarised runs)."""
        if getattr(self, "_wfc", None) is not None:
            return self._wfc[spin][ik]
        name = f"wfc{ik + 1}" if not self.lsda else f"wfc{'up' if spin == 0 else 'dw'}{ik + 1}"
        path = os.path.join(self.dir, f"{name}.dat_nonbin")
        with open(path) as f:
            lines = f.read().split("\n")
        h = lines[0].split()
        scalef = float(h[6])
        ngw, igwx, npol, nbnd = (int(x) for x in lines[1].split())
        if npol != 1:
            raise ValueError("spinor wave functions are outside this library's scope")
        vals = " ".join(lines[3:]).split()
        mill = np.array(vals[:3 * igwx], dtype=np.int64).reshape(igwx, 3)
        c = np.array(vals[3 * igwx:3 * igwx + 2 * igwx * nbnd], dtype=np.float64).reshape(nbnd, igwx, 2)
        return mill, scalef * (c[..., 0] + 1j * c[..., 1])


def tc_rotations(rotation_qe):
    """TC++ keeps the inverse of QE's (integer) rotation (symmetry.cpp:20-30)."""
    return np.array([np.rint(np.linalg.inv(r.astype(np.float64))).astype(np.int32) for r in rotation_qe])


def _matched(v, lst):
    for w in lst:
        d = v - w
        d = d - np.round(d)            # into [-0.5, 0.5]
        if float(d @ d) < 1e-8:
            return True
    return False


def expand_kpoints(kcrys, kweight, U, time_reversal):
    """Kpoints::set_kvectors_by_symmetry (kpoints.cpp:34-91): per irreducible k
    the list of (k', isym, tr) with k' = U^T k (and -k' under time reversal)."""
    seen = [np.asarray(k, dtype=np.float64) for k, w in zip(kcrys, kweight) if w >= 1e-8]
    out = []
    for k, w in zip(kcrys, kweight):
        lst = [(np.asarray(k, dtype=np.float64), 0, False)]
        if w >= 1e-8:
            for isym in range(len(U)):
                v = U[isym].astype(np.float64).T @ k
                v[np.abs(v) < 1e-4] = 0.0
                if not _matched(v, seen):
                    seen.append(v)
                    lst.append((v, isym, False))
                if time_reversal and not _matched(-v, seen):
                    seen.append(-v)
                    lst.append((-v, isym, True))
        out.append(lst)
    return out


def wrap_miller(m, nr):
    """plane_wave_basis.cpp:21-22: into (-(n+1)/2, n/2]"""
    m = np.array(m, dtype=np.int64)
    for d in range(3):
        n = nr[d]
        m[:, d] = np.where(m[:, d] <= -(n + 1) // 2, m[:, d] + n, m[:, d])
        m[:, d] = np.where(m[:, d] > n // 2, m[:, d] - n, m[:, d])
    return m


def gindex_phase(mill, U, t, tr, nr):
    """Gindex / phase of one equivalent k (plane_wave_basis.cpp:121-141)."""
    Gs = mill @ U.astype(np.int64)               # (U^T G) as rows: G^T U
    if tr:
        Gs = -Gs
    gr = Gs.astype(np.float64) @ np.asarray(t, dtype=np.float64)
    ph = np.exp(2j * np.pi * gr)
    w = np.mod(Gs, np.array(nr))
    gi = (w[:, 0] + nr[0] * (w[:, 1] + nr[1] * w[:, 2])).astype(np.int32)
    return gi, ph


def _wfc_full(q, ik, spin):
    """Miller indices and coefficients of all plane waves of k: for a
    gamma_only run QE stores half of them, and the -G partners follow the
    stored list in its order, G = 0 skipped, with c(-G) = conj(c(G))
    (PlaneWaveBasis::set_G_from_mill, plane_wave_basis.cpp:8-43;
    BlochStates::set_phik_qe, bloch_states_initialize.cpp:215-265)."""
    mill, c = q.read_wfc(ik, spin)
    if not q.gamma_only:
        return mill, c
    zero = np.flatnonzero(np.all(mill == 0, axis=1))
    if zero.size != 1:
        raise ValueError("G = 0 not found in a gamma_only wave function")
    rest = np.delete(np.arange(len(mill)), zero[0])
    return np.concatenate([mill, -mill[rest]]), np.concatenate([c, np.conj(c[:, rest])], axis=1)


def system_from_qe(save_dir, method="BITC", A=None, F=None, nbands=None, nb_apply=None, name=None,
                   includes_div_correction=True, smearing="fixed", smearing_width=0.01):
    """TCSystem of the first SCF iteration of a TC++ run on a QE save directory
    (or a QEData, or the .npz written by QEData.save_npz): the QE orbitals as
    right (and, for BITC, left) orbitals, one spin channel per QE spin (lsda),
    the occupations TC++'s set_filling gives the QE eigenvalues (smearing
    "fixed" or "gaussian" with smearing_width in Ha; tc_b200.occupations),
    the density of these orbitals, divergence sums of the SCF mesh.
    A, F: 2x2 RPA Jastrow parameters."""
    from . import synth
    from .occupations import fermi_filling, occupied_counts
    q = save_dir if isinstance(save_dir, QEData) else (
        QEData.load_npz(save_dir) if str(save_dir).endswith(".npz") else QEData(save_dir))
    nspin = q.nspin
    nr = q.nr
    if min(q.kweight) < 1e-8:
        raise ValueError("k-points of zero weight (whose divergence corrections need the kVaux sums of BAND-mode "
                         "runs) are outside this library's scope")
    U = tc_rotations(q.rotation_qe)
    star = expand_kpoints(q.kcrys, q.kweight, U, not q.noinv)
    nk = len(star)
    nbnd = min(q.nbnd_s) if nbands is None else int(nbands)
    if nbnd > min(q.nbnd_s):
        raise ValueError("more bands requested than the QE run has")
    eig = np.array([[q.eig_spin(ik, sp)[:nbnd] for ik in range(nk)] for sp in range(nspin)])
    fill, _ = fermi_filling(eig, q.kweight, q.nelec, nspin, smearing, smearing_width)
    nocc = occupied_counts(fill)
    kvec_all, time_rev, rot_index, nsym_k = [], [], [], []
    gidx, phase, npw = [], [], []
    phik = [[None] * nk for _ in range(nspin)]
    for ik in range(nk):
        mill, _ = _wfc_full(q, ik, 0)
        mill = wrap_miller(mill, nr)
        npw.append(len(mill))
        nsym_k.append(len(star[ik]))
        for v, isym, tr in star[ik]:
            kvec_all.append(v)
            time_rev.append(1 if tr else 0)
            rot_index.append(isym)
            gi, ph = gindex_phase(mill, U[isym], q.translation[isym], tr, nr)
            gidx.append(gi)
            phase.append(ph)
        for sp in range(nspin):
            m2, c = _wfc_full(q, ik, sp)
            if not np.array_equal(wrap_miller(m2, nr), mill):
                raise ValueError("the spin channels of a k-point have different plane-wave sets")
            phik[sp][ik] = c[:nbnd]
    lattice = q.lattice
    recip = q.recip
    omega = abs(float(np.linalg.det(lattice)))
    kvec_all = np.array(kvec_all)
    alpha, sumv = synth.sum_of_vaux(recip, omega, np.array([s[0][0] for s in star]), kvec_all)
    if A is None:
        A = np.zeros((2, 2)) if method == "HF" else None
    Aarr = np.asarray(A, dtype=np.float64) if A is not None else np.zeros((2, 2))
    Farr = np.asarray(F, dtype=np.float64) if F is not None else np.ones((2, 2))
    flat = np.concatenate([np.ascontiguousarray(P).ravel() for sp in range(nspin) for P in phik[sp]])
    s = TCSystem(
        nr=nr, recip=recip, lattice=lattice, omega=omega, method=method, nspin=nspin,
        nsym_k=np.array(nsym_k, dtype=np.int32), kvec=kvec_all, time_rev=np.array(time_rev, dtype=np.uint8),
        rot_index=np.array(rot_index, dtype=np.int32), rotation=U.astype(np.int32),
        translation=np.asarray(q.translation, dtype=np.float64), num_kpoints=int(len(kvec_all)),
        npw=np.array(npw, dtype=np.int32), gindex=np.concatenate(gidx * nspin).astype(np.int32),
        phase=np.concatenate(phase * nspin), jastrow_A=Aarr, jastrow_F=Farr,
        includes_div_correction=includes_div_correction, alpha_Vaux=float(alpha), sum_Vaux=sumv,
        nbands=np.full(nspin, nbnd, dtype=np.int32), nocc=nocc,
        filling=fill.ravel(), phik=flat, phik_left=flat.copy() if method == "BITC" else None,
        density=np.zeros((2, int(np.prod(nr))), dtype=np.complex128), name=name or "qe",
    )
    s.density = synth.density_numpy(s)
    nb = nbnd if nb_apply is None else int(nb_apply)
    s.nb_apply = np.full((nspin, nk), nb, dtype=np.int32)
    s.psi = np.concatenate([np.ascontiguousarray(P[:nb]).ravel() for sp in range(nspin) for P in phik[sp]])
    s.meta["qe"] = q
    s.meta["kweight"] = np.asarray(q.kweight, dtype=np.float64)
    s.meta["nelec"] = float(q.nelec)
    s.meta["eig"] = eig
    s.meta["smearing"] = (smearing, float(smearing_width))
    return s
