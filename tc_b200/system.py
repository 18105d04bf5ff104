"""Host-side data model of one operator application: the flat, packed arrays
behind include/tcg.h's tcg_system_desc / tcg_state_desc, plus the trial
block psi.

Layout mirrors TC++'s containers (reference: src/include/plane_wave_basis.hpp,
bloch_states.hpp, kpoints.hpp):
  gindex / phase : [nspin][nk_all][npw(ik)]      Gindex_at_k_scf, phase_factor_at_k
  phik / phik_left: [nspin][nk_irr][nbands[s]][npw(ik)]   phik_scf / phik_left_scf
  psi / h2 / h3  : [nspin][nk_irr][nb_apply[s][ik]][npw(ik)]  phi / H2phi / H3phi
All complex arrays are complex128 (interleaved re/im in memory).
"""
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import abi


@dataclass
class TCSystem:
    nr: tuple
    recip: np.ndarray          # (3,3) rows b_i
    lattice: np.ndarray        # (3,3) rows a_i
    omega: float
    method: str                # "HF" | "TC" | "BITC"
    nspin: int
    nsym_k: np.ndarray         # (nk_irr,) int32
    kvec: np.ndarray           # (nk_all,3) fractional
    time_rev: np.ndarray       # (nk_all,) uint8
    rot_index: np.ndarray      # (nk_all,) int32
    rotation: np.ndarray       # (nsymop,3,3) int32
    translation: np.ndarray    # (nsymop,3)
    num_kpoints: int
    npw: np.ndarray            # (nk_irr,) int32
    gindex: np.ndarray         # flat int32
    phase: np.ndarray          # flat complex128
    jastrow_A: np.ndarray      # (2,2)
    jastrow_F: np.ndarray      # (2,2)
    includes_div_correction: bool
    alpha_Vaux: float
    sum_Vaux: np.ndarray       # (nk_irr,)
    # state
    nbands: np.ndarray         # (nspin,) int32
    nocc: np.ndarray           # (nspin, nk_irr) int32
    filling: np.ndarray        # flat float64
    phik: np.ndarray           # flat complex128
    phik_left: Optional[np.ndarray]
    density: np.ndarray        # (2, N) complex128
    # trial block
    nb_apply: np.ndarray = None  # (nspin, nk_irr) int32
    psi: np.ndarray = None       # flat complex128
    name: str = ""
    meta: dict = field(default_factory=dict)

    # ---- sizes / offsets -------------------------------------------------
    @property
    def N(self):
        return int(self.nr[0] * self.nr[1] * self.nr[2])

    @property
    def nk_irr(self):
        return len(self.nsym_k)

    @property
    def nk_all(self):
        return int(np.sum(self.nsym_k))

    @property
    def kall_off(self):
        return np.concatenate([[0], np.cumsum(self.nsym_k)]).astype(np.int64)

    def gidx(self, s, a):
        """(gindex, phase) slices of spin s, all-k index a."""
        ik_of_all = np.repeat(np.arange(self.nk_irr), self.nsym_k)
        sizes = self.npw[ik_of_all].astype(np.int64)
        off = np.concatenate([[0], np.cumsum(np.tile(sizes, self.nspin))])
        o = off[s * self.nk_all + a]
        n = sizes[a]
        return self.gindex[o:o + n], self.phase[o:o + n]

    def _band_offsets(self, nb):
        off = {}
        o = 0
        for s in range(self.nspin):
            for k in range(self.nk_irr):
                off[(s, k)] = o
                o += int(nb[s][k]) * int(self.npw[k])
        return off, o

    def orb(self, s, k, b, left=False):
        nb = [[self.nbands[s]] * self.nk_irr for s in range(self.nspin)]
        off, _ = self._band_offsets(nb)
        arr = self.phik_left if (left and self.phik_left is not None) else self.phik
        o = off[(s, k)] + b * int(self.npw[k])
        return arr[o:o + int(self.npw[k])]

    def fill(self, s, k, b):
        o = sum(self.nk_irr * int(self.nbands[x]) for x in range(s))
        return float(self.filling[o + k * int(self.nbands[s]) + b])

    def psi_offsets(self):
        return self._band_offsets(self.nb_apply)

    def band_view(self, flat, s, k, b):
        off, _ = self.psi_offsets()
        o = off[(s, k)] + b * int(self.npw[k])
        return flat[o:o + int(self.npw[k])]

    def psi_size(self):
        return self._band_offsets(self.nb_apply)[1]

    def zeros_like_psi(self):
        return np.zeros(self.psi_size(), dtype=np.complex128)

    # ---- C descriptors ---------------------------------------------------
    def descriptors(self):
        """(SystemDesc, StateDesc, keepalive) for the C-ABI."""
        keep = []

        def c(arr, dtype):
            a = np.ascontiguousarray(arr, dtype=dtype)
            keep.append(a)
            return a

        sysd = abi.SystemDesc()
        sysd.nr[:] = [int(x) for x in self.nr]
        sysd.recip[:] = list(np.asarray(self.recip, dtype=np.float64).ravel())
        sysd.lattice[:] = list(np.asarray(self.lattice, dtype=np.float64).ravel())
        sysd.omega = float(self.omega)
        sysd.calc_method = abi.METHODS[self.method]
        sysd.nspin = int(self.nspin)
        sysd.nk_irr = int(self.nk_irr)
        sysd.num_kpoints = int(self.num_kpoints)
        import ctypes as C
        sysd.nsym_k = abi.ptr(c(self.nsym_k, np.int32), C.c_int32)
        sysd.kvec = abi.ptr(c(self.kvec, np.float64), C.c_double)
        sysd.time_rev = abi.ptr(c(self.time_rev, np.uint8), C.c_uint8)
        sysd.rot_index = abi.ptr(c(self.rot_index, np.int32), C.c_int32)
        sysd.nsymop = int(len(self.rotation))
        sysd.rotation = abi.ptr(c(self.rotation, np.int32), C.c_int32)
        sysd.translation = abi.ptr(c(self.translation, np.float64), C.c_double)
        sysd.npw = abi.ptr(c(self.npw, np.int32), C.c_int32)
        sysd.gindex = abi.ptr(c(self.gindex, np.int32), C.c_int32)
        sysd.phase = abi.ptr(c(self.phase, np.complex128).view(np.float64), C.c_double)
        sysd.jastrow_A[:] = list(np.asarray(self.jastrow_A, dtype=np.float64).ravel())
        sysd.jastrow_F[:] = list(np.asarray(self.jastrow_F, dtype=np.float64).ravel())
        sysd.includes_div_correction = int(bool(self.includes_div_correction))
        sysd.alpha_Vaux = float(self.alpha_Vaux)
        sysd.sum_Vaux = abi.ptr(c(self.sum_Vaux, np.float64), C.c_double)

        st = abi.StateDesc()
        st.nbands = abi.ptr(c(self.nbands, np.int32), C.c_int32)
        st.nocc = abi.ptr(c(self.nocc, np.int32), C.c_int32)
        st.filling = abi.ptr(c(self.filling, np.float64), C.c_double)
        st.phik = abi.ptr(c(self.phik, np.complex128).view(np.float64), C.c_double)
        if self.phik_left is not None and self.method == "BITC":
            st.phik_left = abi.ptr(c(self.phik_left, np.complex128).view(np.float64), C.c_double)
        else:
            st.phik_left = abi.ptr(None, C.c_double)
        st.density = abi.ptr(c(self.density, np.complex128).view(np.float64), C.c_double)
        return sysd, st, keep

    # ---- energy functional (total_energy.cpp:101-168) -------------------
    def energy_terms(self, h2=None, h3=None):
        """E_2, E_3 of the occupied orbitals from H2 psi / H3 psi where psi is
        the occupied set itself: e_n = <chi_i|H_n phi_i>, E = sum f e_n / N_k
        with weights 1/2 (two-body) and 1/3 (three-body); time-reversed
        partners contribute conj(e_n), all isym of a k the same e_n."""
        e2 = 0j
        e3 = 0j
        for s in range(self.nspin):
            for k in range(self.nk_irr):
                a0 = int(self.kall_off[k])
                for b in range(int(self.nb_apply[s][k])):
                    f = self.fill(s, k, b) if b < int(self.nbands[s]) else 0.0
                    if f == 0.0:
                        continue
                    chi = self.orb(s, k, b, left=True)
                    for isym in range(int(self.nsym_k[k])):
                        tr = bool(self.time_rev[a0 + isym])
                        if h2 is not None:
                            e = np.vdot(chi, self.band_view(h2, s, k, b))
                            e2 += f * (np.conj(e) if tr else e) / 2.0
                        if h3 is not None:
                            e = np.vdot(chi, self.band_view(h3, s, k, b))
                            e3 += f * (np.conj(e) if tr else e) / 3.0
        return e2 / self.num_kpoints, e3 / self.num_kpoints


@dataclass
class Pseudo:
    """Pseudopotential data as calc_hamiltonian::pseudo reads it
    (calc_hamiltonian_pseudo.cpp:6-180): local potential on the FFT grid,
    atoms, per-species projector l and D_ij, and per irreducible k the
    projector values <beta_{ip,m}|k+G> at the k's plane waves."""
    vloc: Optional[np.ndarray]          # (N,) float64 or None
    species_of_atom: np.ndarray         # (natoms,) int32
    atom_pos: np.ndarray                # (natoms, 3) Cartesian bohr
    lbeta: list                         # per species: list of l
    dij: list                           # per species: (nproj, nproj) float64
    projector: np.ndarray               # flat complex128 [nk][ncomp][npw_k]

    def descriptor(self):
        import ctypes as C
        c = lambda a, dt: np.ascontiguousarray(a, dtype=dt)
        keep = dict(vloc=None if self.vloc is None else c(self.vloc, np.float64),
                    sp=c(self.species_of_atom, np.int32), pos=c(self.atom_pos, np.float64),
                    nproj=c([len(l) for l in self.lbeta], np.int32),
                    lb=c([x for l in self.lbeta for x in l], np.int32),
                    dij=c(np.concatenate([np.asarray(d, dtype=np.float64).ravel() for d in self.dij]), np.float64),
                    proj=c(self.projector, np.complex128))
        d = abi.PseudoDesc()
        d.vloc = abi.ptr(keep["vloc"], C.c_double)
        d.nspecies = len(self.lbeta)
        d.natoms = len(self.species_of_atom)
        d.species_of_atom = abi.ptr(keep["sp"], C.c_int32)
        d.atom_pos = abi.ptr(keep["pos"], C.c_double)
        d.nproj = abi.ptr(keep["nproj"], C.c_int32)
        d.lbeta = abi.ptr(keep["lb"], C.c_int32)
        d.dij = abi.ptr(keep["dij"], C.c_double)
        d.projector = abi.ptr(keep["proj"].view(np.float64), C.c_double)
        return d, keep
