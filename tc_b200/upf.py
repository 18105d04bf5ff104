"""Norm-conserving pseudopotentials from UPF files, and the RPA Jastrow
parameters of a CASINO parameters.casl file, as TC++ prepares them for the
one-body and transcorrelated terms.  Host-side, once per run.

Follows:
  io_qe_files_read_upf.cpp:196-440     UPF v2 (and v1) reader: PP_R, PP_RAB, PP_LOCAL,
                                       PP_BETA.* with angular_momentum, PP_DIJ (row-major)
  potentials_pseudopot.cpp:10-24       Simpson's rule on the radial mesh with PP_RAB weights
  potentials_pseudopot.cpp:28-41       Rydberg -> Hartree (local potential and D_ij halved)
  potentials_pseudopot.cpp:44-142      local potential per species in G space: the
                                       long-range -Z erf(a r)/r is removed in r space and
                                       added back in G space, a = pi / cbrt(Omega)
  potentials_pseudopot.cpp:144-180     sum over atoms with exp(-i G.R), backward FFT, real part
  potentials_pseudopot.cpp:259-318     projector <beta Y_lm|k+G> without exp(i(k+G)R)
  calc_hamiltonian_pseudo.cpp:25-100   Y_lm(k+G) = prefactor P_l^m(cos theta) e^{i m phi}
  io_qmc_files_read_casl.cpp:160-196   RPA F per spin channel from parameters.casl
  jastrow_initialize.cpp:61-84         cusp condition: A_ss = F_ss^2 / 2, A_s s' = F_s s'^2
"""
import math
import os
import re

import numpy as np

from .system import Pseudo

FOURPI = 4.0 * math.pi


class UPF:
    """The fields of one UPF file that TC++ reads (Rydberg units as stored)."""

    def __init__(self, zval, r, rab, vloc_ry, beta, lbeta, dij_ry, element=""):
        self.zval = float(zval)
        self.r = np.asarray(r, dtype=np.float64)
        self.rab = np.asarray(rab, dtype=np.float64)
        self.vloc_ry = np.asarray(vloc_ry, dtype=np.float64)
        self.beta = np.asarray(beta, dtype=np.float64).reshape(len(lbeta), -1)
        self.lbeta = [int(x) for x in lbeta]
        self.dij_ry = np.asarray(dij_ry, dtype=np.float64).reshape(len(lbeta), len(lbeta))
        self.element = element

    # Hartree units (potentials_pseudopot.cpp:28-41)
    @property
    def vloc(self):
        return self.vloc_ry / 2.0

    @property
    def dij(self):
        return self.dij_ry / 2.0

    def arrays(self):
        return dict(zval=self.zval, r=self.r, rab=self.rab, vloc_ry=self.vloc_ry, beta=self.beta,
                    lbeta=np.array(self.lbeta, dtype=np.int32), dij_ry=self.dij_ry)

    @classmethod
    def from_arrays(cls, d, prefix=""):
        g = lambda k: d[prefix + k]
        return cls(float(g("zval")), g("r"), g("rab"), g("vloc_ry"), g("beta"), [int(x) for x in g("lbeta")],
                   g("dij_ry"))


def _attr(text, name):
    m = re.search(r'\b' + name + r'\s*=\s*"([^"]*)"', text)
    if m is None:
        raise ValueError(f"UPF: attribute {name} not found")
    return m.group(1).strip()


def _block(text, tag):
    """Numbers between <tag ...> and </tag>."""
    m = re.search(r"<" + re.escape(tag) + r"(\s[^>]*)?>(.*?)</" + re.escape(tag) + r">", text, re.S)
    if m is None:
        raise ValueError(f"UPF: {tag} not found")
    return m.group(1) or "", np.array(m.group(2).split(), dtype=np.float64)


def read_upf(path):
    """Read a norm-conserving UPF file (version 2 or 1).  Ultrasoft, PAW,
    Coulomb and non-linear-core-corrected potentials are rejected, as TC++
    rejects them."""
    with open(path) as f:
        text = f.read()
    first = text.lstrip().split("\n", 1)[0]
    if "qe_pp:pseudo" in first:
        raise ValueError("UPF with the XML schema is not supported")
    if "UPF" in first:                                             # version 2
        hm = re.search(r"<PP_HEADER(.*?)/?>", text, re.S)
        h = hm.group(1)
        ptype = _attr(h, "pseudo_type")
        flags = [_attr(h, k).upper() for k in ("is_ultrasoft", "is_paw", "is_coulomb")]
        if ptype in ("US", "PAW") or any(x in ("T", "TRUE", ".TRUE.") for x in flags):
            raise ValueError("ultrasoft, PAW and 1/r (is_coulomb) potentials are not supported")
        if _attr(h, "core_correction").upper() in ("T", "TRUE", ".TRUE."):
            raise ValueError("non-linear core correction is not supported")
        zval = float(_attr(h, "z_valence"))
        mesh = int(_attr(h, "mesh_size"))
        nproj = int(_attr(h, "number_of_proj"))
        element = _attr(h, "element")
        _, r = _block(text, "PP_R")
        _, rab = _block(text, "PP_RAB")
        _, vloc = _block(text, "PP_LOCAL")
        beta, lbeta = [], []
        for ip in range(nproj):
            attrs, b = _block(text, f"PP_BETA.{ip + 1}")
            lbeta.append(int(_attr(attrs, "angular_momentum")))
            if b.size < mesh:                      # trailing zeros may be omitted
                b = np.concatenate([b, np.zeros(mesh - b.size)])
            beta.append(b[:mesh])
        _, dij = _block(text, "PP_DIJ")
        dij = dij.reshape(nproj, nproj)
    else:                                                          # version 1
        lines = text.split("\n")
        i = next(j for j, s in enumerate(lines) if "<PP_HEADER>" in s)
        hdr = [s.split() for s in lines[i + 1:i + 12]]
        element = hdr[1][0]
        if hdr[2][0] != "NC":
            raise ValueError("ultrasoft, PAW and 1/r potentials are not supported")
        if hdr[3][0].upper() in ("T", ".TRUE."):
            raise ValueError("non-linear core correction is not supported")
        zval = float(hdr[5][0])
        mesh = int(hdr[9][0])
        nproj = int(hdr[10][1])
        _, r = _block(text, "PP_R")
        _, rab = _block(text, "PP_RAB")
        _, vloc = _block(text, "PP_LOCAL")
        beta, lbeta = [], []
        for m in re.finditer(r"<PP_BETA>(.*?)</PP_BETA>", text, re.S):
            body = m.group(1).strip().split("\n")
            lbeta.append(int(body[0].split()[1]))
            vals = np.array(" ".join(body[2:]).split(), dtype=np.float64)
            b = np.zeros(mesh)
            b[:min(mesh, vals.size)] = vals[:mesh]
            beta.append(b)
        _, d = _block(text, "PP_DIJ")
        nnz = int(d[0])
        dij = np.zeros((nproj, nproj))
        for e in d[1:1 + 3 * nnz].reshape(nnz, 3):
            dij[int(e[0]) - 1, int(e[1]) - 1] = e[2]
    if r.size != mesh or rab.size != mesh or vloc.size != mesh or len(beta) != nproj:
        raise ValueError("UPF: inconsistent mesh or projector count")
    return UPF(zval, r, rab, vloc, beta, lbeta, dij, element=element)


def simpson_weights(rab):
    """Coefficients c with Potentials::simpson(f) = sum_i c_i f_i
    (potentials_pseudopot.cpp:10-24: pairs of intervals, weight rab)."""
    n = rab.size
    c = np.zeros(n)
    for i in range(0, n - 2, 2):
        c[i] += 1.0
        c[i + 1] += 4.0
        c[i + 2] += 1.0
    return c * rab / 3.0


def _sinc_series(x):
    """sin(x)/x by the nested series of potentials_pseudopot.cpp:106-113 (x <= 0.1)."""
    t = 1.0 - x * x / 110.0
    t = 1.0 - t * x * x / 72.0
    t = 1.0 - t * x * x / 42.0
    t = 1.0 - t * x * x / 20.0
    return 1.0 - t * x * x / 6.0


def fft_miller(nr):
    """Miller indices of every FFT grid point, x fastest, wrapped into
    (-(n+1)/2, n/2] (PlaneWaveBasis::get_Gvector, plane_wave_basis.cpp:205-216)."""
    n0, n1, n2 = nr
    idx = np.arange(n0 * n1 * n2)
    m = np.stack([idx % n0, (idx // n0) % n1, idx // (n0 * n1)], 1)
    n = np.array(nr)
    return np.where(m > n // 2, m - n, m)


def vloc_atom_g(upf, gnorm, omega):
    """FT of one species' local potential at |G| values (Hartree), with
    the G = 0 convention of potentials_pseudopot.cpp:115-141."""
    a = math.pi / np.cbrt(omega)
    r = upf.r
    z = upf.zval
    short = np.where(r > 1e-8, upf.vloc + z / np.where(r > 1e-8, r, 1.0) * _erf(a * r),
                     upf.vloc + z * 2.0 * a / math.sqrt(math.pi))
    w = simpson_weights(upf.rab)
    uniq, inv = np.unique(gnorm, return_inverse=True)
    out = np.empty(uniq.size)
    for i0 in range(0, uniq.size, 256):
        g = uniq[i0:i0 + 256, None]
        gr = g * r[None, :]
        sinc = np.where(gr > 0.1, np.sin(gr) / np.where(gr > 0.1, gr, 1.0), _sinc_series(gr))
        out[i0:i0 + 256] = (sinc * (short * r * r)[None, :]) @ w
    g2 = uniq * uniq
    with np.errstate(divide="ignore", invalid="ignore"):
        tail = np.where(g2 > 0, -z * np.exp(-g2 / (4 * a * a)) / np.where(g2 > 0, g2, 1.0), z / (4 * a * a))
    return ((out + tail) * (FOURPI / omega))[inv]


def _erf(x):
    from math import erf
    return np.vectorize(erf, otypes=[np.float64])(x)


def vpp_local(nr, recip, omega, upfs, species_of_atom, atom_pos):
    """Potentials::Vpp_local on the FFT grid (real, R space): the species'
    local potentials in G space, summed over atoms with exp(-i G.R_atom),
    transformed backward (unscaled) and the real part kept.  G = 0 of every
    FFT grid point is treated as the reference does (index 0 only)."""
    mil = fft_miller(nr).astype(np.float64)
    G = mil @ np.asarray(recip, dtype=np.float64)
    gnorm = np.sqrt(np.einsum("ij,ij->i", G, G))
    gnorm[0] = 0.0
    vg = np.zeros(G.shape[0], dtype=np.complex128)
    per_species = {}
    for ia, isp in enumerate(species_of_atom):
        if isp not in per_species:
            per_species[isp] = vloc_atom_g(upfs[isp], gnorm, omega)
        gr = G @ np.asarray(atom_pos[ia], dtype=np.float64)
        vg += (np.cos(gr) - 1j * np.sin(gr)) * per_species[isp]
    n0, n1, n2 = nr
    grid = vg.reshape(n2, n1, n0)
    vr = np.fft.ifftn(grid) * (n0 * n1 * n2)       # backward: sum_G V(G) e^{+iG.r}
    return np.ascontiguousarray(vr.real.ravel())


def _ylm(kg, lmax):
    """Y_lm(e_{k+G}) for m = 0..l as calc_hamiltonian_pseudo.cpp:25-100
    (Condon-Shortley phase of the associated Legendre function included)."""
    from scipy.special import lpmv
    q = np.linalg.norm(kg, axis=1)
    small = q < 1e-8
    qs = np.where(small, 1.0, q)
    cos_t = kg[:, 2] / qs
    rsin = np.sqrt(kg[:, 0] ** 2 + kg[:, 1] ** 2)
    phase = np.where(rsin > 1e-8, (kg[:, 0] + 1j * kg[:, 1]) / np.where(rsin > 1e-8, rsin, 1.0), 1.0)
    y = []
    for l in range(lmax + 1):
        row = []
        for m in range(l + 1):
            pref = math.sqrt((2 * l + 1) * math.factorial(l - m) / (FOURPI * math.factorial(l + m)))
            v = pref * lpmv(m, l, cos_t) * phase ** m
            v = np.where(small, (1.0 / math.sqrt(FOURPI)) if l == 0 else 0.0, v)
            row.append(v.astype(np.complex128))
        y.append(row)
    return y


def projectors_at_k(upf, kvec, miller, recip, omega):
    """Potentials::projector_nonlocal for every projector of one species at
    one k: list over projectors of arrays [2l+1][npw], m index ordered as the
    reference (l - m <- conj(Y_lm), l <- Y_l0, l + m <- Y_lm)."""
    from scipy.special import spherical_jn
    kg = (np.asarray(kvec, dtype=np.float64)[None, :] + miller) @ np.asarray(recip, dtype=np.float64)
    q = np.linalg.norm(kg, axis=1)
    lmax = max(upf.lbeta) if upf.lbeta else 0
    if lmax > 3:
        raise ValueError("projectors with l > 3 are not supported")
    y = _ylm(kg, lmax)
    w = simpson_weights(upf.rab)
    fac = FOURPI / math.sqrt(omega)
    out = []
    for ip, l in enumerate(upf.lbeta):
        f = upf.r * upf.beta[ip]                       # UPF stores r * beta
        bj = fac * (spherical_jn(l, q[:, None] * upf.r[None, :]) * f[None, :]) @ w
        comp = np.zeros((2 * l + 1, q.size), dtype=np.complex128)
        comp[l] = y[l][0] * bj
        for m in range(1, l + 1):
            comp[l - m] = np.conj(y[l][m]) * bj
            comp[l + m] = y[l][m] * bj
        out.append(comp)
    return out


def pseudo_from_upf(system, upfs, species_of_atom, atom_pos):
    """tc_b200.system.Pseudo of a system from its species' UPF data:
    Vpp_local on the FFT grid and, per irreducible k, the projectors at the
    plane waves of the k's first (isym 0) entry."""
    nr = tuple(int(x) for x in system.nr)
    recip = np.asarray(system.recip, dtype=np.float64)
    vloc = vpp_local(nr, recip, system.omega, upfs, species_of_atom, atom_pos)
    n = np.array(nr)
    proj = []
    nspecies = len(upfs)
    for k in range(system.nk_irr):
        a0 = int(system.kall_off[k])
        gi, _ = system.gidx(0, a0)
        w = np.stack([gi % n[0], (gi // n[0]) % n[1], gi // (n[0] * n[1])], 1)
        mil = np.where(w > n // 2, w - n, w).astype(np.float64)
        comps = []
        for isp in range(nspecies):
            for c in projectors_at_k(upfs[isp], system.kvec[a0], mil, recip, system.omega):
                comps.append(c)
        proj.append(np.concatenate(comps).ravel() if comps else np.zeros(0, dtype=np.complex128))
    return Pseudo(vloc=vloc, species_of_atom=np.asarray(species_of_atom, dtype=np.int32),
                  atom_pos=np.asarray(atom_pos, dtype=np.float64), lbeta=[list(u.lbeta) for u in upfs],
                  dij=[u.dij for u in upfs], projector=np.concatenate(proj))


def read_casl_rpa(path, nspin=1):
    """RPA F parameters of a CASINO parameters.casl file (first TERM) and
    the A parameters the cusp condition gives: returns (A, F) as 2x2."""
    with open(path) as f:
        text = f.read()
    vals = {}
    for ch in ("1-1", "1-2", "2-2"):
        m = re.search(r"Channel\s+" + ch + r"\s*:\s*\n\s*F\s*:\s*\[\s*([-+0-9.eEdD]+)", text)
        if m:
            vals[ch] = float(m.group(1).replace("d", "e").replace("D", "e"))
    if "1-1" not in vals or "1-2" not in vals:
        raise ValueError("parameters.casl: RPA F of channels 1-1 and 1-2 not found")
    f22 = vals["1-1"] if nspin == 1 else vals["2-2"]
    F = np.array([[vals["1-1"], vals["1-2"]], [vals["1-2"], f22]])
    A = np.array([[F[0, 0] ** 2 / 2.0, F[0, 1] ** 2], [F[1, 0] ** 2, F[1, 1] ** 2 / 2.0]])
    return A, F


def species_and_positions(qe):
    """(species index per atom, Cartesian positions in bohr, species names)
    of a tc_b200.qe.QEData, species in order of first appearance."""
    names = []
    sp = []
    for name, _ in qe.atoms:
        if name not in names:
            names.append(name)
        sp.append(names.index(name))
    pos = np.array([p for _, p in qe.atoms], dtype=np.float64)
    return np.array(sp, dtype=np.int32), pos, names


def find_upf(save_dir, element):
    for f in sorted(os.listdir(save_dir)):
        if f.lower().endswith(".upf") and (element.lower() in f.lower()):
            return os.path.join(save_dir, f)
    raise FileNotFoundError(f"no UPF file for {element} in {save_dir}")
