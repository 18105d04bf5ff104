"""Seeded synthetic inputs with the shapes of the benchmark configurations.

No public benchmark suite exists for this path; every input is generated
here with numpy.random.default_rng(seed):

  C1  hf2x, fcc Si a=10.26, 2x2x2 MP (8 k), 1/2|k+G|^2 < 10 Ha, grid 24^3,
      4 occupied + 8 trial bands, complex128
  C2  TC (tc2x + tc3*), same cell / k, RPA A=0.5 F=1.2, grid 32^3, 4 occ + 4 trial
  C3  BITC batched, 4x4x4 MP (64 k), 14 Ha, grid 36^3, 16 bands (4 occ),
      independent left / right orbitals, left bi-orthonormalised to right
  C3s C3 on a 2x2x2 MP mesh (8 k): the reduced case for profiler captures
  C4  HEG, simple cubic, 54 e- at r_s = 2, Gamma only, 27 occupied plane-wave
      shells + 27 trial, 1e-3 seeded noise, grid 40^3
  C5  conventional cubic Si8 a=10.26, 3x3x3 MP (27 k), 20 Ha, grid 48^3,
      16 occ + 32 trial

Helper conventions follow TC++: k fractional, Cartesian = recip^T k
(crystal_structure.hpp:16), Gindex wraps Miller indices into [0, n)
(plane_wave_basis.cpp:118-131), backward FFT unscaled.
"""
import numpy as np

from .system import Pseudo, TCSystem

FOURPI = 4.0 * np.pi


# ---------------------------------------------------------------- cells ----
def lattice_fcc(a):
    return (a / 2.0) * np.array([[-1.0, 0.0, 1.0], [0.0, 1.0, 1.0], [-1.0, 1.0, 0.0]])


def lattice_sc(a):
    return a * np.eye(3)


def recip_of(lattice):
    """rows b_i with lattice . recip^T = 2 pi I."""
    return 2.0 * np.pi * np.linalg.inv(lattice).T


def mp_mesh(n):
    """Gamma-centred n x n x n Monkhorst-Pack mesh, fractional."""
    g = np.arange(n) / n
    return np.array([[x, y, z] for x in g for y in g for z in g], dtype=np.float64)


def pw_sphere(recip, k, ecut, nr):
    """Miller indices m with 1/2 |recip^T (k+m)|^2 < ecut, sorted by |k+G|^2
    then lexicographically.  Raises if the sphere does not fit the FFT box."""
    lim = [nr[d] // 2 for d in range(3)]
    rng = [np.arange(-((nr[d] - 1) // 2), lim[d] + 1) for d in range(3)]
    M = np.stack(np.meshgrid(*rng, indexing="ij"), -1).reshape(-1, 3)
    G = (k[None, :] + M) @ recip
    e = 0.5 * np.einsum("ij,ij->i", G, G)
    sel = e < ecut
    M, e = M[sel], e[sel]
    for d in range(3):
        if np.any(np.abs(M[:, d]) >= nr[d] / 2.0):
            raise ValueError("plane-wave sphere does not fit the FFT grid")
    order = np.lexsort((M[:, 2], M[:, 1], M[:, 0], np.round(e, 12)))
    return M[order].astype(np.int64)


def gindex_of(M, nr):
    w = np.mod(M, np.array(nr))
    return (w[:, 0] + nr[0] * (w[:, 1] + nr[1] * w[:, 2])).astype(np.int32)


def gram_schmidt(X):
    """modified Gram-Schmidt on the columns of X (npw x nb)."""
    Q = X.astype(np.complex128).copy()
    for i in range(Q.shape[1]):
        for j in range(i):
            Q[:, i] -= np.vdot(Q[:, j], Q[:, i]) * Q[:, j]
        Q[:, i] /= np.linalg.norm(Q[:, i])
    return Q


def biorthonormalise(X, Phi):
    """X <- X (Phi^H X)^{-1} so that X^H Phi = I (<chi_i|phi_j> = delta_ij)."""
    S = Phi.conj().T @ X
    return X @ np.linalg.inv(S)


# ------------------------------------------------------ divergence sums ---
def sum_of_vaux(recip, omega, kvec_irr, kvec_all):
    """Potentials::set_sum_of_Vaux_each on the SCF mesh
    (potentials_coulomb.cpp:60-161): shell sums to 1e-20 per (k, q)."""
    alpha = (np.cbrt(omega) / (2.0 * np.pi)) ** 2
    out = np.zeros(len(kvec_irr))
    cache = {}
    for ik, kr in enumerate(kvec_irr):
        total = 0.0
        match = False
        for q in kvec_all:
            kq = kr - q
            for d in range(3):
                while kq[d] < -1e-8:
                    kq[d] += 1.0
                while kq[d] > 1.0 - 1e-8:
                    kq[d] -= 1.0
            m = float(kq @ kq) < 1e-8
            match = match or m
            key = tuple(np.round(kq, 12))
            if key not in cache:
                acc = 0.0
                if not m:
                    v = kq @ recip
                    k2 = float(v @ v)
                    acc += np.exp(-alpha * k2) / k2
                ns = 1
                while True:
                    r = np.arange(-ns, ns + 1)
                    g = np.stack(np.meshgrid(r, r, r, indexing="ij"), -1).reshape(-1, 3)
                    g = g[np.max(np.abs(g), axis=1) == ns]
                    v = (kq[None, :] + g) @ recip
                    g2 = np.einsum("ij,ij->i", v, v)
                    shell = float(np.sum(np.exp(-alpha * g2) / g2))
                    acc += shell
                    if shell < 1e-20:
                        break
                    ns += 1
                cache[key] = acc
            total += cache[key]
        total *= FOURPI
        if match:
            total -= FOURPI * alpha
        out[ik] = total
    return alpha, out


# ------------------------------------------------------------- density ---
def density_numpy(sysm):
    """BlochStates::set_density (first iteration) with numpy FFTs."""
    n0, n1, n2 = sysm.nr
    N = sysm.N
    dens = np.zeros((2, N), dtype=np.complex128)
    koff = sysm.kall_off
    for s in range(sysm.nspin):
        acc = np.zeros(N, dtype=np.complex128)
        for k in range(sysm.nk_irr):
            for isym in range(int(sysm.nsym_k[k])):
                a = int(koff[k] + isym)
                gi, ph = sysm.gidx(s, a)
                tr = bool(sysm.time_rev[a])
                for b in range(int(sysm.nocc[s][k])):
                    def to_r(c):
                        g = np.zeros(N, dtype=np.complex128)
                        g[gi] = (np.conj(c) if tr else c) * ph
                        return (np.fft.ifftn(g.reshape(n2, n1, n0)) * N).ravel()
                    r = to_r(sysm.orb(s, k, b))
                    if sysm.method == "BITC":
                        sub = np.conj(to_r(sysm.orb(s, k, b, left=True))) * r
                    else:
                        sub = np.abs(r) ** 2
                    acc += sysm.fill(s, k, b) * sub
        if sysm.nspin == 1:
            acc /= 2.0
        dens[s] = acc
    if sysm.nspin == 1:
        dens[1] = dens[0]
    return dens


# ------------------------------------------------------------ builder ----
def _tr_invariant(k):
    return np.allclose(np.mod(2 * np.asarray(k), 1.0), 0.0) or np.allclose(np.mod(2 * np.asarray(k), 1.0), 1.0)


def _tr_symmetrise(X, M, k):
    """Make a time-reversal-invariant k-point's orbitals closed under
    conjugation: c(m') = conj(c(m)) with k + m' = -(k + m), so that the state
    is invariant under the time reversal the reduced k-set relies on."""
    shift = np.rint(-2 * np.asarray(k)).astype(np.int64)
    pos = {tuple(m): i for i, m in enumerate(M)}
    idx = np.array([pos[tuple(shift - m)] for m in M])
    return 0.5 * (X + np.conj(X[idx]))



def build(lattice, kvec_irr, ecut, nr, nbands, nocc, method, *, seed=0, left_seed=None,
          A=0.5, F=1.2, nspin=1, tr_partner=None, name="", heg_orbitals=None,
          includes_div_correction=True, nb_apply=None):
    """Assemble a TCSystem.

    tr_partner: optional list, per irreducible k, of True if the k-point has a
    time-reversal partner -k appended as isym = 1 (identity rotation with
    time reversal, Kpoints::set_kvectors_by_symmetry, kpoints.cpp:37-67).
    heg_orbitals: optional callable(k_index, M) -> (npw x nbands) coefficients.
    """
    nr = tuple(int(x) for x in nr)
    recip = recip_of(lattice)
    omega = abs(np.linalg.det(lattice))
    nk = len(kvec_irr)
    tr_partner = tr_partner or [False] * nk
    nsym_k = np.array([2 if t else 1 for t in tr_partner], dtype=np.int32)
    kvec_all, time_rev, rot_index = [], [], []
    for k, t in zip(kvec_irr, tr_partner):
        kvec_all.append(np.array(k, dtype=np.float64))
        time_rev.append(0)
        rot_index.append(0)
        if t:
            kvec_all.append(-np.array(k, dtype=np.float64))
            time_rev.append(1)
            rot_index.append(0)
    kvec_all = np.array(kvec_all)
    rng = np.random.default_rng(seed)
    lrng = np.random.default_rng(left_seed) if left_seed is not None else None

    npw, gidx_list, phase_list, phik, phik_left = [], [], [], [], []
    mills = []
    for ik, k in enumerate(kvec_irr):
        M = pw_sphere(recip, np.asarray(k, dtype=np.float64), ecut, nr)
        mills.append(M)
        npw.append(len(M))
        gidx_list.append(gindex_of(M, nr))
        phase_list.append(np.ones(len(M), dtype=np.complex128))
        if tr_partner[ik]:
            gidx_list.append(gindex_of(-M, nr))
            phase_list.append(np.ones(len(M), dtype=np.complex128))
        G = (np.asarray(k)[None, :] + M) @ recip
        env = np.exp(-np.einsum("ij,ij->i", G, G) / 8.0)
        if heg_orbitals is not None:
            X = heg_orbitals(ik, M, rng)
        else:
            X = (rng.standard_normal((len(M), nbands)) + 1j * rng.standard_normal((len(M), nbands))) * env[:, None]
        if tr_partner[ik] is False and any(tr_partner) and _tr_invariant(k):
            X = _tr_symmetrise(X, M, k)
        Phi = gram_schmidt(X)
        phik.append(Phi)
        if method == "BITC":
            if lrng is not None:
                Xl = (lrng.standard_normal((len(M), nbands)) + 1j * lrng.standard_normal((len(M), nbands))) * env[:, None]
                if tr_partner[ik] is False and any(tr_partner) and _tr_invariant(k):
                    Xl = _tr_symmetrise(Xl, M, k)
                Chi = biorthonormalise(gram_schmidt(Xl), Phi)
            else:
                Chi = Phi.copy()
            phik_left.append(Chi)

    npw = np.array(npw, dtype=np.int32)
    gindex = np.concatenate([np.concatenate(gidx_list)] * nspin).astype(np.int32)
    phase = np.concatenate([np.concatenate(phase_list)] * nspin)
    flat = lambda L: np.concatenate([np.ascontiguousarray(P.T).ravel() for P in L])
    phik_flat = np.concatenate([flat(phik)] * nspin)
    left_flat = np.concatenate([flat(phik_left)] * nspin) if method == "BITC" else None
    fillv = 2.0 if nspin == 1 else 1.0
    filling = np.zeros((nspin, nk, nbands))
    filling[:, :, :nocc] = fillv
    alpha, sumv = sum_of_vaux(recip, omega, np.asarray(kvec_irr, dtype=np.float64), kvec_all)
    Aarr = np.full((2, 2), float(A)) if np.isscalar(A) else np.asarray(A, dtype=np.float64)
    Farr = np.full((2, 2), float(F)) if np.isscalar(F) else np.asarray(F, dtype=np.float64)
    if method == "HF":
        Aarr = np.zeros((2, 2))
        Farr = np.ones((2, 2))
    sysm = TCSystem(
        nr=nr, recip=recip, lattice=np.asarray(lattice, dtype=np.float64), omega=float(omega),
        method=method, nspin=nspin, nsym_k=nsym_k, kvec=kvec_all,
        time_rev=np.array(time_rev, dtype=np.uint8), rot_index=np.array(rot_index, dtype=np.int32),
        rotation=np.eye(3, dtype=np.int32)[None], translation=np.zeros((1, 3)),
        num_kpoints=int(len(kvec_all)), npw=npw, gindex=gindex, phase=phase,
        jastrow_A=Aarr, jastrow_F=Farr, includes_div_correction=includes_div_correction,
        alpha_Vaux=float(alpha), sum_Vaux=sumv,
        nbands=np.full(nspin, nbands, dtype=np.int32), nocc=np.full((nspin, nk), nocc, dtype=np.int32),
        filling=filling.ravel(), phik=phik_flat, phik_left=left_flat,
        density=np.zeros((2, int(np.prod(nr))), dtype=np.complex128), name=name,
    )
    sysm.meta["mills"] = mills
    sysm.density = density_numpy(sysm)
    nb = nbands if nb_apply is None else nb_apply
    sysm.nb_apply = np.full((nspin, nk), nb, dtype=np.int32)
    # trial block = first nb bands of the right orbitals (occupied + trial)
    psi = []
    for s in range(nspin):
        for k in range(nk):
            psi.append(np.ascontiguousarray(phik[k][:, :nb].T).ravel())
    sysm.psi = np.concatenate(psi)
    return sysm


# ------------------------------------------------------------- configs ---
def config(name, **over):
    """The five benchmark configurations plus small test variants."""
    a = 10.26
    if name == "C1":
        kw = dict(lattice=lattice_fcc(a), kvec_irr=mp_mesh(2), ecut=10.0, nr=(24, 24, 24),
                  nbands=12, nocc=4, method="HF", seed=0)
    elif name == "C2":
        kw = dict(lattice=lattice_fcc(a), kvec_irr=mp_mesh(2), ecut=10.0, nr=(32, 32, 32),
                  nbands=8, nocc=4, method="TC", seed=0, A=0.5, F=1.2)
    elif name == "C3":
        kw = dict(lattice=lattice_fcc(a), kvec_irr=mp_mesh(4), ecut=14.0, nr=(36, 36, 36),
                  nbands=16, nocc=4, method="BITC", seed=2, left_seed=1, A=0.5, F=1.2)
    elif name == "C3s":
        # C3's cell, cutoff, grid, bands and Jastrow on a 2x2x2 mesh (8 k): the
        # same kernels at an eighth of the k-points, small enough for ncu captures
        kw = dict(lattice=lattice_fcc(a), kvec_irr=mp_mesh(2), ecut=14.0, nr=(36, 36, 36),
                  nbands=16, nocc=4, method="BITC", seed=2, left_seed=1, A=0.5, F=1.2)
    elif name == "C4":
        return heg_config(**over)
    elif name == "C5":
        kw = dict(lattice=lattice_sc(a), kvec_irr=mp_mesh(3), ecut=20.0, nr=(48, 48, 48),
                  nbands=48, nocc=16, method="TC", seed=0, A=0.5, F=1.2)
    else:
        raise KeyError(name)
    kw.update(over)
    return build(name=name, **kw)


def heg_config(rs=2.0, nelec=54, nr=(40, 40, 40), nocc=27, ntrial=27, noise=1e-3, seed=0,
               method="BITC", **over):
    """Homogeneous electron gas, simple cubic, Gamma only (C4)."""
    omega = nelec * (4.0 * np.pi / 3.0) * rs ** 3
    L = np.cbrt(omega)
    lattice = lattice_sc(L)
    nb = nocc + ntrial
    recip = recip_of(lattice)
    # plane-wave basis: all |m|^2 <= 12 ; orbitals are the lowest shells
    ecut = 0.5 * (2 * np.pi / L) ** 2 * 12.5

    def orbitals(ik, M, rng):
        m2 = np.einsum("ij,ij->i", M, M)
        order = np.lexsort((M[:, 2], M[:, 1], M[:, 0], m2))
        X = np.zeros((len(M), nb), dtype=np.complex128)
        for b in range(nb):
            X[order[b], b] = 1.0
        X += noise * (rng.standard_normal(X.shape) + 1j * rng.standard_normal(X.shape))
        return X

    # RPA default of TC++: A = sqrt(V / (4 pi N)), F from the cusp condition
    # (jastrow_initialize.cpp:28-51, :61-76)
    A0 = np.sqrt(omega / (FOURPI * nelec))
    A = np.full((2, 2), A0)
    F = np.array([[np.sqrt(2 * A0), np.sqrt(A0)], [np.sqrt(A0), np.sqrt(2 * A0)]])
    kw = dict(lattice=lattice, kvec_irr=np.zeros((1, 3)), ecut=ecut, nr=nr, nbands=nb, nocc=nocc,
              method=method, seed=seed, A=A, F=F, heg_orbitals=orbitals)
    kw.update(over)
    s = build(name="C4", **kw)
    s.meta["recip"] = recip
    return s


def small(method="TC", nr=(12, 12, 12), nk=2, ecut=2.5, nbands=3, nocc=2, seed=0, nspin=1,
          tr=False, **over):
    """Small fcc-Si case the CPU oracle finishes in seconds."""
    if tr:
        # 3x3x3 mesh reduced by time reversal: Gamma + 13 (k, -k) pairs
        full = mp_mesh(3)
        irr, partner = [], []
        seen = set()
        for k in full:
            key = tuple(np.round(np.mod(k, 1.0), 6))
            mkey = tuple(np.round(np.mod(-k, 1.0), 6))
            if key in seen:
                continue
            seen.add(key)
            seen.add(mkey)
            irr.append(k)
            partner.append(mkey != key)
        kvec = np.array(irr)
        kw = dict(tr_partner=partner)
    else:
        kvec = mp_mesh(nk)
        kw = {}
    A = over.pop("A", 0.5)
    F = over.pop("F", 1.2)
    kw.update(over)
    return build(lattice=lattice_fcc(10.26), kvec_irr=kvec, ecut=ecut, nr=nr, nbands=nbands,
                 nocc=nocc, method=method, seed=seed, left_seed=(seed + 101 if method == "BITC" else None),
                 A=A, F=F, nspin=nspin, name=f"small-{method}", **kw)


def pseudo(sysm, seed=0, with_local=True):
    """Synthetic pseudopotential with the shape of the reference's Si test
    potential (one species, two projectors with l = 0 and l = 1, D_ij diagonal
    in l; test/example*/Si_test.upf has 2 projectors): smooth seeded radial
    factors times real spherical harmonics of k+G, atoms at (0,0,0) and
    (1/4,1/4,1/4) of the cell, and a smooth real local potential."""
    rng = np.random.default_rng(seed)
    frac = np.array([[0.0, 0.0, 0.0], [0.25, 0.25, 0.25]])
    pos = frac @ np.asarray(sysm.lattice)
    lbeta = [[0, 1]]
    d = rng.standard_normal(2)
    dij = [np.diag(d)]
    radial = rng.uniform(0.5, 1.5, size=2)
    proj = []
    mills = sysm.meta.get("mills")
    for k in range(sysm.nk_irr):
        gi, _ = sysm.gidx(0, int(sysm.kall_off[k]))
        n = np.array(sysm.nr)
        w = np.stack([gi % n[0], (gi // n[0]) % n[1], gi // (n[0] * n[1])], 1)
        m = np.where(w > n // 2, w - n, w)
        kg = (np.asarray(sysm.kvec[int(sysm.kall_off[k])])[None, :] + m) @ np.asarray(sysm.recip)
        q = np.linalg.norm(kg, axis=1)
        qs = np.where(q > 1e-12, q, 1.0)
        comps = [np.exp(-radial[0] * q ** 2 / 4) / np.sqrt(FOURPI) + 0j]                   # l = 0
        f1 = q * np.exp(-radial[1] * q ** 2 / 4) * np.sqrt(3.0 / FOURPI)
        for dd in range(3):                                                             # l = 1, m = x, y, z
            comps.append(-1j * f1 * kg[:, dd] / qs)
        proj.append(np.stack(comps).ravel())
    vloc = None
    if with_local:
        N = sysm.N
        x = np.arange(N)
        n0, n1, n2 = sysm.nr
        i0, i1, i2 = x % n0, (x // n0) % n1, x // (n0 * n1)
        vloc = np.zeros(N)
        for _ in range(4):
            h = rng.integers(-2, 3, size=3)
            vloc += rng.standard_normal() * np.cos(2 * np.pi * (h[0] * i0 / n0 + h[1] * i1 / n1 + h[2] * i2 / n2)
                                                   + rng.uniform(0, 2 * np.pi))
    return Pseudo(vloc=vloc, species_of_atom=np.zeros(2, dtype=np.int32), atom_pos=pos, lbeta=lbeta, dij=dij,
                  projector=np.concatenate(proj))
