"""Python host API of the B200 operator library (ctypes over include/tcg.h).

    ctx = Context(system, precision="fp64")   # or "mixed"
    ctx.set_state(system)                     # once per SCF iteration
    h2, h3 = ctx.apply(TERMS_TC, psi)         # accumulates like TC++ (H += ...)

There is no CPU path: without the CUDA library or a GPU every call raises
TCError.
"""
import ctypes as C

import numpy as np

from . import abi
from ._lib import TCError, check, lib

PRECISIONS = {"fp64": abi.PREC_FP64, "mixed": abi.PREC_MIXED}


def _terms(terms):
    if isinstance(terms, int):
        return terms
    if isinstance(terms, str):
        terms = [terms]
    m = 0
    for t in terms:
        m |= abi.TERM_NAMES[t] if t in abi.TERM_NAMES else abi.TERM_NAMES_EXTRA[t]
    return m


class Context:
    def __init__(self, system, precision="fp64", tmp_budget=None):
        self.system = system
        self.precision = precision
        self._sysd, _, self._keep = system.descriptors()
        h = C.c_void_p()
        check(lib().tcg_ctx_create(C.byref(self._sysd), PRECISIONS[precision], C.byref(h)))
        self._h = h
        if tmp_budget:
            check(lib().tcg_set_tuning(self._h, int(tmp_budget)))
        self._state_keep = None

    # -- life cycle ---------------------------------------------------------
    def close(self):
        if self._h:
            lib().tcg_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        if not self._h:
            raise TCError(abi.TCG_ERR_STATE, "context closed")
        return self._h

    @property
    def launches(self):
        return int(lib().tcg_launch_count(self.handle))

    @property
    def stream(self):
        return lib().tcg_stream(self.handle)

    def set_tuning(self, tmp_budget):
        check(lib().tcg_set_tuning(self.handle, int(tmp_budget)))

    def forms(self):
        """The kernel forms in use (tcg_get_forms) as a dict."""
        f = abi.Forms()
        check(lib().tcg_get_forms(self.handle, C.byref(f)))
        return {n: int(getattr(f, n)) for n, _ in abi.Forms._fields_}

    def set_forms(self, **kw):
        """Change some kernel forms (tcg_set_forms); the others keep their value."""
        cur = self.forms()
        unknown = set(kw) - set(cur)
        if unknown:
            raise KeyError(f"unknown kernel forms {sorted(unknown)}")
        cur.update({k: int(v) for k, v in kw.items()})
        f = abi.Forms(**cur)
        check(lib().tcg_set_forms(self.handle, C.byref(f)))

    # -- state ----------------------------------------------------------------
    def set_state(self, system=None):
        s = system or self.system
        _, st, keep = s.descriptors()
        check(lib().tcg_set_state(self.handle, C.byref(st)))
        self._state_keep = keep

    def refresh_state(self):
        check(lib().tcg_refresh_state(self.handle))

    def profile(self, enable=True):
        check(lib().tcg_profile(self.handle, 1 if enable else 0))

    def profile_read(self):
        """{tag: (launches, device ms, algorithmic bytes)} of recorded launches; "idle>tag"
        entries hold the device time between the previous launch and each launch of tag."""
        cap = 128
        tags = C.create_string_buffer(32 * cap)
        cnt = (C.c_int64 * cap)()
        ms = (C.c_double * cap)()
        by = (C.c_double * cap)()
        n = C.c_int()
        check(lib().tcg_profile_read(self.handle, cap, tags, cnt, ms, by, C.byref(n)))
        out = {}
        for i in range(n.value):
            t = tags.raw[32 * i:32 * i + 32].split(b"\0")[0].decode()
            out[t] = (int(cnt[i]), float(ms[i]), float(by[i]))
        return out

    def density(self, system=None):
        s = system or self.system
        _, st, keep = s.descriptors()
        st.density = abi.ptr(None, C.c_double)
        out = np.zeros((2, s.N), dtype=np.complex128)
        check(lib().tcg_density(self.handle, C.byref(st), out.ctypes.data))
        return out

    # -- apply ------------------------------------------------------------------
    def apply(self, terms, psi=None, nb_apply=None, h2=None, h3=None, owned=None):
        """Host-memory apply; returns (h2, h3) with h += terms(psi)."""
        s = self.system
        mask = _terms(terms)
        nb = np.ascontiguousarray(s.nb_apply if nb_apply is None else nb_apply, dtype=np.int32)
        psi = np.ascontiguousarray(s.psi if psi is None else psi, dtype=np.complex128)
        h2 = np.zeros_like(psi) if h2 is None else h2
        h3 = np.zeros_like(psi) if h3 is None else h3
        assert h2.dtype == np.complex128 and h2.flags["C_CONTIGUOUS"] and h2.shape == psi.shape
        assert h3.dtype == np.complex128 and h3.flags["C_CONTIGUOUS"] and h3.shape == psi.shape
        own = None if owned is None else np.ascontiguousarray(owned, dtype=np.uint8)
        check(lib().tcg_apply(self.handle, C.c_uint32(mask), nb.ctypes.data_as(C.POINTER(C.c_int32)),
                              psi.ctypes.data, h2.ctypes.data, h3.ctypes.data,
                              None if own is None else own.ctypes.data))
        return h2, h3

    def qp_partial(self, rank, nranks):
        """This rank's share of the tc3a2a4b2b5 occupied-pair stage: returns
        (device pointer, bytes) of the FP64 buffer the caller must sum over
        ranks before qp_finish()."""
        p = C.c_void_p()
        n = C.c_size_t()
        check(lib().tcg_qp_partial(self.handle, int(rank), int(nranks), C.byref(p), C.byref(n)))
        return int(p.value or 0), int(n.value)

    def qp_finish(self):
        check(lib().tcg_qp_finish(self.handle))

    def energy_grad(self, terms, dchi_ptr=0, tables=False):
        """(E2, E3, dE_du, dE_dv2) of the current state (tcg_energy_grad); dchi_ptr:
        device buffer (layout of phik_left) for dE/d conj(chi), 0 to skip;
        tables: also the tc2x Jastrow-table gradients [nspin][N] (Gamma only)."""
        s = self.system
        e = (C.c_double * 4)()
        du = dv = None
        if tables:
            du = np.zeros((s.nspin, s.N), dtype=np.complex128)
            dv = np.zeros((s.nspin, s.N), dtype=np.complex128)
        check(lib().tcg_energy_grad(self.handle, C.c_uint32(_terms(terms)), e, C.c_void_p(dchi_ptr or None),
                                    None if du is None else du.ctypes.data, None if dv is None else dv.ctypes.data))
        return complex(e[0], e[1]), complex(e[2], e[3]), du, dv

    def energy_device(self, h2_ptr, h3_ptr, nb_apply=None):
        """(E2, E3) of the applied bands from DEVICE arrays h2 / h3 (packed like
        psi; pointers as ints, 0 = skip), reduced on the GPU in FP64."""
        s = self.system
        nb = np.ascontiguousarray(s.nb_apply if nb_apply is None else nb_apply, dtype=np.int32)
        out = (C.c_double * 4)()
        check(lib().tcg_energy(self.handle, nb.ctypes.data_as(C.POINTER(C.c_int32)), C.c_void_p(h2_ptr or None),
                               C.c_void_p(h3_ptr or None), out))
        return complex(out[0], out[1]), complex(out[2], out[3])

    def set_pseudo(self, pseudo):
        """Upload pseudopotential data (tc_b200.system.Pseudo) for the one-body terms."""
        d, keep = pseudo.descriptor()
        check(lib().tcg_set_pseudo(self.handle, C.byref(d)))
        self._pseudo_keep = keep

    def apply_h1(self, terms, psi=None, nb_apply=None, h1=None, owned=None):
        """One-body terms (kinetic, pseudo) on host arrays; returns h1 with h1 += terms(psi)."""
        s = self.system
        nb = np.ascontiguousarray(s.nb_apply if nb_apply is None else nb_apply, dtype=np.int32)
        psi = np.ascontiguousarray(s.psi if psi is None else psi, dtype=np.complex128)
        h1 = np.zeros_like(psi) if h1 is None else h1
        own = None if owned is None else np.ascontiguousarray(owned, dtype=np.uint8)
        check(lib().tcg_apply_h1(self.handle, C.c_uint32(_terms(terms)), nb.ctypes.data_as(C.POINTER(C.c_int32)),
                                 psi.ctypes.data, h1.ctypes.data, None if own is None else own.ctypes.data))
        return h1

    def apply_device(self, terms, psi_ptr, h2_ptr, h3_ptr, nb_apply=None, owned=None):
        """Device-memory apply on the context's stream (pointers as ints)."""
        s = self.system
        nb = np.ascontiguousarray(s.nb_apply if nb_apply is None else nb_apply, dtype=np.int32)
        own = None if owned is None else np.ascontiguousarray(owned, dtype=np.uint8)
        check(lib().tcg_apply_device(self.handle, C.c_uint32(_terms(terms)), nb.ctypes.data_as(C.POINTER(C.c_int32)),
                                     C.c_void_p(psi_ptr), C.c_void_p(h2_ptr), C.c_void_p(h3_ptr),
                                     None if own is None else own.ctypes.data))


def sum_of_vaux(system):
    """(alpha_Vaux, sum_of_Vaux_scf[nk_irr]) computed on the device."""
    sysd, _, keep = system.descriptors()
    alpha = C.c_double()
    out = np.zeros(system.nk_irr)
    check(lib().tcg_sum_of_vaux(C.byref(sysd), C.byref(alpha), out.ctypes.data))
    return alpha.value, out


def sum_of_vaux_noalloc(system, kirr_dev_ptr, kall_dev_ptr, out_dev_ptr, stream=None):
    """Allocation-free divergence sums: device pointers in, device pointer
    out (see tcg_sum_of_vaux_noalloc in include/tcg.h).  Returns alpha."""
    rec = (C.c_double * 9)(*[float(x) for x in np.asarray(system.recip).ravel()])
    alpha = C.c_double()
    check(lib().tcg_sum_of_vaux_noalloc(rec, float(system.omega), int(system.nk_irr), int(system.nk_all),
                                        C.c_void_p(kirr_dev_ptr), C.c_void_p(kall_dev_ptr), C.c_void_p(out_dev_ptr),
                                        C.byref(alpha), C.c_void_p(stream) if stream else None))
    return alpha.value


def version():
    return lib().tcg_version().decode()


def subspace_ritz(V, HV, nout, Vref=None, biortho=False, stream=None, left=False):
    """Rayleigh-Ritz step of the block Davidson on the device (tcg_subspace_ritz).
    V, Vref: torch complex128 CUDA tensors [ndim, npw]; HV: list of up to three
    tensors [ndim, npw] (H1 V, H2 V, H3 V; None for absent).  Returns
    (eigenvalues [ndim], energies [3, nout], V_out [nout, npw], Vl_out or None);
    the left vectors Vref X_left are computed when Vref is given or left is set."""
    import torch
    ndim, npw = V.shape
    hv = list(HV) + [None] * (3 - len(HV))
    ptr = lambda x: None if x is None else C.c_void_p(x.data_ptr())
    eig = np.zeros(ndim, dtype=np.complex128)
    en = np.zeros((3, max(nout, 1)), dtype=np.complex128)
    Vo = torch.zeros((max(nout, 1), npw), dtype=torch.complex128, device=V.device)
    Vl = torch.zeros_like(Vo) if (Vref is not None or left) else None
    check(lib().tcg_subspace_ritz(int(ndim), int(npw), int(nout), 1 if biortho else 0, ptr(V), ptr(Vref),
                                  ptr(hv[0]), ptr(hv[1]), ptr(hv[2]),
                                  eig.view(np.float64).ctypes.data_as(C.POINTER(C.c_double)),
                                  en.view(np.float64).ctypes.data_as(C.POINTER(C.c_double)), ptr(Vo), ptr(Vl),
                                  None if stream is None else C.c_void_p(stream)))
    return eig, en[:, :nout], Vo[:nout], (None if Vl is None else Vl[:nout])


def gram_schmidt(V, Vl=None, stream=None):
    """In-place Gram-Schmidt (or bi-orthonormalisation with Vl) of the rows of
    the torch complex128 CUDA tensor V [nvec, npw] (tcg_gram_schmidt)."""
    nvec, npw = V.shape
    check(lib().tcg_gram_schmidt(int(nvec), int(npw), C.c_void_p(V.data_ptr()),
                                 None if Vl is None else C.c_void_p(Vl.data_ptr()),
                                 None if stream is None else C.c_void_p(stream)))


def davidson_expand(V, nbasis, phi, H, kG2, eig_ref, stream=None):
    """New trial vectors of one Davidson block (tcg_davidson_expand): V torch
    complex128 CUDA [capacity, npw] with nbasis valid rows; phi [nblock, npw];
    H: list of up to three [nblock, npw] (H1 phi, H2 phi, H3 phi, None for
    absent); kG2 float64 CUDA [npw]; eig_ref complex [nblock] (host).  Returns
    the new number of valid rows of V."""
    nblock, npw = phi.shape
    h = list(H) + [None] * (3 - len(H))
    ptr = lambda x: None if x is None else C.c_void_p(x.data_ptr())
    e = np.ascontiguousarray(np.asarray(eig_ref, dtype=np.complex128)[:nblock])
    out = C.c_int32()
    check(lib().tcg_davidson_expand(int(nbasis), int(nblock), int(npw), ptr(V), ptr(phi), ptr(h[0]), ptr(h[1]),
                                    ptr(h[2]), ptr(kG2), e.view(np.float64).ctypes.data_as(C.POINTER(C.c_double)),
                                    C.byref(out), None if stream is None else C.c_void_p(stream)))
    return int(out.value)

