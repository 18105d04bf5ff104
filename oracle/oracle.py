"""ctypes binding of the CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline / reference arm -- never by the product package.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from tc_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(HERE, "liboracle.so")


def build(force=False):
    if force or not os.path.exists(SO) or os.path.getmtime(SO) < os.path.getmtime(os.path.join(HERE, "tc_oracle.c")):
        subprocess.run(["make", "-C", HERE, "-s"], check=True)
    return SO


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(SO)
        L.tco_apply.argtypes = [C.POINTER(abi.SystemDesc), C.POINTER(abi.StateDesc), C.c_uint32,
                                C.POINTER(C.c_int32), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.tco_apply_h1.argtypes = [C.POINTER(abi.SystemDesc), C.POINTER(abi.PseudoDesc), C.c_uint32,
                                   C.POINTER(C.c_int32), C.c_void_p, C.c_void_p, C.c_void_p]
        L.tco_density.argtypes = [C.POINTER(abi.SystemDesc), C.POINTER(abi.StateDesc), C.c_void_p]
        L.tco_sum_of_vaux.argtypes = [C.POINTER(abi.SystemDesc), C.POINTER(C.c_double), C.c_void_p]
        L.tco_fft3d.argtypes = [C.POINTER(C.c_int32), C.c_void_p, C.c_int]
        L.tco_uk.argtypes = [C.POINTER(abi.SystemDesc), C.POINTER(C.c_double), C.c_int, C.c_int]
        L.tco_uk.restype = C.c_double
        L.tco_tc2body.argtypes = [C.POINTER(abi.SystemDesc), C.POINTER(C.c_double), C.c_int, C.c_int]
        L.tco_tc2body.restype = C.c_double
        L.tco_last_error.restype = C.c_char_p
        L.tco_set_threads.argtypes = [C.c_int]
        L.tco_get_threads.restype = C.c_int
        L.tco_set_qstride.argtypes = [C.c_int]
        L.tco_timers.argtypes = [C.POINTER(C.c_double)] * 3
        _lib = L
    return _lib


def _check(rc):
    if rc != 0:
        raise RuntimeError(f"oracle error {rc}: {lib().tco_last_error().decode()}")


def set_threads(n):
    lib().tco_set_threads(int(n))


def threads():
    return lib().tco_get_threads()


def fft3d(grid, nr, forward):
    """grid: complex128 array of N = nr0*nr1*nr2 (x fastest); returns a new array."""
    g = np.ascontiguousarray(grid, dtype=np.complex128).copy()
    n = (C.c_int32 * 3)(*nr)
    _check(lib().tco_fft3d(n, g.ctypes.data, 1 if forward else 0))
    return g


def apply(sysm, mask, psi=None, nb_apply=None, owned=None):
    """(h2, h3) = oracle terms applied to psi (zero-initialised outputs)."""
    sysd, st, keep = sysm.descriptors()
    nb = np.ascontiguousarray(sysm.nb_apply if nb_apply is None else nb_apply, dtype=np.int32)
    psi = np.ascontiguousarray(sysm.psi if psi is None else psi, dtype=np.complex128)
    h2 = np.zeros_like(psi)
    h3 = np.zeros_like(psi)
    own = None if owned is None else np.ascontiguousarray(owned, dtype=np.uint8)
    _check(lib().tco_apply(C.byref(sysd), C.byref(st), C.c_uint32(mask),
                           nb.ctypes.data_as(C.POINTER(C.c_int32)), psi.ctypes.data, h2.ctypes.data,
                           h3.ctypes.data, None if own is None else own.ctypes.data))
    return h2, h3


def apply_h1(sysm, mask, pseudo=None, psi=None, nb_apply=None, owned=None):
    """h1 = oracle one-body terms (kinetic, pseudopotential) applied to psi."""
    sysd, _, keep = sysm.descriptors()
    pd, pkeep = (None, None) if pseudo is None else pseudo.descriptor()
    nb = np.ascontiguousarray(sysm.nb_apply if nb_apply is None else nb_apply, dtype=np.int32)
    psi = np.ascontiguousarray(sysm.psi if psi is None else psi, dtype=np.complex128)
    h1 = np.zeros_like(psi)
    own = None if owned is None else np.ascontiguousarray(owned, dtype=np.uint8)
    _check(lib().tco_apply_h1(C.byref(sysd), None if pd is None else C.byref(pd), C.c_uint32(mask),
                              nb.ctypes.data_as(C.POINTER(C.c_int32)), psi.ctypes.data, h1.ctypes.data,
                              None if own is None else own.ctypes.data))
    return h1


def density(sysm):
    sysd, st, keep = sysm.descriptors()
    out = np.zeros((2, sysm.N), dtype=np.complex128)
    _check(lib().tco_density(C.byref(sysd), C.byref(st), out.ctypes.data))
    return out


def sum_of_vaux(sysm):
    sysd, st, keep = sysm.descriptors()
    alpha = C.c_double()
    out = np.zeros(sysm.nk_irr)
    _check(lib().tco_sum_of_vaux(C.byref(sysd), C.byref(alpha), out.ctypes.data))
    return alpha.value, out


def uk(sysm, G, s1, s2):
    sysd, st, keep = sysm.descriptors()
    g = (C.c_double * 3)(*[float(x) for x in G])
    return lib().tco_uk(C.byref(sysd), g, s1, s2)


def tc2body(sysm, G, s1, s2):
    sysd, st, keep = sysm.descriptors()
    g = (C.c_double * 3)(*[float(x) for x in G])
    return lib().tco_tc2body(C.byref(sysd), g, s1, s2)


def set_qstride(s):
    lib().tco_set_qstride(int(s))


def timers():
    """(shared occupied-pair stage, total, set-up) seconds since reset."""
    a, b, d = C.c_double(), C.c_double(), C.c_double()
    lib().tco_timers(C.byref(a), C.byref(b), C.byref(d))
    return a.value, b.value, d.value


def reset_timers():
    lib().tco_reset_timers()
