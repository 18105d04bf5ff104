"""ctypes mirror of the C-ABI descriptors in include/tcg.h.

The same structures drive the CUDA library (libtcg_b200.so) and, in the
tests, the CPU oracle, so both see byte-identical inputs.
"""
import ctypes as C

TCG_OK = 0
TCG_ERR_ARG = 1
TCG_ERR_CUDA = 2
TCG_ERR_TIMEOUT = 3
TCG_ERR_UNSUPPORTED = 4
TCG_ERR_STATE = 5
TCG_ERR_NOMEM = 6
TCG_ERR_NUMERIC = 7

METHOD_HF, METHOD_TC, METHOD_BITC = 0, 1, 2
METHODS = {"HF": METHOD_HF, "TC": METHOD_TC, "BITC": METHOD_BITC}

PREC_FP64, PREC_MIXED = 0, 1

TERM_HF2X = 1 << 0
TERM_TC2X = 1 << 1
TERM_TC3A1 = 1 << 2
TERM_TC3B1 = 1 << 3
TERM_TC3A2A4B2B5 = 1 << 4
TERM_TC3A3B3B4B6 = 1 << 5
TERMS_HF = TERM_HF2X
TERMS_TC = TERM_TC2X | TERM_TC3A1 | TERM_TC3B1 | TERM_TC3A2A4B2B5 | TERM_TC3A3B3B4B6
TERM_HF2H = 1 << 6
TERM_TC2H = 1 << 7
TERM_KINETIC = 1 << 8
TERM_PSEUDO = 1 << 9
TERMS_H1 = TERM_KINETIC | TERM_PSEUDO
TERMS_H2 = TERM_HF2X | TERM_TC2X | TERM_HF2H | TERM_TC2H
TERM_NAMES = {
    "hf2x": TERM_HF2X,
    "tc2x": TERM_TC2X,
    "tc3a1": TERM_TC3A1,
    "tc3b1": TERM_TC3B1,
    "tc3a2a4b2b5": TERM_TC3A2A4B2B5,
    "tc3a3b3b4b6": TERM_TC3A3B3B4B6,
}
# terms outside the exchange / three-body hot path (Hartree-type and one-body)
TERM_NAMES_EXTRA = {"hf2h": TERM_HF2H, "tc2h": TERM_TC2H, "kinetic": TERM_KINETIC, "pseudo": TERM_PSEUDO}

_i32p = C.POINTER(C.c_int32)
_u8p = C.POINTER(C.c_uint8)
_f64p = C.POINTER(C.c_double)


class SystemDesc(C.Structure):
    _fields_ = [
        ("nr", C.c_int32 * 3),
        ("recip", C.c_double * 9),
        ("lattice", C.c_double * 9),
        ("omega", C.c_double),
        ("calc_method", C.c_int32),
        ("nspin", C.c_int32),
        ("nk_irr", C.c_int32),
        ("num_kpoints", C.c_int32),
        ("nsym_k", _i32p),
        ("kvec", _f64p),
        ("time_rev", _u8p),
        ("rot_index", _i32p),
        ("nsymop", C.c_int32),
        ("rotation", _i32p),
        ("translation", _f64p),
        ("npw", _i32p),
        ("gindex", _i32p),
        ("phase", _f64p),
        ("jastrow_A", C.c_double * 4),
        ("jastrow_F", C.c_double * 4),
        ("includes_div_correction", C.c_int32),
        ("alpha_Vaux", C.c_double),
        ("sum_Vaux", _f64p),
    ]


class StateDesc(C.Structure):
    _fields_ = [
        ("nbands", _i32p),
        ("nocc", _i32p),
        ("filling", _f64p),
        ("phik", _f64p),
        ("phik_left", _f64p),
        ("density", _f64p),
    ]


class Forms(C.Structure):
    _fields_ = [(n, C.c_int32) for n in ("xy", "z", "prefetch", "prune", "fuse", "qp_sacc", "sacc", "min_targets")]


class PseudoDesc(C.Structure):
    _fields_ = [
        ("vloc", _f64p),
        ("nspecies", C.c_int32),
        ("natoms", C.c_int32),
        ("species_of_atom", _i32p),
        ("atom_pos", _f64p),
        ("nproj", _i32p),
        ("lbeta", _i32p),
        ("dij", _f64p),
        ("projector", _f64p),
    ]


def ptr(arr, ctype):
    """Pointer to a contiguous numpy array (None -> NULL)."""
    if arr is None:
        return C.cast(None, C.POINTER(ctype))
    assert arr.flags["C_CONTIGUOUS"], "array must be C-contiguous"
    return arr.ctypes.data_as(C.POINTER(ctype))
