"""ctypes loader of libtcg_b200.so.  There is no fallback: if the library is
missing or no CUDA device is present, every call raises TCError."""
import ctypes as C
import os

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(HERE, "libtcg_b200.so")


class TCError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"tcg error {code}: {msg}")
        self.code = code


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(SO):
            raise TCError(abi.TCG_ERR_STATE, f"CUDA library not built: {SO} (run tc_b200/build.py)")
        L = C.CDLL(SO)
        vp = C.c_void_p
        L.tcg_ctx_create.argtypes = [C.POINTER(abi.SystemDesc), C.c_int32, C.POINTER(vp)]
        L.tcg_ctx_destroy.argtypes = [vp]
        L.tcg_set_state.argtypes = [vp, C.POINTER(abi.StateDesc)]
        L.tcg_apply.argtypes = [vp, C.c_uint32, C.POINTER(C.c_int32), vp, vp, vp, vp]
        L.tcg_apply_device.argtypes = [vp, C.c_uint32, C.POINTER(C.c_int32), vp, vp, vp, vp]
        L.tcg_sum_of_vaux.argtypes = [C.POINTER(abi.SystemDesc), C.POINTER(C.c_double), vp]
        L.tcg_density.argtypes = [vp, C.POINTER(abi.StateDesc), vp]
        L.tcg_stream.argtypes = [vp]
        L.tcg_stream.restype = vp
        L.tcg_launch_count.argtypes = [vp]
        L.tcg_launch_count.restype = C.c_int64
        L.tcg_last_error.restype = C.c_char_p
        L.tcg_version.restype = C.c_char_p
        L.tcg_set_tuning.argtypes = [vp, C.c_int64]
        L.tcg_profile.argtypes = [vp, C.c_int]
        L.tcg_profile_read.argtypes = [vp, C.c_int, C.c_char_p, C.POINTER(C.c_int64), C.POINTER(C.c_double),
                                       C.POINTER(C.c_double), C.POINTER(C.c_int)]
        L.tcg_refresh_state.argtypes = [vp]
        L.tcg_sum_of_vaux_noalloc.argtypes = [C.POINTER(C.c_double), C.c_double, C.c_int32, C.c_int32, vp, vp, vp,
                                              C.POINTER(C.c_double), vp]
        L.tcg_qp_partial.argtypes = [vp, C.c_int32, C.c_int32, C.POINTER(vp), C.POINTER(C.c_size_t)]
        L.tcg_qp_finish.argtypes = [vp]
        L.tcg_set_pseudo.argtypes = [vp, C.POINTER(abi.PseudoDesc)]
        L.tcg_apply_h1.argtypes = [vp, C.c_uint32, C.POINTER(C.c_int32), vp, vp, vp]
        L.tcg_energy_grad.argtypes = [vp, C.c_uint32, C.POINTER(C.c_double), vp, vp, vp]
        L.tcg_subspace_ritz.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_int32, vp, vp, vp, vp, vp,
                                         C.POINTER(C.c_double), C.POINTER(C.c_double), vp, vp, vp]
        L.tcg_gram_schmidt.argtypes = [C.c_int32, C.c_int32, vp, vp, vp]
        L.tcg_davidson_expand.argtypes = [C.c_int32, C.c_int32, C.c_int32, vp, vp, vp, vp, vp, vp,
                                          C.POINTER(C.c_double), C.POINTER(C.c_int32), vp]
        L.tcg_set_forms.argtypes = [vp, C.POINTER(abi.Forms)]
        L.tcg_get_forms.argtypes = [vp, C.POINTER(abi.Forms)]
        L.tcg_energy.argtypes = [vp, C.POINTER(C.c_int32), vp, vp, C.POINTER(C.c_double)]
        _lib = L
    return _lib


def check(rc):
    if rc != abi.TCG_OK:
        raise TCError(rc, lib().tcg_last_error().decode())


EXPORTS = ["tcg_ctx_create", "tcg_ctx_destroy", "tcg_set_state", "tcg_apply", "tcg_apply_device",
           "tcg_sum_of_vaux", "tcg_density", "tcg_stream", "tcg_launch_count", "tcg_last_error",
           "tcg_version", "tcg_set_tuning", "tcg_profile", "tcg_profile_read", "tcg_refresh_state",
           "tcg_sum_of_vaux_noalloc", "tcg_energy", "tcg_qp_partial", "tcg_qp_finish", "tcg_set_pseudo", "tcg_apply_h1", "tcg_energy_grad",
           "tcg_subspace_ritz", "tcg_gram_schmidt", "tcg_davidson_expand", "tcg_set_forms", "tcg_get_forms"]
