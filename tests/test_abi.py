"""The C-ABI library loads and exports every function include/tcg.h declares;
without a GPU every entry point fails loudly (no CPU fallback)."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SO = os.path.join(ROOT, "tc_b200", "libtcg_b200.so")


def declared():
    txt = open(os.path.join(ROOT, "include", "tcg.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(tcg_[a-z0-9_]+)\s*\(", txt)))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(SO):
        from tc_b200 import build
        build.build()
    return C.CDLL(SO)


def test_exports_every_declared_symbol(lib):
    names = declared()
    assert len(names) >= 14
    for n in names:
        assert hasattr(lib, n), n
    out = subprocess.run(["nm", "-D", "--defined-only", SO], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (tcg_\w+)", out))
    assert set(names) <= exported


def test_python_binding_covers_header():
    from tc_b200 import _lib
    assert set(declared()) == set(_lib.EXPORTS)


def test_version_and_error_without_gpu(lib):
    import torch
    lib.tcg_version.restype = C.c_char_p
    assert b"sm_100a" in lib.tcg_version()
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    from tc_b200 import TCError, synth
    from tc_b200.context import Context
    s = synth.small("HF")
    with pytest.raises(TCError) as e:
        Context(s)
    assert e.value.code == 2            # TCG_ERR_CUDA: no device, no fallback


def test_noalloc_rejects_arguments_before_device_work():
    """tcg_sum_of_vaux_noalloc checks its host arguments before it touches
    the device: oversize k-sets, non-finite or non-positive geometry and null
    pointers are TCG_ERR_ARG (the device pointers are never dereferenced)."""
    from tc_b200 import TCError, synth
    from tc_b200.context import sum_of_vaux_noalloc
    s = synth.config("C1")
    fake = 16  # never used: every case fails on the host

    class Geo:
        recip = s.recip
        omega = s.omega
        nk_irr = s.nk_irr
        nk_all = s.nk_all
    cases = [dict(nk_irr=129, nk_all=128), dict(omega=0.0), dict(omega=float("inf")),
             dict(recip=np.where(np.eye(3) > 0, np.nan, np.asarray(s.recip))), dict(nk_irr=0)]
    for kw in cases:
        g = type("G", (Geo,), kw)
        with pytest.raises(TCError) as e:
            sum_of_vaux_noalloc(g, fake, fake, fake)
        assert e.value.code == 1, kw
    with pytest.raises(TCError) as e:
        sum_of_vaux_noalloc(Geo, 0, fake, fake)
    assert e.value.code == 1


def test_struct_layout_matches_header(tmp_path):
    """ctypes mirrors of the descriptors have the C sizes (compiled check)"""
    from tc_b200 import abi
    src = tmp_path / "size_probe.c"
    exe = tmp_path / "size_probe"
    src.write_text('#include "include/tcg.h"\n#include <stdio.h>\n'
                   'int main(){printf("%zu %zu %zu %zu\\n", sizeof(tcg_system_desc), sizeof(tcg_state_desc), '
                   'sizeof(tcg_pseudo_desc), sizeof(tcg_forms));}\n')
    subprocess.run(["gcc", "-I", ROOT, "-o", str(exe), str(src)], check=True)
    a, b, c, d = map(int, subprocess.run([str(exe)], capture_output=True, text=True).stdout.split())
    assert C.sizeof(abi.SystemDesc) == a
    assert C.sizeof(abi.StateDesc) == b
    assert C.sizeof(abi.PseudoDesc) == c
    assert C.sizeof(abi.Forms) == d


def test_oracle_exports():
    from oracle import oracle as O
    L = O.lib()
    for n in ("tco_apply", "tco_density", "tco_sum_of_vaux", "tco_fft3d", "tco_uk", "tco_tc2body"):
        assert hasattr(L, n)
