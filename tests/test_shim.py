"""The C++ drop-in shim (tc_b200/shim/calc_hamiltonian_tcg.cpp): TC++'s six
routine signatures over the C-ABI, built against stand-in declarations of the
reference's classes (tcpp_standin.hpp) and driven like calc_hamiltonian::all
(shim_check.cpp).

CPU: it compiles and links against libtcg_b200.so, and without a GPU the
library's error reaches the caller through error_messages::stop (no CPU
fallback).  GPU (tests/test_gpu_shim.py): its results equal the Python
binding's, per routine and as one block."""
import os
import subprocess

import pytest

from _shim_io import build_driver, write_system


def test_shim_builds_and_fails_loudly_without_gpu(tmp_path):
    import torch
    from tc_b200 import synth
    exe = build_driver(str(tmp_path))
    if torch.cuda.is_available():
        pytest.skip("GPU present: covered by tests/test_gpu_shim.py")
    s = synth.small("BITC", nk=2, nbands=2, nocc=1)
    inp, out = tmp_path / "in.bin", tmp_path / "out.bin"
    write_system(s, str(inp))
    r = subprocess.run([exe, str(inp), str(out)], capture_output=True, text=True)
    assert r.returncode == 1
    assert "libtcg_b200" in r.stderr and "CUDA" in r.stderr
    assert not os.path.exists(out)
