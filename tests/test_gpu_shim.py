"""The C++ drop-in shim on the GPU: calling TC++'s routines one by one (as
calc_hamiltonian::all does) and the one-call block entry give the Python
binding's H phi, for HF, TC and BITC, with and without symmetry reduction."""
import subprocess

import numpy as np
import pytest

from tc_b200 import abi, synth
from tc_b200.context import Context
from _shim_io import build_driver, read_result, write_system
from test_qe_symmetry import qe_system

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.mark.parametrize("case", ["HF", "TC", "BITC", "BITC-qe-symmetry", "BITC-mixed"])
def test_shim_matches_binding(tmp_path, case):
    prec = 1 if case.endswith("mixed") else 0
    if case == "BITC-qe-symmetry":
        s = qe_system("BITC")
    else:
        s = synth.small(case.split("-")[0], nk=2, nbands=3, nocc=2, seed=31)
    exe = build_driver(str(tmp_path))
    inp, out = tmp_path / "in.bin", tmp_path / "out.bin"
    owned = np.ones(int(np.sum(s.nb_apply)), dtype=np.uint8)
    owned[1::3] = 0                       # a few bands belong to another rank
    write_system(s, str(inp), precision=prec, owned=owned)
    r = subprocess.run([exe, str(inp), str(out)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    h2, h3, b2, b3, launches = read_result(s, str(out))
    assert launches > 0
    mask = abi.TERMS_HF if s.method == "HF" else abi.TERMS_TC
    with Context(s, "mixed" if prec else "fp64") as ctx:
        ctx.set_state()
        g2, g3 = ctx.apply(mask, owned=owned)
    tol = 2e-5 if prec else 1e-12
    assert rel(h2, g2) < tol and rel(b2, g2) < tol
    if s.method != "HF":
        assert rel(h3, g3) < tol and rel(b3, g3) < tol
