"""CUDA path vs the oracle on the reference's own QE test data (fcc Si,
test/example3; tests/golden/qe_si.npz): a symmetry-reduced k-set with 48
space-group operations, 24 of them non-symmorphic (translation (1/4,1/4,1/4)),
and time reversal.  This runs the rotated-k scatter (Gindex / phase of every
equivalent k) and the rotation of the tc3a2a4b2b5 intermediates by U != 1 with
a translation (k_rot_scalar / k_rot_vec) on the device."""
import numpy as np
import pytest

from tc_b200 import abi
from tc_b200.context import Context
from oracle import oracle as O
from test_qe_symmetry import qe_system

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10
MIXED_TOL = 2e-5


def rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


_cache = {}


def sys_and_ref(method, mask):
    key = (method, mask)
    if key not in _cache:
        s = _cache.get(method) or qe_system(method)
        _cache[method] = s
        _cache[key] = O.apply(s, mask)
    return _cache[method], _cache[key]


@pytest.mark.parametrize("prec,tol", [("fp64", FP64_TOL), ("mixed", MIXED_TOL)])
@pytest.mark.parametrize("term", ["hf2x", "tc2x", "tc3a1", "tc3b1", "tc3a2a4b2b5", "tc3a3b3b4b6"])
def test_qe_si_term(term, prec, tol):
    mask = abi.TERM_NAMES[term]
    s, (r2, r3) = sys_and_ref("HF" if term == "hf2x" else "BITC", mask)
    with Context(s, prec) as ctx:
        ctx.set_state()
        g2, g3 = ctx.apply(mask)
    ref, got = (r2, g2) if mask & abi.TERMS_H2 else (r3, g3)
    e = rel(got, ref)
    print(f"QE Si {term} {prec}: rel {e:.3e}")
    assert e < tol


@pytest.mark.parametrize("method", ["TC", "BITC"])
def test_qe_si_all_terms_generic_kernels(monkeypatch, method):
    """the runtime-size pass kernels on the same symmetry-reduced input"""
    monkeypatch.setenv("TCG_GENERIC_PASSES", "1")
    s, (r2, r3) = sys_and_ref(method, abi.TERMS_TC)
    with Context(s, "fp64") as ctx:
        ctx.set_state()
        g2, g3 = ctx.apply(abi.TERMS_TC)
    assert rel(g2, r2) < FP64_TOL
    assert rel(g3, r3) < FP64_TOL
