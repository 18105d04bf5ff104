"""Real symmetry-reduced input: the reference's own QE test data (fcc Si,
test/example3: 3 irreducible k-points, 48 space-group operations of which 24
carry the fractional translation (1/4, 1/4, 1/4), time reversal), read by
tc_b200.qe as TC++ reads it (tests/golden/qe_si.npz is the compact copy made by
tests/golden/make_si_examples.py).

- The k-point star TC++ builds from it (Kpoints::set_kvectors_by_symmetry) is
  the one the reference printed for this run (test/example3/output.out:383-449).
- Oracle, reduced vs expanded: every term applied on the symmetry-reduced set
  (Gindex / phase of rotated k-points, rotation of the tc3a2a4b2b5
  intermediates by U with the translation) equals the same system with every
  k-point of the mesh written out explicitly (nsym = 1).  QE's orbitals are
  eigenstates to about 1e-8, so the identity holds to that level; a wrong
  rotation or translation convention breaks it at O(1) (checked by planting one).
"""
import os

import numpy as np
import pytest

from tc_b200 import abi, qe
from oracle import oracle as O
from _expand import expand

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE = os.path.join(HERE, "golden", "qe_si.npz")
REF_DIR = "/root/reference/test/example3"

# RPA Jastrow of test/example3 as TC++ reports it (output.out:492-497)
A = np.array([[0.9833143351, 1.31108578], [1.31108578, 0.9833143351]])
F = np.array([[1.402365384, 1.145026541], [1.145026541, 1.402365384]])

# equivalent k-points (crystal) and whether the operation carries the
# (1/4,1/4,1/4) translation, per irreducible k (output.out:383-449)
STAR = [
    [((0, 0, 0), 0)],
    [((0, 0, -0.5), 0), ((0.5, 0.5, 0.5), 0), ((0, -0.5, 0), 0), ((-0.5, 0, 0), 0)],
    [((0, -0.5, -0.5), 0), ((0.5, 0, 0.5), 1), ((-0.5, -0.5, 0), 1)],
]


def qe_system(method):
    if method == "HF":
        return qe.system_from_qe(FIXTURE, "HF")
    return qe.system_from_qe(FIXTURE, method, A=A, F=F)


def test_kpoint_star_matches_reference_output():
    q = qe.QEData.load_npz(FIXTURE)
    U = qe.tc_rotations(q.rotation_qe)
    star = qe.expand_kpoints(q.kcrys, q.kweight, U, not q.noinv)
    assert len(star) == len(STAR)
    for got, want in zip(star, STAR):
        assert len(got) == len(want)
        for (v, isym, tr), (kw, has_t) in zip(got, want):
            assert np.allclose(v, kw, atol=1e-12)
            assert not tr
            assert np.allclose(q.translation[isym], 0.25 * has_t)
    # TC++'s k-weight consistency check (kpoints.cpp:100-110): 2/N_k per image
    s = qe_system("BITC")
    assert s.num_kpoints == 8
    assert np.allclose(2.0 / s.num_kpoints * s.nsym_k, q.kweight)


@pytest.mark.skipif(not os.path.isdir(REF_DIR), reason="reference tree not present")
def test_reader_matches_fixture():
    a = qe.QEData(REF_DIR)
    b = qe.QEData.load_npz(FIXTURE)
    for f in qe.QEData._FIELDS:
        assert np.array_equal(np.asarray(getattr(a, f)), np.asarray(getattr(b, f))), f
    for ik in range(len(a.kweight)):
        for x, y in zip(a.read_wfc(ik), b.read_wfc(ik)):
            assert np.array_equal(x, y)


def test_orbitals_and_density():
    s = qe_system("BITC")
    for k in range(s.nk_irr):
        X = np.array([s.orb(0, k, b) for b in range(int(s.nbands[0]))])
        assert np.allclose(X.conj() @ X.T, np.eye(len(X)), atol=1e-10)
    # 4 electrons per spin channel per k-point of the mesh
    assert abs(s.density[0].sum() / s.N / s.num_kpoints - 4.0) < 1e-10
    assert np.allclose(s.density, O.density(s), rtol=0, atol=1e-12 * np.abs(s.density).max())


def _compare_reduced_expanded(s, e, mask):
    r2, r3 = O.apply(s, mask)
    x2, x3 = O.apply(e, mask)
    ref, got = (r2, x2) if mask & abi.TERMS_H2 else (r3, x3)
    fi = e.meta["first_of_irr"]
    d = m = 0.0
    for k in range(s.nk_irr):
        for b in range(int(s.nb_apply[0][k])):
            a = s.band_view(ref, 0, k, b)
            d = max(d, np.abs(a - e.band_view(got, 0, int(fi[k]), b)).max())
            m = max(m, np.abs(a).max())
    return d / m


@pytest.mark.parametrize("term", ["hf2x", "tc2x", "tc3a1", "tc3b1", "tc3a2a4b2b5", "tc3a3b3b4b6"])
def test_oracle_reduced_equals_expanded(term):
    s = qe_system("HF" if term == "hf2x" else "BITC")
    e = expand(s)
    err = _compare_reduced_expanded(s, e, abi.TERM_NAMES[term])
    print(f"{term}: reduced vs expanded {err:.2e}")
    assert err < 1e-6


def test_planted_translation_error_is_caught():
    """the identity is sensitive to the rotation convention: flipping the sign
    of the fractional translation in the reduced system's symmetry table
    (a planted mistake, on the CPU) breaks it"""
    s = qe_system("BITC")
    e = expand(s)
    s.translation = -s.translation
    err = _compare_reduced_expanded(s, e, abi.TERM_TC3A2A4B2B5)
    assert err > 1e-3
