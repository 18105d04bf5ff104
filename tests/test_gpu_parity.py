"""CUDA path vs the CPU oracle, term by term, on small seeded systems.

FP64 mode: relative error <= 1e-10 on H psi (max |diff| / max |oracle| per
term).  Mixed mode (complex64 FFTs, FP64 accumulation): <= 2e-5.
"""
import numpy as np
import pytest

from tc_b200 import abi, synth
from tc_b200.context import Context, sum_of_vaux
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10
MIXED_TOL = 2e-5

CASES = {
    "HF": dict(method="HF"),
    "TC": dict(method="TC"),
    "BITC": dict(method="BITC"),
}


def rel(a, b):
    d = np.abs(a - b).max()
    m = np.abs(b).max()
    return d / m if m > 0 else d


_sys_cache = {}


def system(method, **kw):
    key = (method, tuple(sorted(kw.items())))
    if key not in _sys_cache:
        _sys_cache[key] = synth.small(method, **kw)
    return _sys_cache[key]


_oracle_cache = {}


def oracle_terms(s, mask):
    key = (id(s), mask)
    if key not in _oracle_cache:
        _oracle_cache[key] = O.apply(s, mask)
    return _oracle_cache[key]


@pytest.mark.parametrize("prec,tol", [("fp64", FP64_TOL), ("mixed", MIXED_TOL)])
@pytest.mark.parametrize("method,term", [("HF", "hf2x")] + [(m, t) for m in ("TC", "BITC") for t in
                                                            ("tc2x", "tc3a1", "tc3b1", "tc3a2a4b2b5", "tc3a3b3b4b6")])
def test_term_parity(method, term, prec, tol):
    s = system(method)
    mask = abi.TERM_NAMES[term]
    r2, r3 = oracle_terms(s, mask)
    with Context(s, prec) as ctx:
        ctx.set_state()
        g2, g3 = ctx.apply(mask)
    ref, got = (r2, g2) if mask & abi.TERMS_H2 else (r3, g3)
    assert np.abs(ref).max() > 0
    e = rel(got, ref)
    print(f"{method} {term} {prec}: rel err {e:.3e}")
    assert e < tol


@pytest.mark.parametrize("method", ["TC", "BITC"])
def test_all_terms_symmetry_tr(method):
    """time-reversal-reduced k-set (rotated intermediates of tc3a2a4b2b5)"""
    s = system(method, tr=True, nr=(16, 16, 16), ecut=1.5, nbands=2, nocc=1)
    r2, r3 = O.apply(s, abi.TERMS_TC)
    with Context(s, "fp64") as ctx:
        ctx.set_state()
        g2, g3 = ctx.apply(abi.TERMS_TC)
    assert rel(g2, r2) < FP64_TOL
    assert rel(g3, r3) < FP64_TOL


def test_spin_polarised_bitc():
    s = system("BITC", nspin=2)
    r2, r3 = O.apply(s, abi.TERMS_TC)
    with Context(s, "fp64") as ctx:
        ctx.set_state()
        g2, g3 = ctx.apply(abi.TERMS_TC)
    assert rel(g2, r2) < FP64_TOL
    assert rel(g3, r3) < FP64_TOL


def test_hf_spin_polarised():
    s = system("HF", nspin=2)
    r2, _ = O.apply(s, abi.TERM_HF2X)
    with Context(s, "fp64") as ctx:
        ctx.set_state()
        g2, _ = ctx.apply(abi.TERM_HF2X)
    assert rel(g2, r2) < FP64_TOL


def test_owned_mask_and_accumulate():
    """ownership flags skip bands; outputs accumulate (H += ...)"""
    s = system("TC")
    nbt = int(np.sum(s.nb_apply))
    owned = np.ones(nbt, dtype=np.uint8)
    owned[::2] = 0
    r2, r3 = O.apply(s, abi.TERMS_TC, owned=owned)
    with Context(s, "fp64") as ctx:
        ctx.set_state()
        base2 = np.full(s.psi.shape, 1.0 + 2.0j)
        base3 = np.full(s.psi.shape, -0.5j)
        g2, g3 = ctx.apply(abi.TERMS_TC, h2=base2.copy(), h3=base3.copy(), owned=owned)
    assert rel(g2 - base2, r2) < FP64_TOL
    assert rel(g3 - base3, r3) < FP64_TOL


def test_sum_of_vaux_device():
    s = system("HF")
    a, v = sum_of_vaux(s)
    a0, v0 = O.sum_of_vaux(s)
    assert abs(a - a0) < 1e-15
    assert np.abs(v - v0).max() / np.abs(v0).max() < 1e-12


@pytest.mark.parametrize("method", ["TC", "BITC"])
def test_density_device(method):
    s = system(method)
    d0 = O.density(s)
    with Context(s, "fp64") as ctx:
        d = ctx.density()
    assert rel(d, d0) < 1e-12


def test_errors():
    from tc_b200 import TCError
    s = system("TC")
    with Context(s, "fp64") as ctx:
        with pytest.raises(TCError) as e:
            ctx.apply(abi.TERMS_TC)
        assert e.value.code == abi.TCG_ERR_STATE
        ctx.set_state()
        with pytest.raises(TCError) as e:
            ctx.apply(abi.TERM_HF2X)
        assert e.value.code == abi.TCG_ERR_ARG
        bad = s.psi.copy()
        bad[3] = np.nan
        with pytest.raises(TCError) as e:
            ctx.apply(abi.TERMS_TC, psi=bad)
        assert e.value.code == abi.TCG_ERR_NUMERIC


@pytest.mark.parametrize("nr", [(24, 24, 24), (36, 36, 36)])
@pytest.mark.parametrize("prec,tol", [("fp64", FP64_TOL), ("mixed", MIXED_TOL)])
def test_fast_path_sizes(nr, prec, tol):
    """compile-time-size pass kernels at production grid sizes"""
    s = system("BITC", nr=nr, nk=2, ecut=2.0, nbands=2, nocc=1)
    r2, r3 = oracle_terms(s, abi.TERMS_TC)
    with Context(s, prec) as ctx:
        ctx.set_state()
        g2, g3 = ctx.apply(abi.TERMS_TC)
    assert rel(g2, r2) < tol
    assert rel(g3, r3) < tol


@pytest.mark.parametrize("xy", ["t6", "line"])
@pytest.mark.parametrize("method", ["HF", "TC", "BITC"])
@pytest.mark.parametrize("prec,tol", [("fp64", FP64_TOL), ("mixed", MIXED_TOL)])
def test_36_xy_forms(monkeypatch, method, xy, prec, tol):
    """36^3: XY passes with six threads per line (the default there) and one thread per line"""
    monkeypatch.setenv("TCG_XY_KERNELS", xy)
    s = system(method, nr=(36, 36, 36), nk=2, ecut=2.0, nbands=2, nocc=1)
    mask = abi.TERMS_HF if method == "HF" else abi.TERMS_TC
    r2, r3 = oracle_terms(s, mask)
    with Context(s, prec) as ctx:
        ctx.set_state()
        g2, g3 = ctx.apply(mask)
    assert rel(g2, r2) < tol
    if method != "HF":
        assert rel(g3, r3) < tol


@pytest.mark.parametrize("zform", ["line", "split", "t6", "t6r"])
@pytest.mark.parametrize("method", ["HF", "TC", "BITC"])
@pytest.mark.parametrize("prec,tol", [("fp64", FP64_TOL), ("mixed", MIXED_TOL)])
def test_36_z_forms(monkeypatch, method, zform, prec, tol):
    """36^3: every Z pass form (one thread, a lane pair, six threads per z-line with the inputs in shared
    memory or in registers)"""
    monkeypatch.setenv("TCG_Z_KERNELS", zform)
    s = system(method, nr=(36, 36, 36), nk=2, ecut=2.0, nbands=2, nocc=1)
    mask = abi.TERMS_HF if method == "HF" else abi.TERMS_TC
    r2, r3 = oracle_terms(s, mask)
    with Context(s, prec) as ctx:
        ctx.set_state()
        g2, g3 = ctx.apply(mask)
    assert rel(g2, r2) < tol
    if method != "HF":
        assert rel(g3, r3) < tol


@pytest.mark.parametrize("method", ["HF", "BITC"])
def test_generic_path_noncubic(method):
    """non-cubic grid -> generic (runtime-size) pass kernels"""
    s = system(method, nr=(12, 15, 10), nk=1, ecut=1.2, nbands=2, nocc=1)
    mask = abi.TERMS_HF if method == "HF" else abi.TERMS_TC
    r2, r3 = oracle_terms(s, mask)
    with Context(s, "fp64") as ctx:
        ctx.set_state()
        g2, g3 = ctx.apply(mask)
    assert rel(g2, r2) < FP64_TOL
    if method != "HF":
        assert rel(g3, r3) < FP64_TOL


def test_generic_path_forced(monkeypatch):
    """cubic grid with the generic kernels forced must agree too"""
    monkeypatch.setenv("TCG_GENERIC_PASSES", "1")
    s = system("TC")
    r2, r3 = oracle_terms(s, abi.TERMS_TC)
    with Context(s, "fp64") as ctx:
        ctx.set_state()
        g2, g3 = ctx.apply(abi.TERMS_TC)
    assert rel(g2, r2) < FP64_TOL
    assert rel(g3, r3) < FP64_TOL


@pytest.mark.parametrize("prec,tol", [("fp64", FP64_TOL), ("mixed", MIXED_TOL)])
@pytest.mark.parametrize("xy", ["line", "pair"])
@pytest.mark.parametrize("method", ["TC", "BITC"])
def test_xy_kernel_forms(monkeypatch, method, xy, prec, tol):
    """every term through both fast XY kernel forms (one thread per line, lane pairs)"""
    monkeypatch.setenv("TCG_XY_KERNELS", xy)
    s = system(method)
    r2, r3 = oracle_terms(s, abi.TERMS_TC)
    with Context(s, prec) as ctx:
        ctx.set_state()
        g2, g3 = ctx.apply(abi.TERMS_TC)
    assert rel(g2, r2) < tol
    assert rel(g3, r3) < tol


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_bitwise_deterministic(prec):
    """fixed-order accumulation: two applies give identical bits"""
    s = system("BITC")
    with Context(s, prec) as ctx:
        ctx.set_state()
        a2, a3 = ctx.apply(abi.TERMS_TC)
        ctx.refresh_state()
        b2, b3 = ctx.apply(abi.TERMS_TC)
    assert np.array_equal(a2.view(np.uint64), b2.view(np.uint64))
    assert np.array_equal(a3.view(np.uint64), b3.view(np.uint64))


@pytest.mark.parametrize("name", ["small_hf", "small_tc", "small_bitc", "small_bitc_tr"])
def test_gpu_matches_golden_fixture(name):
    """CUDA path (FP64) against the committed oracle fixtures"""
    import os
    from golden.make_golden import mask_of, system
    s = system(name)
    ref = np.load(os.path.join(os.path.dirname(__file__), "golden", name + ".npz"))
    with Context(s, "fp64") as ctx:
        ctx.set_state()
        g2, g3 = ctx.apply(mask_of(s))
    for got, want in ((g2, ref["h2"]), (g3, ref["h3"])):
        if np.abs(want).max() > 0:
            assert rel(got, want) < FP64_TOL


@pytest.mark.parametrize("prec,tol", [("fp64", FP64_TOL), ("mixed", MIXED_TOL)])
@pytest.mark.parametrize("method", ["TC", "BITC"])
def test_unequal_jastrow_channels(method, prec, tol):
    """parallel / antiparallel Jastrow channels differ (cusp-like F): the
    general spin-branch path of tc3a3b3b4b6 and tc3a2a4b2b5"""
    A = np.array([[0.5, 0.7], [0.7, 0.5]])
    F = np.array([[1.2, 0.9], [0.9, 1.2]])
    s = synth.small(method, A=A, F=F, seed=5)
    mask = abi.TERM_TC3A2A4B2B5 | abi.TERM_TC3A3B3B4B6
    r2, r3 = O.apply(s, mask)
    with Context(s, prec) as ctx:
        ctx.set_state()
        g2, g3 = ctx.apply(mask)
    assert rel(g3, r3) < tol


def test_unequal_channels_spin_polarised():
    A = np.array([[0.5, 0.6], [0.6, 0.4]])
    F = np.array([[1.0, 0.8], [0.8, 1.1]])
    s = synth.small("BITC", A=A, F=F, nspin=2, seed=6)
    r2, r3 = O.apply(s, abi.TERMS_TC)
    with Context(s, "fp64") as ctx:
        ctx.set_state()
        g2, g3 = ctx.apply(abi.TERMS_TC)
    assert rel(g2, r2) < FP64_TOL
    assert rel(g3, r3) < FP64_TOL


@pytest.mark.parametrize("prec,tol", [("fp64", FP64_TOL), ("mixed", MIXED_TOL)])
@pytest.mark.parametrize("method,term", [("HF", "hf2h"), ("TC", "tc2h"), ("BITC", "tc2h")])
def test_hartree_terms(method, term, prec, tol):
    """hf2h / tc2h (local potentials of the density) on the device vs the oracle,
    alone and together with the exchange term of the same H2 accumulator"""
    s = system(method)
    bit = abi.TERM_NAMES_EXTRA[term]
    for mask in (bit, bit | (abi.TERM_HF2X if method == "HF" else abi.TERM_TC2X)):
        r2, _ = O.apply(s, mask)
        with Context(s, prec) as ctx:
            ctx.set_state()
            g2, _ = ctx.apply(mask)
        assert rel(g2, r2) < tol


@pytest.mark.parametrize("prec,tol", [("fp64", FP64_TOL), ("mixed", MIXED_TOL)])
@pytest.mark.parametrize("tr", [False, True])
def test_one_body_terms(prec, tol, tr):
    """kinetic + pseudopotential (non-local projectors, local potential) vs the oracle"""
    s = system("TC", tr=tr, nr=(16, 16, 16), ecut=1.5, nbands=2, nocc=1) if tr else system("TC")
    pp = synth.pseudo(s, seed=44)
    for mask in (abi.TERM_KINETIC, abi.TERM_PSEUDO, abi.TERMS_H1):
        ref = O.apply_h1(s, mask, pp)
        with Context(s, prec) as ctx:
            ctx.set_pseudo(pp)
            got = ctx.apply_h1(mask)
        assert rel(got, ref) < tol


@pytest.mark.parametrize("prec,tol", [("fp64", FP64_TOL), ("mixed", MIXED_TOL)])
@pytest.mark.parametrize("method", ["HF", "TC", "BITC"])
@pytest.mark.parametrize("prune", [True, False])
def test_36_pruned_transforms(monkeypatch, method, prune, prec, tol):
    """36^3 default kernels with the band-limited grids pruned to the pencils
    their support meets (default) and without (TCG_NO_PRUNE), vs the oracle;
    a cutoff large enough that the support balls cover a good part of the grid"""
    if not prune:
        monkeypatch.setenv("TCG_NO_PRUNE", "1")
    s = system(method, nr=(36, 36, 36), nk=2, ecut=6.0, nbands=2, nocc=1)
    mask = abi.TERMS_HF if method == "HF" else abi.TERMS_TC
    r2, r3 = oracle_terms(s, mask)
    with Context(s, prec) as ctx:
        ctx.set_state()
        g2, g3 = ctx.apply(mask)
    assert rel(g2, r2) < tol
    if method != "HF":
        assert rel(g3, r3) < tol


@pytest.mark.parametrize("method", ["TC", "BITC"])
@pytest.mark.parametrize("sacc", ["qp-default", "qp-off", "3a3b6A-on"])
def test_36_shared_memory_accumulation(monkeypatch, method, sacc):
    """36^3 mixed precision: the inverse XY pass summing a chunk's sources in
    FP32 shared-memory planes -- on by default for the occupied-pair stage of
    tc3a2a4b2b5 (TCG_NO_QP_SACC turns it off), optional for the first stage
    of tc3a3b3b4b6 (TCG_SACC) -- vs the oracle"""
    if sacc == "qp-off":
        monkeypatch.setenv("TCG_NO_QP_SACC", "1")
    if sacc == "3a3b6A-on":
        monkeypatch.setenv("TCG_SACC", "1")
    s = system(method, nr=(36, 36, 36), nk=2, ecut=4.0, nbands=3, nocc=2)
    for mask in (abi.TERM_TC3A2A4B2B5, abi.TERM_TC3A3B3B4B6):
        _, r3 = oracle_terms(s, mask)
        with Context(s, "mixed") as ctx:
            ctx.set_state()
            _, g3 = ctx.apply(mask)
        assert rel(g3, r3) < MIXED_TOL


@pytest.mark.parametrize("prec,tol", [("fp64", FP64_TOL), ("mixed", MIXED_TOL)])
@pytest.mark.parametrize("method", ["TC", "BITC"])
@pytest.mark.parametrize("fuse", [True, False])
def test_36_shared_transforms(monkeypatch, method, fuse, prec, tol):
    """36^3, all TC terms at once: tc2x, tc3a3b3b4b6 and the band part of
    tc3a2a4b2b5 sharing their pair-density transforms (default) and as
    separate passes (TCG_NO_FUSE), vs the oracle"""
    if not fuse:
        monkeypatch.setenv("TCG_NO_FUSE", "1")
    s = system(method, nr=(36, 36, 36), nk=2, ecut=6.0, nbands=2, nocc=1)
    r2, r3 = oracle_terms(s, abi.TERMS_TC)
    with Context(s, prec) as ctx:
        ctx.set_state()
        g2, g3 = ctx.apply(abi.TERMS_TC)
    assert rel(g2, r2) < tol
    assert rel(g3, r3) < tol
