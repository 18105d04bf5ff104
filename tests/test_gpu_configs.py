"""CUDA path vs the CPU oracle at the benchmark configurations' own sizes.

C1  hf2x, fcc Si, 8 k, 12 bands (4 occupied), 10 Ha (~410 PW/k), grid 24^3: in full.
C2  tc2x + tc3*, same cell and k, 8 bands, grid 32^3: in full, TC and BITC.
C3  batched BITC, 64 k, 16 bands, 14 Ha, grid 36^3: a dozen bands against the
    committed oracle fixture (tests/golden/c3_subset.npz, made by
    tests/golden/make_c3_subset.py), and the total two- plus three-body energy
    of all occupied orbitals against the oracle's.
Plus every compiled fast grid size not covered elsewhere (32, 40, 48).

Tolerances: FP64 relative 1e-10 on H psi (max |diff| / max |oracle|);
mixed precision 2e-5 on H psi and |E_mixed - E_oracle| <= 1e-6 Ha on the
energy (the target of the mixed form).
"""
import os

import numpy as np
import pytest

from tc_b200 import abi, synth
from tc_b200.context import Context
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10
MIXED_TOL = 2e-5
ENERGY_TOL = 1e-6          # Ha, mixed precision vs the FP64 oracle
HERE = os.path.dirname(os.path.abspath(__file__))


def rel(a, b):
    d = np.abs(a - b).max()
    m = np.abs(b).max()
    return d / m if m > 0 else d


_cache = {}


def cfg(name, **kw):
    key = (name, tuple(sorted(kw.items())))
    if key not in _cache:
        _cache[key] = synth.config(name, **kw)
    return _cache[key]


def oracle(s, mask, owned=None):
    key = (id(s), mask, None if owned is None else owned.tobytes())
    if key not in _cache:
        _cache[key] = O.apply(s, mask, owned=owned)
    return _cache[key]


def occupied_mask(s):
    m = []
    for sp in range(s.nspin):
        for k in range(s.nk_irr):
            nb = int(s.nb_apply[sp][k])
            no = int(s.nocc[sp][k])
            m += [1] * min(no, nb) + [0] * max(0, nb - no)
    return np.array(m, dtype=np.uint8)


def gpu_apply(s, prec, mask, owned=None):
    with Context(s, prec) as ctx:
        ctx.set_state()
        return ctx.apply(mask, owned=owned)


@pytest.mark.parametrize("prec,tol", [("fp64", FP64_TOL), ("mixed", MIXED_TOL)])
def test_c1_full(prec, tol):
    s = cfg("C1")
    r2, _ = oracle(s, abi.TERMS_HF)
    g2, _ = gpu_apply(s, prec, abi.TERMS_HF)
    e = rel(g2, r2)
    e_ref, _ = s.energy_terms(r2, None)
    e_got, _ = s.energy_terms(g2, None)
    print(f"C1 {prec}: rel {e:.3e}, E2 oracle {e_ref.real:.12f}, |dE| {abs(e_got - e_ref):.3e} Ha")
    assert e < tol
    assert abs(e_got - e_ref) <= (1e-10 if prec == "fp64" else ENERGY_TOL)


@pytest.mark.parametrize("prec,tol", [("fp64", FP64_TOL), ("mixed", MIXED_TOL)])
@pytest.mark.parametrize("method", ["TC", "BITC"])
def test_c2_full(method, prec, tol):
    s = cfg("C2", method=method, **({"left_seed": 1} if method == "BITC" else {}))
    r2, r3 = oracle(s, abi.TERMS_TC)
    g2, g3 = gpu_apply(s, prec, abi.TERMS_TC)
    e2, e3 = rel(g2, r2), rel(g3, r3)
    E_ref = sum(s.energy_terms(r2, r3))
    E_got = sum(s.energy_terms(g2, g3))
    print(f"C2 {method} {prec}: rel H2 {e2:.3e} H3 {e3:.3e}, E oracle {E_ref.real:.12f}, "
          f"|dE| {abs(E_got - E_ref):.3e} Ha")
    assert e2 < tol and e3 < tol
    assert abs(E_got - E_ref) <= (1e-10 if prec == "fp64" else ENERGY_TOL)


@pytest.fixture(scope="module")
def c3():
    return cfg("C3"), np.load(os.path.join(HERE, "golden", "c3_subset.npz"))


@pytest.mark.parametrize("prec,tol", [("fp64", FP64_TOL), ("mixed", MIXED_TOL)])
def test_c3_subset_vs_fixture(c3, prec, tol):
    s, ref = c3
    nb = int(s.nb_apply[0][0])
    owned = np.zeros(s.nk_irr * nb, dtype=np.uint8)
    for k, b in ref["subset"]:
        owned[k * nb + b] = 1
    g2, g3 = gpu_apply(s, prec, abi.TERMS_TC, owned=owned)
    got2 = np.concatenate([s.band_view(g2, 0, k, b) for k, b in ref["subset"]])
    got3 = np.concatenate([s.band_view(g3, 0, k, b) for k, b in ref["subset"]])
    e2, e3 = rel(got2, ref["h2"]), rel(got3, ref["h3"])
    print(f"C3 subset {prec}: rel H2 {e2:.3e} H3 {e3:.3e}")
    assert e2 < tol and e3 < tol


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_c3_energy_vs_oracle(c3, prec):
    """two- plus three-body energy of all 256 occupied orbitals of C3"""
    s, ref = c3
    g2, g3 = gpu_apply(s, prec, abi.TERMS_TC, owned=occupied_mask(s))
    E2, E3 = s.energy_terms(g2, g3)
    dE = abs((E2 + E3) - (complex(ref["E2"]) + complex(ref["E3"])))
    print(f"C3 {prec}: E2 {E2.real:.12f} E3 {E3.real:.12f}, |dE| vs oracle {dE:.3e} Ha")
    assert dE <= (1e-9 if prec == "fp64" else ENERGY_TOL)


def small_n(n):
    key = ("small", n)
    if key not in _cache:
        _cache[key] = synth.small("BITC", nr=(n, n, n), nk=2, ecut=2.0, nbands=2, nocc=1, seed=3)
    return _cache[key]


@pytest.mark.parametrize("n", [32, 40, 48])
@pytest.mark.parametrize("prec,tol", [("fp64", FP64_TOL), ("mixed", MIXED_TOL)])
def test_fast_sizes_32_40_48(n, prec, tol):
    """compile-time-size kernels of the C2, C4 and C5 grids (radix 2, 5, 3)"""
    s = small_n(n)
    r2, r3 = oracle(s, abi.TERMS_TC)
    g2, g3 = gpu_apply(s, prec, abi.TERMS_TC)
    assert rel(g2, r2) < tol
    assert rel(g3, r3) < tol


FORMS_48 = {"default": {}, "z-shared": {"z": 3}, "z-registers": {"z": 4}, "xy-split": {"xy": 3},
            "one-thread-lines": {"xy": 1, "z": 1}, "separate-terms": {"fuse": 0}, "unpruned": {"prune": 0}}


@pytest.mark.parametrize("form", list(FORMS_48))
@pytest.mark.parametrize("prec,tol", [("fp64", FP64_TOL), ("mixed", MIXED_TOL)])
def test_48_split_line_forms(form, prec, tol):
    """48^3 (the C5 grid): the split-line kernels (four threads per line,
    48 = 4 x 12) on pruned band-limited grids, in every kernel form, all TC
    terms with and without shared transforms, vs the oracle"""
    s = small_n(48)
    r2, r3 = oracle(s, abi.TERMS_TC)
    with Context(s, prec) as ctx:
        ctx.set_state()
        ctx.set_forms(**FORMS_48[form])
        g2, g3 = ctx.apply(abi.TERMS_TC)
    assert rel(g2, r2) < tol
    assert rel(g3, r3) < tol


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_energy_reduction_on_device(prec):
    """tcg_energy (FP64 reduction on the GPU) against the host formula, on the
    C2 BITC system with time-reversal-free mesh and on a time-reversal-reduced
    system (conjugated images)"""
    import torch
    from tc_b200.context import Context
    for s in (cfg("C2", method="BITC", left_seed=1), synth.small("BITC", tr=True, nr=(16, 16, 16), ecut=1.5,
                                                                 nbands=2, nocc=1)):
        with Context(s, prec) as ctx:
            ctx.set_state()
            g2, g3 = ctx.apply(abi.TERMS_TC)
            d2 = torch.from_numpy(g2.view(np.float64)).cuda()
            d3 = torch.from_numpy(g3.view(np.float64)).cuda()
            torch.cuda.synchronize()
            E2, E3 = ctx.energy_device(d2.data_ptr(), d3.data_ptr())
            F2, F3 = ctx.energy_device(d2.data_ptr(), d3.data_ptr())
        h2, h3 = s.energy_terms(g2, g3)
        assert (E2, E3) == (F2, F3)                 # fixed-order reduction: same bits
        assert abs(E2 - h2) <= 1e-13 * max(1.0, abs(h2))
        assert abs(E3 - h3) <= 1e-13 * max(1.0, abs(h3))
