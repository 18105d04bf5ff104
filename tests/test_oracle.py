"""CPU checks of the oracle (the FP64 restatement the CUDA path is compared
with) and of the host-side input generation.  No GPU is used here."""
import numpy as np
import pytest

from tc_b200 import abi, synth
from oracle import oracle as O

FOURPI = 4 * np.pi


@pytest.mark.parametrize("nr", [(12, 10, 8), (9, 15, 7), (16, 16, 16), (20, 25, 14)])
def test_fft_matches_numpy(nr):
    rng = np.random.default_rng(1)
    N = int(np.prod(nr))
    g = rng.standard_normal(N) + 1j * rng.standard_normal(N)
    shape = (nr[2], nr[1], nr[0])
    fwd = O.fft3d(g, nr, True)
    ref = np.fft.fftn(g.reshape(shape)).ravel() / N
    assert np.abs(fwd - ref).max() <= 1e-14 * np.abs(ref).max()
    bwd = O.fft3d(g, nr, False)
    ref = (np.fft.ifftn(g.reshape(shape)) * N).ravel()
    assert np.abs(bwd - ref).max() <= 1e-14 * np.abs(ref).max()


def test_jastrow_formulas():
    """u(G) and V_2body(G) of the RPA Jastrow (jastrow_functions.cpp:58-97)"""
    s = synth.small("TC")
    A, F = 0.5, 1.2
    for G in ([0.3, -0.2, 0.5], [1.7, 0.0, 0.0], [0.0, 0.0, 0.0], [2.5, -1.1, 0.4]):
        g2 = float(np.dot(G, G))
        u = O.uk(s, G, 0, 0)
        v = O.tc2body(s, G, 0, 1)
        if g2 < 1e-12:
            assert u == pytest.approx(-FOURPI * A * F * F, rel=1e-15)
            assert v == pytest.approx(-2 * np.pi * A * A / F, rel=1e-15)
        else:
            g = np.sqrt(g2)
            assert u == pytest.approx(FOURPI * A / (g2 * (1 + F * F * g2)), rel=1e-14)
            ref = (FOURPI / g2 - FOURPI * A / (1 + F * F * g2)
                   + np.pi * A * A / (F * F * g) * (np.pi * F * F * g2 + (4 + 2 * F * F * g2) * np.arctan(F * g / 2)
                                                      - (4 + 4 * F * F * g2) * np.arctan(F * g)))
            assert v == pytest.approx(ref, rel=1e-12, abs=1e-14)


def test_divergence_sums_numpy_vs_oracle():
    s = synth.config("C1")
    a, v = O.sum_of_vaux(s)
    assert a == pytest.approx(s.alpha_Vaux, rel=1e-15)
    assert np.abs(v - s.sum_Vaux).max() <= 1e-13 * np.abs(v).max()


@pytest.mark.parametrize("method", ["TC", "BITC"])
def test_density_numpy_vs_oracle(method):
    s = synth.small(method)
    d = O.density(s)
    assert np.abs(d - s.density).max() <= 1e-12 * np.abs(d).max()
    # electrons per cell: sum n / (N N_k) per spin = occupied bands (f = 2 split over spins)
    ne = d[0].sum().real / (s.N * s.num_kpoints)
    assert ne == pytest.approx(2.0, rel=1e-12)


@pytest.mark.parametrize("method", ["TC", "BITC"])
def test_symmetry_reduced_equals_expanded(method):
    """A time-reversal-reduced k-set gives the same H psi at the irreducible k
    as the explicitly expanded full-BZ description (alias-free grid)."""
    from _expand import expand
    s = synth.small(method, tr=True, nr=(16, 16, 16), ecut=1.5, nbands=2, nocc=1)
    e = expand(s)
    h2, h3 = O.apply(s, abi.TERMS_TC)
    g2, g3 = O.apply(e, abi.TERMS_TC)
    err = mx = 0.0
    for k in range(s.nk_irr):
        a = int(e.meta["first_of_irr"][k])
        for b in range(int(s.nb_apply[0][k])):
            x = s.band_view(h2 + h3, 0, k, b)
            y = e.band_view(g2 + g3, 0, a, b)
            err = max(err, np.abs(x - y).max())
            mx = max(mx, np.abs(y).max())
    assert err <= 1e-13 * mx


def _pw_system(method):
    return synth.heg_config(nr=(20, 20, 20), nocc=7, ntrial=7, noise=0.0, method=method, nelec=14)


def test_hf2x_plane_waves_known_answer():
    """HF exchange of plane-wave orbitals: H psi_j(G_j) = -(4pi/2 Omega) sum_i f_i / |G_j-G_i|^2
    (i != j) + f_j d_corr (hf2x.cpp:93-104, 150-200), by direct summation."""
    s = _pw_system("HF")
    h2, _ = O.apply(s, abi.TERM_HF2X)
    M = s.meta["mills"][0]
    Gv = M @ s.recip
    occ = [int(np.argmax(np.abs(s.orb(0, 0, b)))) for b in range(int(s.nbands[0]))]
    dc = -(1 / np.sqrt(np.pi * s.alpha_Vaux) - s.sum_Vaux[0] / (s.num_kpoints * s.omega)) / 2
    tbf = -FOURPI / (s.num_kpoints * s.omega) / 2
    for j in range(int(s.nb_apply[0][0])):
        pj = occ[j]
        ref = 0.0
        for i in range(int(s.nocc[0][0])):
            d = Gv[pj] - Gv[occ[i]]
            d2 = d @ d
            ref += s.fill(0, 0, i) * (0.0 if d2 < 1e-8 else 1.0 / d2)
        ref *= tbf
        if j < int(s.nocc[0][0]):
            ref += s.fill(0, 0, j) * dc
        got = s.band_view(h2, 0, 0, j)
        assert got[pj] == pytest.approx(ref, rel=1e-12, abs=1e-14)
        others = np.delete(np.abs(got), pj)
        assert others.max() <= 1e-13


def test_tc2x_plane_waves_known_answer():
    """tc2x of plane-wave orbitals: H psi_j(G_j) = -(1/2 Omega) sum_i f_i [V_2body(D) + |D|^2 u(D)],
    D = G_j - G_i, plus f_j d_corr (tc2x.cpp:349-388, 408-511)."""
    s = _pw_system("TC")
    h2, _ = O.apply(s, abi.TERM_TC2X)
    M = s.meta["mills"][0]
    Gv = M @ s.recip
    occ = [int(np.argmax(np.abs(s.orb(0, 0, b)))) for b in range(int(s.nbands[0]))]
    dc = -(1 / np.sqrt(np.pi * s.alpha_Vaux) - s.sum_Vaux[0] / (s.num_kpoints * s.omega)) / 2
    tbf = -1.0 / (s.num_kpoints * s.omega) / 2
    for j in range(int(s.nb_apply[0][0])):
        pj = occ[j]
        ref = 0.0
        for i in range(int(s.nocc[0][0])):
            d = Gv[pj] - Gv[occ[i]]
            ref += s.fill(0, 0, i) * (O.tc2body(s, d, 0, 0) + (d @ d) * O.uk(s, d, 0, 0))
        ref *= tbf
        if j < int(s.nocc[0][0]):
            ref += s.fill(0, 0, j) * dc
        got = s.band_view(h2, 0, 0, j)
        assert got[pj] == pytest.approx(ref, rel=1e-11, abs=1e-13)


@pytest.mark.parametrize("name", ["small_hf", "small_tc", "small_bitc", "small_bitc_tr"])
def test_oracle_matches_golden_fixture(name):
    import os
    from golden.make_golden import mask_of, system
    s = system(name)
    ref = np.load(os.path.join(os.path.dirname(__file__), "golden", name + ".npz"))
    assert np.array_equal(ref["psi"], s.psi)
    h2, h3 = O.apply(s, mask_of(s))
    for got, want in ((h2, ref["h2"]), (h3, ref["h3"])):
        m = np.abs(want).max()
        if m > 0:
            assert np.abs(got - want).max() <= 1e-12 * m


def test_config_shapes():
    """plane-wave counts of the benchmark cells at their Ha cutoffs"""
    c1 = synth.config("C1")
    assert (int(c1.npw.min()), int(c1.npw.max())) == (410, 412)
    assert c1.N == 24 ** 3 and c1.num_kpoints == 8 and int(c1.nb_apply.sum()) == 96
    c2 = synth.config("C2")
    assert c2.N == 32 ** 3 and int(c2.nb_apply.sum()) == 64


def test_energy_functional_weights():
    """E_n = sum f e_n / N_k with 1/2 (two-body), 1/3 (three-body)"""
    s = synth.small("TC")
    h2 = s.psi.copy()     # <phi_i|phi_i> = 1 -> e_2 = 1 for every occupied band
    h3 = 2 * s.psi
    e2, e3 = s.energy_terms(h2, h3)
    n_occ = int(s.nocc.sum())
    assert e2.real == pytest.approx(2.0 * n_occ / 2.0 / s.num_kpoints)
    assert e3.real == pytest.approx(2.0 * 2.0 * n_occ / 3.0 / s.num_kpoints)
