"""The Davidson subspace step on the device (tcg_subspace_ritz,
tcg_gram_schmidt) against a numpy restatement of the reference's FP64 steps
(diagonalization_davidson.cpp:462-600, diagonalization_utils.cpp:7-119):
subspace matrices <Vref_i|H_n V_j>, eigenpairs sorted by the real part, left
vectors (X^-1)^H, Ritz vectors V X, energies diag(L^H H_n X), Gram-Schmidt
and its bi-orthogonal form.  Eigenvectors carry an arbitrary phase (Eigen and
LAPACK choose differently), so the comparison uses phase-free quantities:
eigenvalues, energies, and each Ritz vector up to its phase."""
import numpy as np
import pytest

from tc_b200.context import gram_schmidt, subspace_ritz

pytestmark = pytest.mark.gpu


def rnd(rng, *shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def ritz_numpy(V, Vref, HV, nout, biortho):
    Hn = [None if h is None else Vref.conj() @ h.T for h in HV]           # (i, j) = <Vref_i | H V_j>
    H = sum(h for h in Hn if h is not None)
    w, X = np.linalg.eig(H)
    order = np.argsort(w.real, kind="stable")
    w, X = w[order], X[:, order]
    XL = np.linalg.inv(X).conj().T
    L = XL if biortho else X
    e = np.array([np.zeros(nout) if h is None else np.einsum("ai,ab,bi->i", L[:, :nout].conj(), h, X[:, :nout])
                  for h in Hn])
    return w, e, (X[:, :nout].T @ V), (XL[:, :nout].T @ Vref)


def same_up_to_phase(a, b):
    for x, y in zip(a, b):
        ov = np.vdot(x, y)
        assert abs(abs(ov) - np.linalg.norm(x) * np.linalg.norm(y)) <= 1e-9 * np.linalg.norm(x) * np.linalg.norm(y)
        assert abs(np.linalg.norm(x) - np.linalg.norm(y)) <= 1e-9 * np.linalg.norm(y)


@pytest.mark.parametrize("biortho", [False, True])
@pytest.mark.parametrize("ndim,npw,nout", [(12, 180, 6), (64, 700, 32)])
def test_subspace_ritz(ndim, npw, nout, biortho):
    import torch
    rng = np.random.default_rng(ndim + npw + biortho)
    V = rnd(rng, ndim, npw)
    Vref = rnd(rng, ndim, npw) if biortho else V
    HV = [rnd(rng, ndim, npw), rnd(rng, ndim, npw), None]
    dev = lambda a: None if a is None else torch.from_numpy(np.ascontiguousarray(a)).cuda()
    w, e, Vo, Vl = subspace_ritz(dev(V), [dev(h) for h in HV], nout, Vref=dev(Vref) if biortho else None,
                                 biortho=biortho)
    w0, e0, V0, L0 = ritz_numpy(V, Vref, HV, nout, biortho)
    assert np.abs(w - w0).max() <= 1e-10 * np.abs(w0).max()
    assert np.abs(e[:2] - e0[:2]).max() <= 1e-9 * np.abs(e0[:2]).max()
    assert np.all(e[2] == 0)
    Vo = Vo.cpu().numpy()
    same_up_to_phase(Vo, V0)
    if biortho:
        Vl = Vl.cpu().numpy()
        P = Vo.T @ Vl.conj()            # sum_i |V_i><Vl_i|: phase-free
        P0 = V0.T @ L0.conj()
        assert np.abs(P - P0).max() <= 1e-9 * np.abs(P0).max()


def gs_numpy(V, Vl=None):
    V = V.copy()
    Vl = None if Vl is None else Vl.copy()
    for j in range(len(V)):
        for i in range(j):
            V[j] -= np.vdot(V[i] if Vl is None else Vl[i], V[j]) * V[i]
        V[j] /= np.linalg.norm(V[j])
        if Vl is not None:
            for i in range(j):
                Vl[j] -= np.vdot(V[i], Vl[j]) * Vl[i]
            Vl[j] /= np.conj(np.vdot(Vl[j], V[j]))
    return V, Vl


@pytest.mark.parametrize("biortho", [False, True])
def test_gram_schmidt(biortho):
    import torch
    rng = np.random.default_rng(7 + biortho)
    V = rnd(rng, 16, 300)
    Vl = rnd(rng, 16, 300) if biortho else None
    tV = torch.from_numpy(V.copy()).cuda()
    tL = torch.from_numpy(Vl.copy()).cuda() if biortho else None
    gram_schmidt(tV, tL)
    V0, L0 = gs_numpy(V, Vl)
    # the bi-orthogonal form divides by <l_j|v_j>, which amplifies rounding
    assert np.abs(tV.cpu().numpy() - V0).max() <= (1e-10 if biortho else 1e-12)
    if biortho:
        got = tL.cpu().numpy()
        assert np.abs(got - L0).max() <= 1e-10 * np.abs(L0).max()
        assert np.abs(got.conj() @ tV.cpu().numpy().T - np.eye(16)).max() <= 1e-10
    else:
        G = tV.cpu().numpy()
        assert np.abs(G.conj() @ G.T - np.eye(16)).max() <= 1e-12


def test_linear_dependence_is_reported():
    import torch
    from tc_b200 import TCError
    rng = np.random.default_rng(3)
    V = rnd(rng, 4, 50)
    V[3] = V[1] * (2 - 1j)
    t = torch.from_numpy(V).cuda()
    with pytest.raises(TCError) as e:
        gram_schmidt(t)
    assert e.value.code == 7
