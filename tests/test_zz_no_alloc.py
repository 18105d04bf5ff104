"""The allocation-free divergence-sum entry point (tcg_sum_of_vaux_noalloc)
against the regular one (tcg_sum_of_vaux), on two calls in a row.

Some hosts cannot allocate device memory from inside the library: their memory
pool has reserved the GPU up front, or they must avoid the device-wide
synchronisation that cudaMalloc / cudaFree imply.  They pass device inputs and
outputs, and the library works in a static device array.  This file is
collected last so that a failure here does not hide the other GPU tests; it
also passes alone in a fresh process."""
import numpy as np
import pytest

from tc_b200 import synth
from tc_b200.context import sum_of_vaux, sum_of_vaux_noalloc

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["C1", "small-tr"])
def test_noalloc_matches_regular_twice(name):
    import torch
    s = synth.config("C1") if name == "C1" else synth.small("TC", tr=True)
    alpha_ref, ref = sum_of_vaux(s)
    kirr = np.ascontiguousarray(s.kvec[s.kall_off[:-1]])
    dev = torch.device("cuda", 0)
    kirr_t = torch.from_numpy(kirr).to(dev)
    kall_t = torch.from_numpy(np.ascontiguousarray(s.kvec)).to(dev)
    # every output buffer exists before the free-memory reading, so that the
    # only device work inside the window is the library's own
    outs = [torch.full((s.nk_irr,), float("nan"), dtype=torch.float64, device=dev) for _ in range(3)]
    torch.cuda.synchronize()
    # warm-up: the first call on a device looks the static array up and may
    # load the kernels' module; it is checked like the others
    sum_of_vaux_noalloc(s, kirr_t.data_ptr(), kall_t.data_ptr(), outs[0].data_ptr())
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(dev)[0]
    for out in outs[1:]:
        alpha = sum_of_vaux_noalloc(s, kirr_t.data_ptr(), kall_t.data_ptr(), out.data_ptr())
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info(dev)[0] == free0, "device free memory changed across the call"
    for out in outs:
        got = out.cpu().numpy()
        assert abs(alpha - alpha_ref) <= 1e-15 * abs(alpha_ref)
        assert np.all(np.isfinite(got))
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


def test_noalloc_rejects_oversize():
    import torch
    from tc_b200 import TCError
    s = synth.config("C1")
    dev = torch.device("cuda", 0)
    k = torch.zeros((200, 3), dtype=torch.float64, device=dev)
    out = torch.zeros(200, dtype=torch.float64, device=dev)

    class Big:
        recip = s.recip
        omega = s.omega
        nk_irr = 200
        nk_all = 200
    with pytest.raises(TCError):
        sum_of_vaux_noalloc(Big, k.data_ptr(), k.data_ptr(), out.data_ptr())


def test_noalloc_rejects_nonfinite_k():
    """A NaN k-vector sets the failure flag of its (k, q) blocks before the
    fractional wrap loops; the call returns TCG_ERR_NUMERIC, and the next call
    with good inputs is unaffected."""
    import torch
    from tc_b200 import TCError
    s = synth.config("C1")
    dev = torch.device("cuda", 0)
    kirr = np.ascontiguousarray(s.kvec[s.kall_off[:-1]]).copy()
    kirr[0, 1] = np.nan
    kirr_t = torch.from_numpy(kirr).to(dev)
    kall_t = torch.from_numpy(np.ascontiguousarray(s.kvec)).to(dev)
    out = torch.zeros(s.nk_irr, dtype=torch.float64, device=dev)
    with pytest.raises(TCError):
        sum_of_vaux_noalloc(s, kirr_t.data_ptr(), kall_t.data_ptr(), out.data_ptr())
    alpha_ref, ref = sum_of_vaux(s)
    kirr_t.copy_(torch.from_numpy(np.ascontiguousarray(s.kvec[s.kall_off[:-1]])))
    sum_of_vaux_noalloc(s, kirr_t.data_ptr(), kall_t.data_ptr(), out.data_ptr())
    torch.cuda.synchronize()
    assert np.abs(out.cpu().numpy() - ref).max() <= 1e-12 * np.abs(ref).max()
