"""gsb_permute_records, the device reordering between the caller's stamp order and the FFT-size
bucket order of the draw and adjoint calls, against numpy fancy indexing."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('count,words', [(1, 1), (37, 17), (4096, 17), (1000, 3), (513, 40)])
def test_gather_and_scatter_match_numpy(count, words):
    import torch
    from galsim_b200 import _lib
    dev = _lib.Device.torch_device()
    rng = np.random.default_rng(count * 131 + words)
    src = rng.integers(0, 2**63, size=(count, words), dtype=np.int64)
    perm = rng.permutation(count).astype(np.int64)
    d_src = torch.from_numpy(src).to(dev)
    d_perm = torch.from_numpy(perm).to(dev)
    d_dst = torch.empty_like(d_src)
    _lib.permute_records(d_dst, d_src, d_perm)
    np.testing.assert_array_equal(d_dst.cpu().numpy(), src[perm])
    d_back = torch.empty_like(d_src)
    _lib.permute_records(d_back, d_dst, d_perm, scatter=True)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(d_back.cpu().numpy(), src)


def test_out_of_range_entries_are_skipped():
    import torch
    from galsim_b200 import _lib
    dev = _lib.Device.torch_device()
    src = torch.arange(8 * 2, dtype=torch.float64, device=dev).reshape(8, 2)
    perm = torch.tensor([7, -1, 5, 8, 3, 2, 1, 100], dtype=torch.int64, device=dev)
    dst = torch.full_like(src, -5.)
    _lib.permute_records(dst, src, perm)
    out = dst.cpu().numpy()
    ref = np.full((8, 2), -5.)
    s = src.cpu().numpy()
    for i, p in enumerate(perm.cpu().numpy()):
        if 0 <= p < 8:
            ref[i] = s[p]
    np.testing.assert_array_equal(out, ref)
