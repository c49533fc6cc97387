"""GPU: the table stage's FP64 exponentials (Tang's table-driven method, 32- and 256-entry
tables) against CUDA's exp (torch.exp on the same device) -- within 2 ulp on [-708, 709], 0 below -708."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip('torch')


@pytest.mark.parametrize('table_size', [32, 256])
def test_exp_fp64_within_two_ulp_of_cuda_exp(table_size):
    from galsim_b200 import _lib
    dev = _lib.Device.torch_device()
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.uniform(-708., 709., 200000), rng.uniform(-1., 1., 100000),
                        rng.uniform(-1e-8, 1e-8, 1000), np.arange(-700, 700, 0.5),
                        [0., -708., 709., np.log(2.) / 64, -np.log(2.) / 64]])
    dx = torch.as_tensor(x, device=dev)
    dy = torch.empty_like(dx)
    _lib.check(_lib.lib().gsb_exp_fp64_ex(_lib.ptr(dx), _lib.ptr(dy), len(x), table_size, _lib.Device.stream()))
    ref = torch.exp(dx)
    y = dy.cpu().numpy()
    r = ref.cpu().numpy()
    ulp = np.abs(y - r) / np.spacing(np.abs(r))
    assert ulp.max() <= 2.0, ulp.max()
    z = torch.as_tensor(np.array([-708.5, -750., -1e4]), device=dev)
    zo = torch.empty_like(z)
    _lib.check(_lib.lib().gsb_exp_fp64_ex(_lib.ptr(z), _lib.ptr(zo), 3, table_size, _lib.Device.stream()))
    assert np.all(zo.cpu().numpy() == 0.)
