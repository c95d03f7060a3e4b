"""The libtorch extension (torch.ops.sagittasbr.rcs, a C++ torch::autograd::Function
over the C ABI) against the C ABI itself: sigma from sbr_run, gradients from
sbr_adjoint with the cotangent 8 pi w S, on CPU and CUDA tensors."""
import numpy as np
import pytest

import sagittasbr_b200 as sbr
from sagittasbr_b200 import meshes as M

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("device", ["cpu", "cuda"])
def test_cpp_autograd_function_matches_c_abi(device):
    import torch
    from sagittasbr_b200 import torch_ext
    v, t = M.ellipsoid_sh(n_theta=24, n_phi=48)
    th, ph = np.array([90.0, 60.0, 75.0]), np.array([0.0, 45.0, 10.0])
    verts = torch.tensor(v, dtype=torch.float64, device=device, requires_grad=True)
    freqs = torch.tensor([3e9, 5e9], dtype=torch.float64, device=device, requires_grad=True)
    sigma = torch_ext.rcs(verts, t, th, ph, freqs, 64, 64, 4.0, 3, precision=sbr.PREC_FP64)
    assert sigma.shape == (3, 2) and sigma.device.type == device
    wt = torch.tensor([[1.0, 2.0], [0.5, 1.0], [3.0, 0.25]], dtype=torch.float64, device=device)
    (sigma * wt).sum().backward()
    assert verts.grad.device.type == device and freqs.grad.device.type == device
    with sbr.Scene(v, t, want_fp64=True) as sc:
        job = sbr.JobSpec(th, ph, [3e9, 5e9], 64, 64, 4.0, 3)
        base = sbr.run(sc, job, precision=sbr.PREC_FP64)
        w = wt.cpu().numpy().ravel()
        g, gf = sbr.adjoint(sc, job, 8.0 * np.pi * w * base.field, precision=sbr.PREC_FP64)
    np.testing.assert_allclose(sigma.detach().cpu().numpy().ravel(), base.sigma_m2, rtol=1e-12)
    np.testing.assert_allclose(verts.grad.cpu().numpy(), g, rtol=1e-9, atol=1e-12 * np.abs(g).max())
    np.testing.assert_allclose(freqs.grad.cpu().numpy(), gf.reshape(3, 2).sum(axis=0), rtol=1e-9)


def test_cpp_and_python_autograd_agree_in_mixed_precision():
    import torch
    from sagittasbr_b200 import torch_ext
    from sagittasbr_b200.autograd import rcs as rcs_py
    v, t = M.ellipsoid_sh(n_theta=24, n_phi=48)
    th, ph = np.array([90.0, 80.0]), np.array([0.0, 30.0])
    out = []
    for fn in (torch_ext.rcs, rcs_py):
        verts = torch.tensor(v, dtype=torch.float64, requires_grad=True)
        freqs = torch.tensor([4e9], dtype=torch.float64, requires_grad=True)
        s = fn(verts, t, th, ph, freqs, 80, 80, 4.0, 4, precision=sbr.PREC_MIXED)
        s.mean().backward()
        out.append((s.detach().numpy(), verts.grad.numpy(), freqs.grad.numpy()))
    np.testing.assert_array_equal(out[0][0], out[1][0])
    np.testing.assert_allclose(out[0][1], out[1][1], rtol=1e-9, atol=1e-12 * np.abs(out[1][1]).max())
    np.testing.assert_allclose(out[0][2], out[1][2], rtol=1e-9)
