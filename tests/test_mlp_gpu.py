"""The learned-guess kernels (include/polymer_guess.h) against CPU references.

* pfe_mlp_gemm in its four transpose forms equals the product of the BF16-rounded
  operands accumulated in FP64, to FP32 accumulation error (1e-5 relative);
* the MLP's gradients (tensor-core forward and backward, SiLU, weighted MSE)
  equal those of the same network in FP64 on CPU with the same BF16 rounding
  of the GEMM operands, to 2e-3 relative (the BF16 rounding of dZ in the
  backward products);
* a few hundred Adam steps fit a smooth function.
"""
import ctypes

import numpy as np
import pytest
import torch

from polymer_b200 import capi
from polymer_b200.mlp import MLP

pytestmark = pytest.mark.gpu


def _bf(x):
    return x.to(torch.bfloat16).to(torch.float64)


@pytest.mark.parametrize('ta,tb', [(0, 0), (0, 1), (1, 0), (1, 1)])
def test_gemm_matches_reference(ta, tb):
    g = torch.Generator().manual_seed(ta * 2 + tb)
    m, n, k = 128, 192, 256
    a = torch.randn((k, m) if ta else (m, k), generator=g)
    b = torch.randn((n, k) if tb else (k, n), generator=g)
    ad, bd = a.to(torch.bfloat16).cuda(), b.to(torch.bfloat16).cuda()
    c = torch.zeros(m, n, device='cuda', dtype=torch.float32)
    L = capi.lib()
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    capi.check(L, L.pfe_mlp_gemm(ctypes.c_void_p(ad.data_ptr()), ctypes.c_void_p(bd.data_ptr()),
                                 ctypes.c_void_p(c.data_ptr()), m, n, k, ta, tb, 0, s))
    ref = (_bf(a).T if ta else _bf(a)) @ (_bf(b).T if tb else _bf(b))
    err = float((c.double().cpu() - ref).abs().max())
    assert err <= 1e-5 * float(ref.abs().max())


def _reference_grads(net, x, t, w):
    """FP64 CPU forward/backward of the same network, GEMM operands rounded to BF16."""
    W = [wi.double().cpu() for wi in net.W]
    b = [bi.double().cpu() for bi in net.b]
    xp = torch.zeros(x.shape[0], net.dims[0], dtype=torch.float64)
    xp[:, :x.shape[1]] = x.double()
    acts, pres = [xp], []
    h = xp
    for l in range(len(W)):
        z = _bf(h) @ _bf(W[l]) + b[l]
        pres.append(z)
        h = z * torch.sigmoid(z) if l < len(W) - 1 else z
        acts.append(h)
    y = h[:, :net.dout]
    wsum = float(w.sum())
    dy = torch.zeros_like(h)
    dy[:, :net.dout] = 2.0 * w.double() * (y - t.double()) / wsum
    gW, gb = [None] * len(W), [None] * len(W)
    dh = dy
    for l in reversed(range(len(W))):
        z = pres[l]
        if l < len(W) - 1:
            s = torch.sigmoid(z)
            dz = dh * s * (1.0 + z * (1.0 - s))
        else:
            dz = dh
        gW[l] = _bf(acts[l]).T @ _bf(dz)
        gb[l] = dz.sum(0)
        dh = _bf(dz) @ _bf(W[l]).T
    return gW, gb


def test_mlp_gradients_match_reference():
    torch.manual_seed(0)
    net = MLP(40, (256, 256, 256), 100, seed=3)
    x = torch.randn(64, 40)
    t = torch.randn(64, 100) * 0.1
    w = (torch.rand(64, 100) > 0.3).float()
    loss, gW, gb = net.loss_and_grads(x, t, w)
    rW, rb = _reference_grads(net, x, t, w)
    for l in range(len(gW)):
        for got, ref in ((gW[l], rW[l]), (gb[l], rb[l])):
            err = float((got.double().cpu() - ref).abs().max())
            assert err <= 2e-3 * float(ref.abs().max()) + 1e-7, (l, err, float(ref.abs().max()))


def test_adam_fits_a_smooth_function():
    torch.manual_seed(1)
    net = MLP(8, (256, 256, 256), 4, seed=1)
    x = torch.rand(512, 8) * 2 - 1
    t = torch.stack([torch.sin(x[:, 0] + x[:, 1]), x[:, 2] * x[:, 3], torch.cos(x[:, 4]), x[:, 5] ** 2], dim=1)
    w = torch.ones_like(t)
    first = net.loss_and_grads(x, t, w)[0]
    for _ in range(300):
        loss, gW, gb = net.loss_and_grads(x, t, w)
        net.adam_step(gW, gb, lr=2e-3)
    assert loss < 0.05 * first
