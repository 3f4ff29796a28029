"""A multilayer perceptron trained and evaluated on the GPU by the library's own
kernels (include/polymer_guess.h): BF16 tensor-core products with FP32
accumulation, FP32 bias/SiLU/loss/Adam.  No counterpart in the reference; it
backs the learned initial guess (polymer_b200/guess.py).

Layout: activations [batch, features] row-major; layer l maps din_l -> dout_l
with W_l [din_l, dout_l] (FP32 master copy + BF16 copy used by the GEMMs) and
b_l.  All widths and the batch are padded to multiples of 64 (the GEMM's tile);
padded input columns are zero, padded outputs carry zero loss weight.
"""
from __future__ import annotations

import ctypes
import math
from typing import List, Optional, Sequence

import numpy as np
import torch

from . import capi

BF16 = torch.bfloat16
F32 = torch.float32


def pad64(n: int) -> int:
    return ((n + 63) // 64) * 64


def _p(t: Optional[torch.Tensor]):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


class MLP:
    def __init__(self, din: int, hidden: Sequence[int], dout: int, device='cuda', seed: int = 0):
        self.L = capi.lib()
        self.din, self.dout = din, dout
        self.dims = [pad64(din)] + [pad64(h) for h in hidden] + [pad64(dout)]
        self.device = torch.device(device)
        g = torch.Generator().manual_seed(seed)
        self.W: List[torch.Tensor] = []
        self.Wb: List[torch.Tensor] = []
        self.b: List[torch.Tensor] = []
        for l in range(len(self.dims) - 1):
            di, do = self.dims[l], self.dims[l + 1]
            real_in = din if l == 0 else hidden[l - 1]
            w = torch.zeros(di, do)
            w[:real_in] = torch.randn(real_in, do, generator=g) * math.sqrt(2.0 / real_in)
            if l == len(self.dims) - 2:
                w *= 0.1        # small initial outputs
            self.W.append(w.to(self.device, F32).contiguous())
            self.Wb.append(self.W[-1].to(BF16).contiguous())
            self.b.append(torch.zeros(do, device=self.device, dtype=F32))
        self.opt_m = [torch.zeros_like(t) for t in self.W + self.b]
        self.opt_v = [torch.zeros_like(t) for t in self.W + self.b]
        self.step = 0

    # ---------------------------------------------------------------- kernels
    def _stream(self):
        return ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def _gemm(self, a, b, c, m, n, k, ta=0, tb=0, acc=0):
        capi.check(self.L, self.L.pfe_mlp_gemm(_p(a), _p(b), _p(c), m, n, k, ta, tb, acc, self._stream()))

    def _pad_input(self, x: torch.Tensor) -> torch.Tensor:
        bsz = x.shape[0]
        xp = torch.zeros(pad64(bsz), self.dims[0], device=self.device, dtype=F32)
        xp[:bsz, :x.shape[1]] = x.to(self.device, F32)
        return xp

    def forward(self, x: torch.Tensor, keep: bool = False) -> torch.Tensor:
        """x [batch, din] -> y [batch, dout] (FP32)."""
        bsz = x.shape[0]
        xp = self._pad_input(x)
        m = xp.shape[0]
        hb = torch.empty(m, self.dims[0], device=self.device, dtype=BF16)
        capi.check(self.L, self.L.pfe_mlp_to_bf16(_p(xp), _p(hb), hb.numel(), self._stream()))
        self._acts = [hb]
        self._pre = []
        nl = len(self.W)
        h = None
        for l in range(nl):
            do = self.dims[l + 1]
            z = torch.empty(m, do, device=self.device, dtype=F32)
            self._gemm(hb, self.Wb[l], z, m, do, self.dims[l])
            h = torch.empty_like(z)
            act = 1 if l < nl - 1 else 0
            hb = torch.empty(m, do, device=self.device, dtype=BF16) if l < nl - 1 else None
            capi.check(self.L, self.L.pfe_mlp_bias_act(_p(z), _p(self.b[l]), _p(h), _p(hb), m, do, act,
                                                       self._stream()))
            self._pre.append(z)
            if hb is not None:
                self._acts.append(hb)
        if not keep:
            self._acts, self._pre = [], []
        return h[:bsz, :self.dout]

    def loss_and_grads(self, x: torch.Tensor, target: torch.Tensor, weight: torch.Tensor):
        """Weighted MSE over [batch, dout]; returns (loss, grads of W..., grads of b...)."""
        bsz = x.shape[0]
        y = self.forward(x, keep=True)
        m = self._pre[0].shape[0]
        do = self.dims[-1]
        yp = torch.zeros(m, do, device=self.device, dtype=F32)
        yp[:bsz, :self.dout] = y
        tp = torch.zeros_like(yp)
        tp[:bsz, :self.dout] = target.to(self.device, F32)
        wp = torch.zeros_like(yp)
        wp[:bsz, :self.dout] = weight.to(self.device, F32)
        wsum = float(wp.sum())
        dy = torch.empty_like(yp)
        loss = torch.zeros(1, device=self.device, dtype=F32)
        capi.check(self.L, self.L.pfe_mlp_mse(_p(yp), _p(tp), _p(wp), 1.0 / max(wsum, 1e-30), _p(dy), _p(loss),
                                              yp.numel(), self._stream()))
        gW = [None] * len(self.W)
        gb = [None] * len(self.W)
        dh = dy
        for l in reversed(range(len(self.W))):
            di, dout = self.dims[l], self.dims[l + 1]
            act = 1 if l < len(self.W) - 1 else 0
            dz = torch.empty_like(dh)
            dzb = torch.empty(dh.shape, device=self.device, dtype=BF16)
            capi.check(self.L, self.L.pfe_mlp_act_grad(_p(dh), _p(self._pre[l]), _p(dz), _p(dzb), dz.numel(), act,
                                                       self._stream()))
            gW[l] = torch.empty(di, dout, device=self.device, dtype=F32)
            self._gemm(self._acts[l], dzb, gW[l], di, dout, m, ta=1)        # X^T dZ
            gb[l] = torch.empty(dout, device=self.device, dtype=F32)
            capi.check(self.L, self.L.pfe_mlp_colsum(_p(dz), _p(gb[l]), m, dout, self._stream()))
            if l > 0:
                dh = torch.empty(m, di, device=self.device, dtype=F32)
                self._gemm(dzb, self.Wb[l], dh, m, di, dout, tb=1)          # dZ W^T
        self._acts, self._pre = [], []
        return float(loss.item()), gW, gb

    def adam_step(self, gW, gb, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8, decay=0.0):
        self.step += 1
        params = self.W + self.b
        copies = self.Wb + [None] * len(self.b)
        for i, (w, wb, g) in enumerate(zip(params, copies, gW + gb)):
            capi.check(self.L, self.L.pfe_mlp_adam(_p(w), _p(wb), _p(g), _p(self.opt_m[i]), _p(self.opt_v[i]),
                                                   w.numel(), lr, beta1, beta2, eps, self.step,
                                                   decay if i < len(self.W) else 0.0, self._stream()))

    # ---------------------------------------------------------------- state
    def state(self) -> dict:
        return {'dims': self.dims, 'din': self.din, 'dout': self.dout,
                'W': [w.cpu() for w in self.W], 'b': [b.cpu() for b in self.b]}

    def load(self, st: dict) -> None:
        self.W = [w.to(self.device, F32).contiguous() for w in st['W']]
        self.Wb = [w.to(BF16).contiguous() for w in self.W]
        self.b = [b.to(self.device, F32).contiguous() for b in st['b']]
