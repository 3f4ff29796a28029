"""The steps of a batched SCF iteration around the Fock build, on a group of
molecules of equal size (batch_scf._Group): the density of the next build,
Fock assembly with the energy, the DIIS commutator and Pulay extrapolation,
SP2 projector steps and the iteration's statistics.

Two implementations with one interface:

* ``DeviceOps`` -- the CUDA kernels of libpolymer_fock (include/polymer_scf.h)
  on CUDA tensors, one to three launches per step on the current stream (so a
  whole iteration can be captured into a CUDA graph).  The dense products
  between the steps are batched cuBLAS GEMMs (``torch.bmm``).
* ``TorchOps`` -- the same arithmetic as tensor expressions: the formulation
  the kernels are tested against, and what the CPU tests of the batched SCF's
  host logic run on CPU tensors.

``ops_for(device)`` picks ``DeviceOps`` for CUDA devices (the library must
load; there is no fallback) and ``TorchOps`` otherwise.
"""
from __future__ import annotations

import ctypes

import torch

F64 = torch.float64


def _trace(x: torch.Tensor) -> torch.Tensor:
    return x.diagonal(dim1=-2, dim2=-1).sum(-1)


class TorchOps:
    """Tensor-expression formulation of every step (any device)."""

    def prepare(self, g) -> None:
        pass

    def next_density(self, g, p, p_new, p_nuc, take, restart, incr, live, p_ref, dp) -> None:
        upd = torch.where(take[:, None, None], p_new, p)
        if p_nuc is not None:
            upd = torch.where(restart[:, None, None], p_nuc, upd)
            g.valid &= ~restart[:, None]
        p.copy_(upd)
        dp.copy_((p - p_ref * incr[:, None, None]) * live[:, None, None])

    def fock_assemble(self, g, dc, dx, c_ref, x_ref, p, p_ref, incr):
        im = incr[:, None, None]
        cv = dc + c_ref * im
        xv = dx + x_ref * im
        c_ref.copy_(cv)
        x_ref.copy_(xv)
        p_ref.copy_(p)
        f = g.h + cv - 0.5 * g.hfx * xv
        f = 0.5 * (f + f.transpose(1, 2))
        e = (p * (g.h + 0.5 * cv - 0.25 * g.hfx * xv)).sum((1, 2)) + g.e_nuc
        return f, e

    def commutator(self, g, a, fo, slot) -> torch.Tensor:
        err = a - a.transpose(1, 2)
        g.hist_f.index_copy_(1, slot, fo.unsqueeze(1))
        g.hist_e.index_copy_(1, slot, err.unsqueeze(1))
        g.valid.index_fill_(1, slot, True)
        return err.abs().amax((1, 2))

    def diis(self, g, slot) -> torch.Tensor:
        c = pulay_coefficients(g.hist_e, g.valid, slot)
        return torch.einsum('bd,bdij->bij', c, g.hist_f)

    def sp2_init(self, f, pad) -> torch.Tensor:
        d = f.diagonal(dim1=-2, dim2=-1)
        r = f.abs().sum(-1) - d.abs()
        big = torch.finfo(F64).max
        lo = torch.where(pad, torch.full_like(d, big), d - r).amin(-1)
        hi = torch.where(pad, torch.full_like(d, -big), d + r).amax(-1)
        hi = torch.maximum(hi, lo + 1e-8)
        n = f.shape[-1]
        eye = torch.eye(n, dtype=F64, device=f.device)
        x = (hi[:, None, None] * eye - f) / (hi - lo)[:, None, None]
        # padded slots: X0 = 0 there, a fixed point of both maps
        return torch.where(pad[:, :, None] | pad[:, None, :], torch.zeros_like(x), x)

    def sp2_step(self, x, x2, nocc) -> torch.Tensor:
        t1, t2 = _trace(x), _trace(x2)
        defect = (t1 - t2).abs()
        up = (t2 - nocc).abs() < (2.0 * t1 - t2 - nocc).abs()
        x.copy_(torch.where(up[:, None, None], x2, 2.0 * x - x2))
        return defect

    def finish(self, g, scale, q, p, p_new, e, fe, defect, stats) -> None:
        pn = scale * q
        p_new.copy_(pn)
        dchg = torch.sqrt(((pn - p) ** 2).sum((1, 2)) / float(g.n * g.n))
        stats.copy_(torch.stack([e, fe, dchg, defect], 1))


def _spd_solve(a: torch.Tensor, b: torch.Tensor) -> torch.Tensor:
    """Solve a x = b for a batch of small symmetric positive definite a [B, m, m]
    (Cholesky, unrolled over m in tensor operations: no host synchronisation,
    no solver workspace -- usable inside a CUDA graph)."""
    m = a.shape[-1]
    L = torch.zeros_like(a)
    for j in range(m):
        s = a[:, j, j] - (L[:, j, :j] ** 2).sum(-1)
        ljj = torch.sqrt(s.clamp_min(1e-300))
        L[:, j, j] = ljj
        if j + 1 < m:
            L[:, j + 1:, j] = (a[:, j + 1:, j] - (L[:, j + 1:, :j] * L[:, j:j + 1, :j]).sum(-1)) / ljj[:, None]
    y = torch.zeros_like(b)
    for j in range(m):
        y[:, j] = (b[:, j] - (L[:, j, :j] * y[:, :j]).sum(-1)) / L[:, j, j]
    x = torch.zeros_like(b)
    for j in reversed(range(m)):
        x[:, j] = (y[:, j] - (L[:, j + 1:, j] * x[:, j + 1:]).sum(-1)) / L[:, j, j]
    return x


def pulay_coefficients(hist_e: torch.Tensor, valid: torch.Tensor, slot: torch.Tensor) -> torch.Tensor:
    """Pulay coefficients per molecule over the valid history slots [B, D]:
    c = G^-1 1 / (1^T G^-1 1) with G the Gram matrix of the commutators, scaled
    by its largest valid diagonal and with 1e-12 added to that diagonal; the
    newest slot alone when the solve is not finite."""
    B, D = valid.shape
    e = hist_e.view(B, D, -1)
    g = torch.bmm(e, e.transpose(1, 2))
    vm = valid.to(F64)
    scale = (g.diagonal(dim1=-2, dim2=-1) * vm).amax(-1).clamp_min(1e-300)
    g = g / scale[:, None, None]
    a = g * vm[:, :, None] * vm[:, None, :] + torch.diag_embed(1.0 - vm + vm * 1e-12)
    y = _spd_solve(a, vm)
    c = y / y.sum(-1, keepdim=True)
    ok = torch.isfinite(c).all(-1)
    newest = torch.nn.functional.one_hot(slot.expand(B), D).to(F64)
    return torch.where(ok[:, None], c, newest)


class DeviceOps:
    """The CUDA kernels of include/polymer_scf.h on CUDA tensors (current stream)."""

    def __init__(self, device: torch.device):
        from . import capi
        self.L = capi.lib()
        self.capi = capi
        self.device = device

    @staticmethod
    def _p(t):
        return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(None)

    def _s(self):
        return ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def _check(self, rc):
        self.capi.check(self.L, rc)

    def prepare(self, g) -> None:
        """Scratch and the persistent DIIS Gram matrices of group g (before any capture)."""
        D = g.hist_e.shape[1]
        nw = int(self.L.pfe_scf_workspace(g.B, g.n, D))
        g.work = torch.empty(max(nw, 1), dtype=F64, device=self.device)
        g.gram = torch.zeros((g.B, D, D), dtype=F64, device=self.device)
        g.coef = torch.zeros((g.B, D), dtype=F64, device=self.device)

    def next_density(self, g, p, p_new, p_nuc, take, restart, incr, live, p_ref, dp) -> None:
        D = g.hist_e.shape[1]
        P = self._p
        self._check(self.L.pfe_scf_next_density(g.B, g.n, D, P(p), P(p_new), P(p_nuc), P(take),
                                                P(restart if p_nuc is not None else None), P(incr), P(live),
                                                P(p_ref), P(dp), P(g.valid), self._s()))

    def fock_assemble(self, g, dc, dx, c_ref, x_ref, p, p_ref, incr):
        P = self._p
        f = torch.empty((g.B, g.n, g.n), dtype=F64, device=self.device)
        e = torch.empty(g.B, dtype=F64, device=self.device)
        self._check(self.L.pfe_scf_fock_assemble(g.B, g.n, P(g.h), P(dc), P(dx), P(c_ref), P(x_ref), P(p), P(p_ref),
                                                 P(incr), P(g.hfx), P(g.e_nuc), P(f), P(e), P(g.work), self._s()))
        return f, e

    def commutator(self, g, a, fo, slot) -> torch.Tensor:
        P = self._p
        fe = torch.empty(g.B, dtype=F64, device=self.device)
        self._check(self.L.pfe_scf_commutator(g.B, g.n, g.hist_e.shape[1], P(a.contiguous()), P(fo.contiguous()),
                                              P(slot), P(g.hist_e), P(g.hist_f), P(g.valid), P(fe), P(g.work),
                                              self._s()))
        return fe

    def diis(self, g, slot) -> torch.Tensor:
        P = self._p
        fx = torch.empty((g.B, g.n, g.n), dtype=F64, device=self.device)
        self._check(self.L.pfe_scf_diis(g.B, g.n, g.hist_e.shape[1], P(g.hist_e), P(g.hist_f), P(g.valid), P(slot),
                                        P(g.gram), P(g.coef), P(fx), P(g.work), self._s()))
        return fx

    def sp2_init(self, f, pad) -> torch.Tensor:
        f = f.contiguous()
        x = torch.empty_like(f)
        self._check(self.L.pfe_scf_sp2_init(f.shape[0], f.shape[-1], self._p(f), self._p(pad), self._p(x), self._s()))
        return x

    def sp2_step(self, x, x2, nocc) -> torch.Tensor:
        B, n = x.shape[0], x.shape[-1]
        defect = torch.empty(B, dtype=F64, device=self.device)
        work = torch.empty(B, dtype=F64, device=self.device)
        self._check(self.L.pfe_scf_sp2_step(B, n, int(nocc), self._p(x), self._p(x2), self._p(defect),
                                            self._p(work), self._s()))
        return defect

    def finish(self, g, scale, q, p, p_new, e, fe, defect, stats) -> None:
        P = self._p
        self._check(self.L.pfe_scf_finish(g.B, g.n, float(scale), P(q.contiguous()), P(p), P(p_new), P(e), P(fe),
                                          P(defect), P(stats), P(g.work), self._s()))


def ops_for(device: torch.device):
    return DeviceOps(device) if device.type == 'cuda' else TorchOps()
