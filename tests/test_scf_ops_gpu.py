"""The SCF iteration kernels (include/polymer_scf.h, polymer_b200/scf_ops.py
DeviceOps) against the tensor-expression formulation of the same steps
(TorchOps, FP64) on seeded inputs: ragged orders (not multiples of the 32 x 32
tiles, more than one 8192-element chunk), several molecules per batch.

* next density: take / restart / incremental / live patterns, valid history
  cleared on restart;
* Fock assembly: F symmetrised, C/X/P references, the energy (fixed-order sum);
* commutator + DIIS over twelve iterations with the history slot cycling and a
  restart in the middle (the kernels keep the Gram matrix row by row, the
  formulation recomputes it): the same extrapolated Fock matrices;
* SP2: the start matrix, every step, and the projector against eigh;
* the finishing step: the new density and the statistics row.
"""
import types

import numpy as np
import pytest
import torch

from polymer_b200 import batch_scf, scf_ops

pytestmark = pytest.mark.gpu
F64 = torch.float64
DEV = torch.device('cuda', 0)


def _sym(gen, B, n):
    a = torch.randn((B, n, n), generator=gen, dtype=F64)
    return (a + a.transpose(1, 2)).to(DEV)


def _group(B, n, D, nocc, seed):
    gen = torch.Generator().manual_seed(seed)
    g = types.SimpleNamespace(B=B, n=n, nocc=nocc)
    g.h = _sym(gen, B, n)
    g.hfx = torch.rand((B, 1, 1), generator=gen, dtype=F64).to(DEV)
    g.e_nuc = torch.randn(B, generator=gen, dtype=F64).to(DEV)
    g.hist_e = torch.zeros((B, D, n, n), dtype=F64, device=DEV)
    g.hist_f = torch.zeros_like(g.hist_e)
    g.valid = torch.zeros((B, D), dtype=torch.bool, device=DEV)
    g.pad = torch.zeros((B, n), dtype=torch.bool, device=DEV)
    return g, gen


def _clone(g):
    c = types.SimpleNamespace(**vars(g))
    for k in ('hist_e', 'hist_f', 'valid'):
        setattr(c, k, getattr(g, k).clone())
    return c


def _close(a, b, rel=1e-13):
    scale = max(float(b.abs().max()), 1e-300)
    assert float((a - b).abs().max()) <= rel * scale, (float((a - b).abs().max()), scale)


@pytest.mark.parametrize('B,n', [(3, 37), (2, 130), (4, 64)])
def test_next_density_and_fock_assembly(B, n):
    dev_ops, ref_ops = scf_ops.DeviceOps(DEV), scf_ops.TorchOps()
    g, gen = _group(B, n, 4, 5, seed=11 + n)
    dev_ops.prepare(g)
    gr = _clone(g)
    gr.valid.fill_(True)
    g.valid.fill_(True)
    mats = {k: _sym(gen, B, n) for k in ('p', 'p_new', 'p_nuc', 'p_ref', 'dc', 'dx', 'c_ref', 'x_ref')}
    take = torch.tensor([True, False, True, False][:B], device=DEV)
    restart = torch.tensor([False, False, True, True][:B], device=DEV)
    incr = torch.tensor([1.0, 0.0, 1.0, 0.0][:B], dtype=F64, device=DEV)
    live = torch.tensor([1.0, 1.0, 0.0, 1.0][:B], dtype=F64, device=DEV)
    md = {k: v.clone() for k, v in mats.items()}
    mr = {k: v.clone() for k, v in mats.items()}
    dp_d, dp_r = torch.empty_like(mats['p']), torch.empty_like(mats['p'])
    dev_ops.next_density(g, md['p'], md['p_new'], md['p_nuc'], take, restart, incr, live, md['p_ref'], dp_d)
    ref_ops.next_density(gr, mr['p'], mr['p_new'], mr['p_nuc'], take, restart, incr, live, mr['p_ref'], dp_r)
    assert torch.equal(md['p'], mr['p']) and torch.equal(dp_d, dp_r)
    assert torch.equal(g.valid, gr.valid)
    f_d, e_d = dev_ops.fock_assemble(g, md['dc'], md['dx'], md['c_ref'], md['x_ref'], md['p'], md['p_ref'], incr)
    f_r, e_r = ref_ops.fock_assemble(gr, mr['dc'], mr['dx'], mr['c_ref'], mr['x_ref'], mr['p'], mr['p_ref'], incr)
    for k in ('c_ref', 'x_ref', 'p_ref'):
        assert torch.equal(md[k], mr[k]), k
    _close(f_d, f_r, 1e-15)
    assert torch.equal(f_d, f_d.transpose(1, 2))
    _close(e_d, e_r, 1e-13)


@pytest.mark.parametrize('B,n,D', [(3, 37, 8), (2, 130, 6)])
def test_commutator_and_diis_over_cycling_history(B, n, D):
    dev_ops, ref_ops = scf_ops.DeviceOps(DEV), scf_ops.TorchOps()
    g, gen = _group(B, n, D, 5, seed=29 + n)
    dev_ops.prepare(g)
    gr = _clone(g)
    slot = torch.zeros(1, dtype=torch.long, device=DEV)
    for it in range(12):
        if it == 7:   # a restart of molecule 1: its history is forgotten
            g.valid[1] = False
            gr.valid[1] = False
        fo = _sym(gen, B, n)
        # a commutator-sized perturbation that shrinks like a converging SCF
        a = torch.bmm(fo, _sym(gen, B, n)) * (0.7 ** it)
        fe_d = dev_ops.commutator(g, a, fo, slot)
        fe_r = ref_ops.commutator(gr, a, fo, slot)
        assert torch.equal(g.hist_e, gr.hist_e) and torch.equal(g.hist_f, gr.hist_f)
        assert torch.equal(g.valid, gr.valid) and torch.equal(fe_d, fe_r)
        fx_d = dev_ops.diis(g, slot)
        fx_r = ref_ops.diis(gr, slot)
        c_r = scf_ops.pulay_coefficients(gr.hist_e, gr.valid, slot)
        assert float((g.coef - c_r).abs().max()) < 1e-9 * max(1.0, float(c_r.abs().max())), it
        _close(fx_d, fx_r, 1e-9)
        slot.add_(1).remainder_(D)


@pytest.mark.parametrize('B,n,nocc', [(3, 37, 9), (2, 130, 20)])
def test_sp2_steps_and_projector(B, n, nocc):
    dev_ops, ref_ops = scf_ops.DeviceOps(DEV), scf_ops.TorchOps()
    gen = torch.Generator().manual_seed(5 + n)
    f = _sym(gen, B, n)
    pad = torch.zeros((B, n), dtype=torch.bool, device=DEV)
    pad[1, -3:] = True
    f[1, -3:, :] = 0.0
    f[1, :, -3:] = 0.0
    x_d, x_r = dev_ops.sp2_init(f, pad), ref_ops.sp2_init(f, pad)
    _close(x_d, x_r, 1e-14)
    x_r = x_d.clone()
    for _ in range(6):
        x2 = torch.bmm(x_d, x_d)
        d_d = dev_ops.sp2_step(x_d, x2, nocc)
        d_r = ref_ops.sp2_step(x_r, x2.clone(), nocc)
        assert torch.equal(x_d, x_r)
        _close(d_d, d_r, 1e-12)
    x, steps, defect = batch_scf.sp2_projector(f, nocc, pad, tol=1e-13, ops=dev_ops)
    assert float(defect.max()) < 1e-13 and steps < 120
    for b in range(B):
        m = n - int(pad[b].sum())
        e, v = np.linalg.eigh(f[b, :m, :m].cpu().numpy())
        ref = v[:, :nocc] @ v[:, :nocc].T
        assert np.abs(x[b, :m, :m].cpu().numpy() - ref).max() < 1e-10
        if m < n:
            assert float(x[b, m:, :].abs().max()) == 0.0


def test_finish_statistics():
    dev_ops, ref_ops = scf_ops.DeviceOps(DEV), scf_ops.TorchOps()
    B, n = 3, 130
    g, gen = _group(B, n, 4, 5, seed=71)
    dev_ops.prepare(g)
    q, p = _sym(gen, B, n), _sym(gen, B, n)
    e, fe, defect = (torch.randn(B, generator=gen, dtype=F64).to(DEV) for _ in range(3))
    pn_d, pn_r = torch.empty_like(q), torch.empty_like(q)
    st_d = torch.zeros((B, 4), dtype=F64, device=DEV)
    st_r = torch.zeros_like(st_d)
    dev_ops.finish(g, 2.0, q, p, pn_d, e, fe, defect, st_d)
    ref_ops.finish(g, 2.0, q, p, pn_r, e, fe, defect, st_r)
    assert torch.equal(pn_d, pn_r)
    _close(st_d, st_r, 1e-13)


def test_bad_arguments_are_refused():
    from polymer_b200 import capi
    L = capi.lib()
    assert L.pfe_scf_sp2_init(1, 0, None, None, None, None) == -1
    assert L.pfe_scf_diis(1, 4, 17, None, None, None, None, None, None, None, None, None) == -1
    assert 'pfe_scf_diis' in capi.last_error(L)
