"""The batched SCF driver (polymer_b200/batch_scf.py) on the CPU with the oracle
as the Fock builder of every molecule.

* SP2 projection gives the spectral projector of a symmetric matrix (checked
  against eigh), leaving decoupled padded slots empty;
* the batched DIIS (a Cholesky solve in tensor operations, usable in a CUDA
  graph) gives the Pulay coefficients of the bordered system, over the valid
  history slots only; SP2 with a fixed step count matches the adaptive one;
* a batch of molecules of two sizes converges every molecule to the energy of
  the reference loop within 1e-8 Eh (the oracle ignores the screening knobs,
  so incremental builds are exact up to rounding), including the core guess.
"""
import numpy as np
import pytest
import torch

import oracle
from conftest import deck_of
from polymer_b200 import batch_scf, geometry, scf, system


def test_sp2_projector_matches_eigh():
    rng = np.random.default_rng(7)
    B, n, nocc = 3, 12, 4
    a = rng.normal(size=(B, n, n))
    f = torch.tensor(a + a.transpose(0, 2, 1))
    pad = torch.zeros((B, n), dtype=torch.bool)
    pad[1, -2:] = True
    f[1, -2:, :] = 0.0
    f[1, :, -2:] = 0.0
    x, steps, defect = batch_scf.sp2_projector(f, nocc, pad, tol=1e-13)
    xf, steps_f, defect_f = batch_scf.sp2_projector(f, nocc, pad, fixed_steps=steps + 4)
    assert float(defect.max()) < 1e-13 and float(defect_f.max()) < 1e-12
    assert float((xf - x).abs().max()) < 1e-11
    for b in range(B):
        m = n - int(pad[b].sum())
        e, v = np.linalg.eigh(f[b, :m, :m].numpy())
        ref = v[:, :nocc] @ v[:, :nocc].T
        assert np.abs(x[b, :m, :m].numpy() - ref).max() < 1e-10
        if m < n:
            assert np.abs(x[b, m:, :].numpy()).max() == 0.0
    assert steps < 100


def test_diis_coefficients_match_the_pulay_system():
    rng = np.random.default_rng(3)
    B, D, n = 4, 6, 5
    e = torch.tensor(rng.normal(size=(B, D, n, n)))
    valid = torch.ones((B, D), dtype=torch.bool)
    valid[1, 4:] = False
    valid[2, :] = False
    valid[2, 3] = True
    slot = torch.tensor([3])
    c = batch_scf.pulay_coefficients(e, valid, slot).numpy()
    for b in range(B):
        idx = np.nonzero(valid[b].numpy())[0]
        m = len(idx)
        ev = e[b].reshape(D, -1).numpy()[idx]
        a = np.zeros((m + 1, m + 1))
        a[:m, :m] = ev @ ev.T
        a[:m, m] = a[m, :m] = -1.0
        rhs = np.zeros(m + 1)
        rhs[m] = -1.0
        ref = np.linalg.solve(a, rhs)[:m]
        assert np.abs(c[b, idx] - ref).max() < 1e-9
        assert np.abs(np.delete(c[b], idx)).max(initial=0.0) == 0.0


class OracleBatch:
    """The DeviceBatch interface over the CPU oracle (one Fock build per molecule)."""

    def __init__(self, systems):
        self.systems = list(systems)
        self.ncgs = [s.basis.ncgs for s in self.systems]
        self.off = [0]
        for n in self.ncgs:
            self.off.append(self.off[-1] + n * n)
        self.f = [oracle.fock_builder(s) for s in self.systems]
        self.screen = [(0.0, 0.0)] * len(self.systems)
        self.builds = 0

    def __len__(self):
        return len(self.systems)

    def set_instance_screening(self, k, mixed_cutoff=0.0, density_tol=0.0):
        self.screen[k] = (mixed_cutoff, density_tol)

    def view(self, packed, k):
        n = self.ncgs[k]
        return packed[self.off[k]:self.off[k + 1]].view(n, n).t()

    def run_packed(self, p_c, out_c, out_x, stream=None):
        self.builds += 1
        for k, s in enumerate(self.systems):
            pc = self.view(p_c, k)
            if self.screen[k][1] > 0.0 and not bool(pc.abs().max() > 0):
                self.view(out_c, k).zero_()
                self.view(out_x, k).zero_()
                continue
            cc = torch.tensor(s.basis.cc, dtype=torch.float64)
            c, x = self.f[k]((cc.T @ pc @ cc)[None], None)
            self.view(out_c, k).copy_(c[0])
            self.view(out_x, k).copy_(x[0])

    def close(self):
        pass


@pytest.fixture(scope='module')
def molecules(reference_runs):
    w0 = system.build_system(deck_of(reference_runs['H2O_CCSD_ccpVDZ']), oracle.onee)
    w1 = system.build_system(geometry.water_deck(1, seed=4321), oracle.onee)
    ch4 = system.build_system(geometry.alkane_deck(1), oracle.onee)
    return [w0, ch4, w1]


@pytest.mark.parametrize('guess', ['nuclear', 'core'])
def test_batch_scf_reaches_the_reference_state(molecules, guess):
    plain = [scf.run_scf(s, scf_fock(s), variational=True).energy_variational for s in molecules]
    order = batch_scf.sorted_order(molecules)
    fb = OracleBatch([molecules[k] for k in order])
    res = batch_scf.run_batch_scf(molecules, batch_scf.BatchOptions(guess=guess, reset_every=4), device='cpu',
                                  batch=fb)
    assert res.converged.all()
    for k in range(len(molecules)):
        assert abs(res.energy[k] - plain[k]) < 1e-8, (k, res.energy[k], plain[k])
    assert res.builds == fb.builds


def scf_fock(s):
    f = oracle.fock_builder(s)
    return lambda p_p, p_ph=None: f(p_p, p_ph)
