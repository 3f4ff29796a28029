"""The time-to-solution SCF driver (commutator DIIS, incremental builds) on the
CPU, with the oracle as its Fock builder.

It must converge to the same RHF state as the reference's loop: E[P] of the
final idempotent densities agree within 1e-8 Eh (the bar the fast path is held
to), in fewer iterations.  The incremental path is exercised by the same
builder (the oracle ignores the screening knobs, so J(P0) + J(P - P0) is exact
up to rounding).
"""
import numpy as np
import pytest
import torch

import oracle
from conftest import deck_of
from polymer_b200 import scf, system


class OracleDeviceFock:
    """The DeviceFock interface (from_pc, set_screening) over the CPU oracle."""

    def __init__(self, sysm):
        self.sys = sysm
        self.f = oracle.fock_builder(sysm)
        self.calls = 0

    def set_screening(self, mixed_cutoff=0.0, density_tol=0.0):
        pass

    def from_pc(self, p_c):
        self.calls += 1
        pc = p_c.reshape((1,) + tuple(p_c.shape[-2:]))
        cc = torch.tensor(self.sys.basis.cc, dtype=torch.float64)
        return self.f(cc.T @ pc @ cc, None)

    def __call__(self, p_p, p_ph=None):
        self.calls += 1
        return self.f(p_p, p_ph)


@pytest.fixture(scope='module')
def water(reference_runs):
    return system.build_system(deck_of(reference_runs['H2O_CCSD_ccpVDZ']), oracle.onee)


def test_fast_scf_reaches_the_reference_state(water):
    plain = scf.run_scf(water, OracleDeviceFock(water), variational=True)
    for opts in (scf.FastOptions(incremental=False), scf.FastOptions(incremental=True, reset_every=4)):
        fast = scf.run_scf_fast(water, OracleDeviceFock(water), opts=opts, device='cpu')
        assert fast.converged
        assert abs(fast.energy - plain.energy_variational) < 1e-8
        assert len(fast.iterations) < len(plain.iterations)


def test_variational_energy_matches_the_converged_reference_energy(water, reference_runs):
    plain = scf.run_scf(water, OracleDeviceFock(water), variational=True)
    assert abs(plain.energy_variational - reference_runs['H2O_CCSD_ccpVDZ']['expected']['total']) < 1e-8
