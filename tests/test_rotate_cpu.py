"""ROTATE_DENSITYMATRIX and the primitive half of FORM_C2H against the oracle.

The host mirror builds P2H in polymer_b200/basis.py:form_c2h and rotates the
primitive density into P_P_HELIX in polymer_b200/scf.py:rotate (torch matrix
products: the same code runs on the GPU beside the CUDA Fock build).  The
oracle restates both in the reference's loop order (oracle_form_p2h,
src/pbasis.f90:134-413; oracle_rotate_density, src/pdensitymatrix.f90:516-563)
so the helical inputs of FOURINDEX_ERI are pinned by a second implementation.
"""
import numpy as np
import pytest
import torch

import oracle
from polymer_b200 import geometry, scf, system


def _chain(basis, c1, c2):
    return system.build_system(geometry.polyethylene_deck(basis, cutoff1=c1, cutoff2=c2, kpoints=4), oracle.onee)


def _density(s, seed):
    rng = np.random.default_rng(seed)
    n = s.basis.ncgs
    pc = rng.normal(size=(s.ncell1, n, n)) * 0.1
    return np.einsum('ai,cab,bj->cij', s.basis.cc, pc, s.basis.cc, optimize=True)


CASES = [('STO-3G', 1, 2), ('6-31G', 2, 3), ('6-31Gss', 1, 2)]


@pytest.mark.parametrize('basis,c1,c2', CASES)
def test_p2h_matches_oracle(basis, c1, c2):
    s = _chain(basis, c1, c2)
    p2h = oracle.form_p2h(s)
    assert p2h.shape == s.p2h.shape
    assert np.abs(p2h - s.p2h).max() <= 1e-15
    # it is a rotation: orthogonal blocks
    for k in range(p2h.shape[0]):
        assert np.abs(p2h[k] @ p2h[k].T - np.eye(s.basis.npgs)).max() <= 1e-14


@pytest.mark.parametrize('basis,c1,c2', CASES)
def test_rotate_matches_oracle(basis, c1, c2):
    s = _chain(basis, c1, c2)
    pp = _density(s, seed=c1 + 10 * c2)
    ref = oracle.rotate_density(s, pp)
    got = scf.rotate(scf.HostState(s), torch.tensor(pp)).numpy()
    assert got.shape == ref.shape
    assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max()
    # blocks outside the |Q1-Q2| <= CEL1 window are zero on both sides
    h3 = c1 + c2
    for q1 in range(-h3, h3 + 1):
        for q2 in range(-c2, c2 + 1):
            if abs(q1 - q2) > c1:
                assert not ref[q1 + h3, q2 + c2].any() and not got[q1 + h3, q2 + c2].any()
