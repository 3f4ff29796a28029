"""The two-electron nuclear gradient (pfe_fourindex_eri_gradient, the molecular
branch of FOURINDEX_ERI_GRADIENT, src/pfourindexgradient.f90) against central
finite differences of the oracle's two-electron energy at fixed density.

For a fixed contracted density P_C (P_P = CC^T P_C CC: CC does not depend on
the geometry) the oracle's FOURINDEX_ERI gives J(R) and K(R); the gradient's
J part must be d/dR of E_J = 1/2 tr(P_C J(R)) and its K part d/dR of
E_K = -1/4 tr(P_C K(R)).  Displacements of +-h = 1e-4 bohr per atom and axis
(truncation error ~h^2); tolerance 1e-6 of the largest component + 1e-8.
"""
import numpy as np
import pytest

import oracle
from conftest import deck_of
from polymer_b200 import fock, geometry, inputdeck, system

pytestmark = pytest.mark.gpu

H = 1.0e-4


def _energies(deck, pc):
    s = system.build_system(deck, oracle.onee_overlap_only)
    pp = np.einsum('ai,cab,bj->cij', s.basis.cc, pc[None], s.basis.cc, optimize=True)
    c, x = oracle.fourindex_eri(s, pp)
    return 0.5 * np.sum(pc * c[0]), -0.25 * np.sum(pc * x[0])


def _displaced(deck, atom, axis, dh):
    coords = [list(c) for c in deck.coords]
    coords[atom][axis] += dh
    return inputdeck.make_deck(deck.atoms, coords, deck.basisset, spherical=deck.spherical, inttol=deck.inttol)


def _check(deck, atoms, seed):
    s = system.build_system(deck, oracle.onee_overlap_only)
    rng = np.random.default_rng(seed)
    n = s.basis.ncgs
    a = rng.normal(size=(n, n)) * 0.2
    pc = a + a.T
    pp = np.einsum('ai,cab,bj->cij', s.basis.cc, pc[None], s.basis.cc, optimize=True)
    gj, gk = fock.fourindex_eri_gradient(s, pp)
    assert gj.shape == (deck.natom, 3) and gk.shape == (deck.natom, 3)
    # translational invariance holds by construction; the J and K parts are not zero
    assert np.abs(gj.sum(0)).max() <= 1e-9 * np.abs(gj).max()
    scale_j, scale_k = np.abs(gj).max(), np.abs(gk).max()
    assert scale_j > 0.0 and scale_k > 0.0
    for at in atoms:
        for ax in range(3):
            ejp, ekp = _energies(_displaced(deck, at, ax, +H), pc)
            ejm, ekm = _energies(_displaced(deck, at, ax, -H), pc)
            fj, fk = (ejp - ejm) / (2 * H), (ekp - ekm) / (2 * H)
            assert abs(gj[at, ax] - fj) <= 1e-6 * scale_j + 1e-8, ('J', at, ax, gj[at, ax], fj)
            assert abs(gk[at, ax] - fk) <= 1e-6 * scale_k + 1e-8, ('K', at, ax, gk[at, ax], fk)


def test_water_ccpvdz_gradient_matches_finite_differences(reference_runs):
    """The reference's sample water, cc-pVDZ spherical (s, p and d shells), INTTOL 0."""
    _check(deck_of(reference_runs['H2O_CCSD_ccpVDZ']), atoms=(0, 1, 2), seed=3)


def test_ethane_631gss_gradient_matches_finite_differences():
    """6-31G** (cumulative sp shells and pure d), two of the eight atoms."""
    _check(geometry.alkane_deck(2, inttol=1e-14), atoms=(0, 2), seed=4)


def test_gradient_refuses_a_lattice():
    s = system.build_system(geometry.polyethylene_deck('STO-3G', cutoff1=1, cutoff2=1, kpoints=2), oracle.onee)
    pp = np.zeros((s.ncell1, s.basis.npgs, s.basis.npgs))
    with pytest.raises(RuntimeError):
        fock.fourindex_eri_gradient(s, pp)
