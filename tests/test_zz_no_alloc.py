"""pfe_overlap_kinetic_noalloc (fixed device scratch, no allocation) against
pfe_overlap_kinetic (the allocating entry point), through the C ABI.

Both run the same kernel on the same inputs, so the results agree to the last
bit; the test allows 1e-14 relative to max|S_P|, |T_P|.  Two calls in a row
check that nothing left in the shared scratch leaks into the next call.  The
file is named to be collected last so it also runs after every other GPU test
in the same process.
"""
import ctypes

import numpy as np
import pytest

import oracle
from polymer_b200 import capi, fock, geometry, system

pytestmark = pytest.mark.gpu

RTOL = 1e-14


def _args(sysm):
    return fock.onee_args(sysm)


def _run(fn, a, n):
    s, t = np.full(n, np.nan), np.full(n, np.nan)
    L = capi.lib()
    capi.check(L, fn(ctypes.byref(a), capi.dptr(s), capi.dptr(t)))
    return s, t


CASES = {
    'h2o3_ccpvdz': lambda: geometry.water_deck(3, seed=2001),
    'c10h22_631gss': lambda: geometry.alkane_deck(10),
    'helix_pe_631g': lambda: geometry.polyethylene_deck('6-31G', cutoff1=2, cutoff2=3, kpoints=4),
}


@pytest.mark.parametrize('name', sorted(CASES))
def test_noalloc_matches_allocating_entry_point(name):
    sysm = system.build_system(CASES[name](), oracle.onee)
    a, keep = _args(sysm)
    n = sysm.basis.npgs ** 2 * sysm.ncell1
    L = capi.lib()
    s_ref, t_ref = _run(L.pfe_overlap_kinetic, a, n)
    for _ in range(2):
        s, t = _run(L.pfe_overlap_kinetic_noalloc, a, n)
        assert np.abs(s - s_ref).max() <= RTOL * np.abs(s_ref).max()
        assert np.abs(t - t_ref).max() <= RTOL * np.abs(t_ref).max()


def test_noalloc_matches_the_oracle_in_every_cell():
    """The shared kernel itself against the oracle's OVERLAP_KINETIC on a helical
    chain: S_P and T_P of every lattice cell (the helical image of the second
    centre included), not only the home cell."""
    from polymer_b200.system import from_fortran
    sysm = system.build_system(CASES['helix_pe_631g'](), oracle.onee)
    assert sysm.ncell1 > 1
    a, keep = _args(sysm)
    npgs, nc = sysm.basis.npgs, sysm.ncell1
    s_o, t_o, _ = oracle.onee_overlap(sysm)
    L = capi.lib()
    for _ in range(2):
        s, t = _run(L.pfe_overlap_kinetic_noalloc, a, npgs * npgs * nc)
        s, t = from_fortran(s, (nc,), npgs), from_fortran(t, (nc,), npgs)
        for c in range(nc):
            assert np.abs(s[c] - s_o[c]).max() <= 1e-13 * np.abs(s_o).max() + 1e-15, c
            assert np.abs(t[c] - t_o[c]).max() <= 1e-13 * np.abs(t_o).max() + 1e-15, c


def test_noalloc_refuses_inputs_beyond_its_scratch():
    """C40H82 6-31G** (1936 primitives) needs ~60 MB of results: refused with the size in the message."""
    sysm = system.build_system(geometry.alkane_deck(40), oracle.onee)
    a, keep = _args(sysm)
    n = sysm.basis.npgs ** 2 * sysm.ncell1
    L = capi.lib()
    s, t = np.zeros(n), np.zeros(n)
    rc = L.pfe_overlap_kinetic_noalloc(ctypes.byref(a), capi.dptr(s), capi.dptr(t))
    assert rc == -1  # PFE_EINVAL
    assert 'scratch' in capi.last_error(L)
