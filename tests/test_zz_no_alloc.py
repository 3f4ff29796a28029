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
from polymer_b200 import capi, geometry, system

pytestmark = pytest.mark.gpu

RTOL = 1e-14


def _args(sysm):
    b, d = sysm.basis, sysm.deck
    keep = dict(p_shell=np.asfortranarray(b.p_shell.astype(np.int32)),
                ang=np.ascontiguousarray(b.p_shell_ang.astype(np.int32)),
                atom=np.ascontiguousarray(b.pgs_atom.astype(np.int32)),
                x=np.ascontiguousarray(b.pgs[:, 0]), y=np.ascontiguousarray(b.pgs[:, 1]),
                z=np.ascontiguousarray(b.pgs[:, 2]), zt=np.ascontiguousarray(b.zt),
                iatom=np.array(d.atoms, dtype=np.int32),
                ax=np.array([c[0] for c in d.coords]), ay=np.array([c[1] for c in d.coords]),
                az=np.array([c[2] for c in d.coords]), ig=np.asfortranarray(sysm.igamma))
    a = capi.PfeOneeArgs()
    a.npgs, a.npshell, a.natom = b.npgs, b.npshell, d.natom
    a.p_shell = capi.iptr(keep['p_shell'])
    a.p_shell_ang = capi.iptr(keep['ang'])
    a.pgs_atom = capi.iptr(keep['atom'])
    a.pgsx, a.pgsy, a.pgsz = capi.dptr(keep['x']), capi.dptr(keep['y']), capi.dptr(keep['z'])
    a.zt = capi.dptr(keep['zt'])
    a.iatom = capi.iptr(keep['iatom'])
    a.atomx, a.atomy, a.atomz = capi.dptr(keep['ax']), capi.dptr(keep['ay']), capi.dptr(keep['az'])
    for k in range(3):
        a.cel1[k], a.cel2[k], a.period[k] = d.cel1[k], d.cel2[k], d.period[k]
    a.helix = d.helix
    a.igamma = capi.dptr(keep['ig'])
    return a, keep


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
