"""CPU oracle: the checker for the CUDA Fock build.  TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this package.  It wraps oracle/oracle.c, a plain-C restatement of the
reference's FOURINDEX_ERI, OVERLAP_KINETIC, NUCLEAR_ATTRACTION,
FMT_PRELIMINARY, the primitive half of FORM_C2H and the P_P_HELIX part of
ROTATE_DENSITYMATRIX (see that file's header for the file:line map), through the
same pfe_args C-ABI block the product takes.

Pinned against the reference's recorded outputs in tests/test_oracle_golden.py
(SCF energies and components of data/H2O_CCSD_ccpVDZ_out, data/BH_MBGF_out,
data/FH_finiteT_MBPT_*_out, and the helical-polyethylene overlap/lattice
numbers of data/Polyethylene_B3LYP_631G_out).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, '_build', 'liboracle.so')

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int32)


class OneeArgs(ctypes.Structure):
    _fields_ = [('npgs', ctypes.c_int32), ('npshell', ctypes.c_int32), ('natom', ctypes.c_int32),
                ('p_shell', _ip), ('p_shell_ang', _ip), ('pgs_atom', _ip),
                ('pgsx', _dp), ('pgsy', _dp), ('pgsz', _dp), ('zt', _dp),
                ('iatom', _ip), ('atomx', _dp), ('atomy', _dp), ('atomz', _dp),
                ('cel1', ctypes.c_int32 * 3), ('cel2', ctypes.c_int32 * 3),
                ('period', ctypes.c_double * 3), ('helix', ctypes.c_double),
                ('igamma', _dp)]


def build():
    """Compile oracle.c with gcc (make) into oracle/_build/liboracle.so."""
    subprocess.run(['make', '-s', '-C', HERE], check=True)


_L = None


def lib():
    global _L
    if _L is None:
        if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(os.path.join(HERE, 'oracle.c')):
            build()
        from polymer_b200.capi import PfeArgs
        L = ctypes.CDLL(LIB)
        L.oracle_fourindex_eri.argtypes = [ctypes.POINTER(PfeArgs), _dp, _dp]
        L.oracle_fourindex_eri.restype = ctypes.c_int32
        L.oracle_fourindex_eri_sample.argtypes = [ctypes.POINTER(PfeArgs), _dp, _dp, ctypes.c_int32, ctypes.c_int32]
        L.oracle_fourindex_eri_sample.restype = ctypes.c_int32
        L.oracle_fmt_table.argtypes = [_dp]
        L.oracle_overlap_kinetic.argtypes = [ctypes.POINTER(OneeArgs), _dp, _dp]
        L.oracle_overlap_kinetic.restype = ctypes.c_int32
        L.oracle_nuclear_attraction.argtypes = [ctypes.POINTER(OneeArgs), _dp]
        L.oracle_nuclear_attraction.restype = ctypes.c_int32
        L.oracle_form_p2h.argtypes = [ctypes.c_int32, _ip, _ip, _ip, _ip, ctypes.c_double, ctypes.c_int32, _dp]
        L.oracle_form_p2h.restype = None
        L.oracle_rotate_density.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _dp, _dp, _dp]
        L.oracle_rotate_density.restype = None
        _L = L
    return _L


def fmt_table() -> np.ndarray:
    out = np.zeros((1701, 28), order='F')
    lib().oracle_fmt_table(out.ctypes.data_as(_dp))
    return out


def onee(sysm):
    """(S_P, T_P, N_P) cell-major, from the oracle's OVERLAP_KINETIC / NUCLEAR_ATTRACTION."""
    return _onee(sysm, with_v=True)


def _onee(sysm, with_v):
    from polymer_b200.system import from_fortran
    b, d = sysm.basis, sysm.deck
    keep = dict(p_shell=np.asfortranarray(b.p_shell.astype(np.int32)),
                ang=b.p_shell_ang.astype(np.int32), atom=b.pgs_atom.astype(np.int32),
                x=np.ascontiguousarray(b.pgs[:, 0]), y=np.ascontiguousarray(b.pgs[:, 1]),
                z=np.ascontiguousarray(b.pgs[:, 2]), zt=np.ascontiguousarray(b.zt),
                iatom=np.array(d.atoms, dtype=np.int32),
                ax=np.array([c[0] for c in d.coords]), ay=np.array([c[1] for c in d.coords]),
                az=np.array([c[2] for c in d.coords]), ig=np.asfortranarray(sysm.igamma))
    a = OneeArgs()
    a.npgs, a.npshell, a.natom = b.npgs, b.npshell, d.natom
    a.p_shell = keep['p_shell'].ctypes.data_as(_ip)
    a.p_shell_ang = keep['ang'].ctypes.data_as(_ip)
    a.pgs_atom = keep['atom'].ctypes.data_as(_ip)
    a.pgsx, a.pgsy, a.pgsz = (keep[k].ctypes.data_as(_dp) for k in ('x', 'y', 'z'))
    a.zt = keep['zt'].ctypes.data_as(_dp)
    a.iatom = keep['iatom'].ctypes.data_as(_ip)
    a.atomx, a.atomy, a.atomz = (keep[k].ctypes.data_as(_dp) for k in ('ax', 'ay', 'az'))
    for k in range(3):
        a.cel1[k], a.cel2[k], a.period[k] = d.cel1[k], d.cel2[k], d.period[k]
    a.helix = d.helix
    a.igamma = keep['ig'].ctypes.data_as(_dp)
    nc = sysm.ncell1
    s = np.zeros(b.npgs * b.npgs * nc)
    t = np.zeros_like(s)
    n = np.zeros_like(s)
    L = lib()
    assert L.oracle_overlap_kinetic(ctypes.byref(a), s.ctypes.data_as(_dp), t.ctypes.data_as(_dp)) == 0
    if with_v:
        assert L.oracle_nuclear_attraction(ctypes.byref(a), n.ctypes.data_as(_dp)) == 0
    return (from_fortran(s, (nc,), b.npgs).copy(), from_fortran(t, (nc,), b.npgs).copy(),
            from_fortran(n, (nc,), b.npgs).copy())


def onee_overlap_only(sysm):
    """(S_P, T_P, zeros) -- a system for the Fock build and energies of J/K only."""
    s, t, _ = _onee(sysm, with_v=False)
    return s, t, np.zeros_like(t)


def onee_overlap(sysm):
    """(S_P, T_P) only -- what the Fock build needs from the one-electron set-up."""
    s, t, _ = _onee(sysm, with_v=False)
    return s, t, None


def fourindex_eri(sysm, p_p: np.ndarray, p_p_helix=None, **kw):
    """(C_C, X_C) cell-major for cell-major P_P (and P_P_HELIX when helical)."""
    from polymer_b200.system import from_fortran
    b = sysm.basis
    a, keep = sysm.pfe_args(p_p, p_p_helix, **kw)
    nc = sysm.ncell1
    c = np.zeros(b.ncgs * b.ncgs * nc)
    x = np.zeros_like(c)
    rc = lib().oracle_fourindex_eri(ctypes.byref(a), c.ctypes.data_as(_dp), x.ctypes.data_as(_dp))
    if rc != 0:
        raise RuntimeError('oracle_fourindex_eri failed with %d' % rc)
    return from_fortran(c, (nc,), b.ncgs).copy(), from_fortran(x, (nc,), b.ncgs).copy()


def fourindex_eri_sample(sysm, p_p: np.ndarray, stride: int, offset: int, **kw):
    """The oracle restricted to bra shells I = offset (mod stride): a bounded CPU sample."""
    from polymer_b200.system import from_fortran
    b = sysm.basis
    a, keep = sysm.pfe_args(p_p, None, **kw)
    nc = sysm.ncell1
    c = np.zeros(b.ncgs * b.ncgs * nc)
    x = np.zeros_like(c)
    rc = lib().oracle_fourindex_eri_sample(ctypes.byref(a), c.ctypes.data_as(_dp), x.ctypes.data_as(_dp),
                                           stride, offset)
    if rc != 0:
        raise RuntimeError('oracle_fourindex_eri_sample failed with %d' % rc)
    return from_fortran(c, (nc,), b.ncgs).copy(), from_fortran(x, (nc,), b.ncgs).copy()


def fock_builder(sysm):
    """A FockBuilder for polymer_b200.scf.run_scf backed by the oracle (CPU)."""
    import torch

    def f(p_p, p_ph):
        pp = p_p.detach().cpu().numpy()
        ph = p_ph.detach().cpu().numpy() if p_ph is not None else None
        c, x = fourindex_eri(sysm, pp, ph)
        return (torch.tensor(c, dtype=torch.float64, device=p_p.device),
                torch.tensor(x, dtype=torch.float64, device=p_p.device))
    return f


def form_p2h(sysm) -> np.ndarray:
    """P2H cell-major [q + NH] (NH = CEL2X + CEL1X), each (npgs, npgs), from the
    oracle's FORM_C2H restatement."""
    from polymer_b200.basis import p2c_map
    b, d = sysm.basis, sysm.deck
    nh = d.cel2[0] + d.cel1[0]
    pax, pay, paz = (np.ascontiguousarray(x.astype(np.int32)) for x in (b.pax, b.pay, b.paz))
    p2c = np.ascontiguousarray(p2c_map(b, ghost_value=-1).astype(np.int32))
    out = np.zeros(b.npgs * b.npgs * (2 * nh + 1))
    lib().oracle_form_p2h(b.npgs, pax.ctypes.data_as(_ip), pay.ctypes.data_as(_ip), paz.ctypes.data_as(_ip),
                          p2c.ctypes.data_as(_ip), float(d.helix), nh, out.ctypes.data_as(_dp))
    from polymer_b200.system import from_fortran
    return from_fortran(out, (2 * nh + 1,), b.npgs).copy()


def rotate_density(sysm, p_p: np.ndarray, p2h: np.ndarray = None) -> np.ndarray:
    """P_P_HELIX [q1 + NH, q2 + CEL2X] (the layout of scf.rotate) from the
    oracle's ROTATE_DENSITYMATRIX restatement; p_p is cell-major over the x
    cells -CEL1X..CEL1X of a chain, p2h as form_p2h returns it (default: that)."""
    d = sysm.deck
    n = sysm.basis.npgs
    c1, c2 = d.cel1[0], d.cel2[0]
    nh = c1 + c2
    if p2h is None:
        p2h = form_p2h(sysm)
    cells = [sysm.cell_index(q, 0, 0) for q in range(-c1, c1 + 1)]
    pp_f = np.ascontiguousarray(np.swapaxes(np.asarray(p_p)[cells], -1, -2)).reshape(-1)
    p2h_f = np.ascontiguousarray(np.swapaxes(p2h, -1, -2)).reshape(-1)
    out = np.zeros(n * n * (2 * c2 + 1) * (2 * nh + 1))
    lib().oracle_rotate_density(n, c1, c2, p2h_f.ctypes.data_as(_dp), pp_f.ctypes.data_as(_dp),
                                out.ctypes.data_as(_dp))
    # column-major (n, n, q2, q1) -> [q1][q2][i][j]
    o = out.reshape(2 * nh + 1, 2 * c2 + 1, n, n)
    return np.swapaxes(o, -1, -2).copy()
