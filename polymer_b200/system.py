"""The module state FOURINDEX_ERI reads, assembled on the host.

In the reference this state lives in Fortran module globals filled by
SINGLEPOINT (src/psinglepoint.f90:29-212): the basis (READ3), C2S/C2H,
S_P/S_C/T_C (OVERLAP_KINETIC), REDUCED_CEL1 (src/ponee.f90:359-409), the Boys
table IGAMMA (FMT_PRELIMINARY) and N_C (NUCLEAR_ATTRACTION).  :class:`System`
holds the same arrays.  Per-cell matrices are kept cell-major as
``M[c, i, j] = A(i, j, cell c)`` with the Fortran cell order (x fastest);
:func:`to_fortran` produces the column-major buffers the C ABI takes.

The one-electron integrals come from a pluggable provider: the CUDA library in
production (:mod:`polymer_b200.fock`), the CPU oracle in tests.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Callable, Optional, Tuple

import numpy as np

from . import basis as basis_mod
from .capi import PfeArgs, dptr, iptr, PFE_PREC_FP64
from .inputdeck import Deck, nuclear_repulsion

N_IGAMMA_T = 1701
N_IGAMMA_M = 28


def fmt_table() -> np.ndarray:
    """IGAMMA(0:1700,0:27) column-major, FMT_PRELIMINARY (src/pbasis.f90:1-27).

    F_m(i/20) by downward recursion from m = 50 + i/3; element-for-element the
    same arithmetic as the reference's scalar loop, vectorised over i.
    """
    i = np.arange(N_IGAMMA_T, dtype=np.float64)
    a = i / 20.0
    b = np.exp(-a)
    k = (50.0 + i / 3.0).astype(np.int64)
    c = np.zeros(N_IGAMMA_T)
    out = np.zeros((N_IGAMMA_T, N_IGAMMA_M), order='F')
    for j in range(int(k.max()), -1, -1):
        act = j <= k
        c = np.where(act, (2.0 * a * c + b) / float(2 * j + 1), c)
        if j < N_IGAMMA_M:
            out[:, j] = c
    return out


def cells_of(cel) -> list:
    """Cell triples in Fortran order (x fastest) for bounds -cel..cel."""
    return [(qx, qy, qz) for qz in range(-cel[2], cel[2] + 1)
            for qy in range(-cel[1], cel[1] + 1) for qx in range(-cel[0], cel[0] + 1)]


def to_fortran(m: np.ndarray) -> np.ndarray:
    """Cell-major (..., n, n) array -> column-major buffer with the same element map."""
    return np.ascontiguousarray(np.swapaxes(m, -1, -2))


def from_fortran(buf: np.ndarray, lead_shape, n: int) -> np.ndarray:
    return np.swapaxes(buf.reshape(tuple(lead_shape) + (n, n)), -1, -2)


@dataclasses.dataclass
class System:
    deck: Deck
    basis: basis_mod.Basis
    c2s: np.ndarray
    c2h: np.ndarray            # (2*(cel2x+cel1x)+1, ncgs, ncgs), index q + h3
    p2h: np.ndarray            # (2*(cel2x+cel1x)+1, npgs, npgs)
    igamma: np.ndarray         # (1701, 28) Fortran order
    s_p: np.ndarray            # (ncell1, npgs, npgs)
    t_p: np.ndarray
    n_p: np.ndarray
    s_c: np.ndarray            # (ncell1, ncgs, ncgs), helical-transformed like the reference
    t_c: np.ndarray
    n_c: np.ndarray
    reduced_cel1: Tuple[int, int, int]
    max_overlap: list          # per x cell, the printed MAXIMUM OVERLAP column
    e_nuc: float
    cells: list

    @property
    def ncell1(self) -> int:
        return len(self.cells)

    @property
    def h3(self) -> int:
        return self.deck.cel2[0] + self.deck.cel1[0]

    def cell_index(self, qx: int, qy: int = 0, qz: int = 0) -> int:
        c1 = self.deck.cel1
        n1x, n1y = 2 * c1[0] + 1, 2 * c1[1] + 1
        return (qx + c1[0]) + n1x * ((qy + c1[1]) + n1y * (qz + c1[2]))

    # ---- C ABI -----------------------------------------------------------------
    def pfe_args(self, p_p: Optional[np.ndarray] = None, p_p_helix: Optional[np.ndarray] = None,
                 *, precision: int = PFE_PREC_FP64, mixed_cutoff: float = 1.0e-6,
                 myid: int = 0, numprocs: int = 1, inttol: Optional[float] = None):
        """Build the C-ABI argument block; the returned tuple keeps buffers alive."""
        b, d = self.basis, self.deck
        keep = {}
        keep['p_shell'] = np.asfortranarray(b.p_shell.astype(np.int32))
        keep['ang'] = np.ascontiguousarray(b.p_shell_ang.astype(np.int32))
        keep['x'] = np.ascontiguousarray(b.pgs[:, 0])
        keep['y'] = np.ascontiguousarray(b.pgs[:, 1])
        keep['z'] = np.ascontiguousarray(b.pgs[:, 2])
        keep['zt'] = np.ascontiguousarray(b.zt)
        keep['cc'] = np.asfortranarray(b.cc)
        keep['s_p'] = to_fortran(self.s_p)
        keep['c2h'] = to_fortran(self.c2h) if d.helix != 0.0 else None
        keep['p_p'] = to_fortran(p_p) if p_p is not None else None
        keep['p_p_helix'] = to_fortran(p_p_helix) if (p_p_helix is not None and d.helix != 0.0) else None
        keep['igamma'] = np.asfortranarray(self.igamma)
        a = PfeArgs()
        a.npgs, a.ncgs, a.npshell, a.lmax = b.npgs, b.ncgs, b.npshell, basis_mod.BASIS_LMAX
        a.p_shell, a.p_shell_ang = iptr(keep['p_shell']), iptr(keep['ang'])
        a.pgsx, a.pgsy, a.pgsz, a.zt = dptr(keep['x']), dptr(keep['y']), dptr(keep['z']), dptr(keep['zt'])
        a.cc = dptr(keep['cc'])
        a.c2h = dptr(keep['c2h'])
        a.s_p = dptr(keep['s_p'])
        a.p_p = dptr(keep['p_p'])
        a.p_p_helix = dptr(keep['p_p_helix'])
        a.igamma = dptr(keep['igamma'])
        for k in range(3):
            a.cel1[k], a.cel2[k], a.reduced_cel1[k] = d.cel1[k], d.cel2[k], self.reduced_cel1[k]
            a.period[k] = d.period[k]
        a.helix = d.helix
        a.inttol = d.inttol if inttol is None else inttol
        a.print_level = d.print_level
        a.myid, a.numprocs = myid, numprocs
        a.precision_mode = precision
        a.mixed_cutoff = mixed_cutoff
        return a, keep


def onee_contract(sys_basis: basis_mod.Basis, m_p: np.ndarray) -> np.ndarray:
    """Per cell CC . M_P . CC^T (src/ponee.f90:285-293)."""
    cc = sys_basis.cc
    return np.einsum('ai,cij,bj->cab', cc, m_p, cc, optimize=True)


def helical_transform(m_c: np.ndarray, c2h: np.ndarray, deck: Deck, cells: list) -> np.ndarray:
    """M(i,j,q) <- sum_jj C2H(j,jj,q) M(i,jj,q) along x (src/ponee.f90:304-332)."""
    if deck.helix == 0.0:
        return m_c
    h3 = deck.cel2[0] + deck.cel1[0]
    out = m_c.copy()
    for c, (qx, qy, qz) in enumerate(cells):
        if qy == 0 and qz == 0:
            out[c] = m_c[c] @ c2h[qx + h3].T
    return out


OneElectron = Callable[['System'], Tuple[np.ndarray, np.ndarray, np.ndarray]]


def build_system(deck: Deck, onee: Callable, library: Optional[dict] = None) -> System:
    """SINGLEPOINT set-up order: READ3, C2S, C2H, S/T, REDUCED_CEL1, E_nuc, IGAMMA, V.

    ``onee(system_partial)`` returns cell-major (S_P, T_P, N_P) primitive
    matrices; it is called with a System whose integral fields are unset.
    """
    b = basis_mod.build_basis(deck, library)
    c2s = basis_mod.form_c2s(b, deck.spherical)
    h3 = deck.cel2[0] + deck.cel1[0]
    c2h, p2h = basis_mod.form_c2h(b, deck.helix, h3)
    cells = cells_of(deck.cel1)
    sysm = System(deck=deck, basis=b, c2s=c2s, c2h=c2h, p2h=p2h, igamma=fmt_table(),
                  s_p=None, t_p=None, n_p=None, s_c=None, t_c=None, n_c=None,
                  reduced_cel1=(0, 0, 0), max_overlap=[], e_nuc=nuclear_repulsion(deck), cells=cells)
    s_p, t_p, n_p = onee(sysm)
    sysm.s_p, sysm.t_p, sysm.n_p = s_p, t_p, n_p
    sysm.s_c = helical_transform(onee_contract(b, s_p), c2h, deck, cells)
    sysm.t_c = helical_transform(onee_contract(b, t_p), c2h, deck, cells)
    sysm.n_c = helical_transform(onee_contract(b, n_p), c2h, deck, cells)
    if deck.helix != 0.0:
        for qx in range(1, deck.cel1[0] + 1):
            a = sysm.s_c[sysm.cell_index(qx)]
            bm = sysm.s_c[sysm.cell_index(-qx)]
            if np.max(np.abs(a - bm.T)) > 1.0e-11:
                raise ValueError('HELIX IS INCORRECT')
    red, maxo = [0, 0, 0], []
    for ax in range(3):
        for k in range(0, deck.cel1[ax] + 1):
            q = [0, 0, 0]
            q[ax] = k
            m = float(np.max(np.abs(sysm.s_c[sysm.cell_index(*q)])))
            if ax == 0:
                maxo.append(m)
            if m > 1.0e-15:
                red[ax] = k
    sysm.reduced_cel1 = tuple(red)
    sysm.max_overlap = maxo
    return sysm
