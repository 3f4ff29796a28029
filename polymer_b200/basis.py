"""Primitive / contracted Gaussian basis exactly as the reference builds it.

Restates READ3 (src/pread.f90:584-1482): primitives are created per basis-file
line with exponent ``ZT = A*scale`` and contraction coefficients
``CC = b*(2A/PI)^(3/4)*(4A)^(L/2)/sqrt(norm)`` (src/pread.f90:641,671,811,844,
921,954); primitive *shells* group the Cartesian components of one centre and
exponent (src/pread.f90:1079-1102); a p/d/f primitive without a same-exponent
s (and p, d) partner gets zero-coefficient *ghost* primitives and zero
contracted rows (src/pread.f90:1103-1421) so that every shell is cumulative:
a shell of angular momentum L carries every Cartesian component of total
power <= L.  ``P_SHELL(shell, i, j, k)`` maps powers to 1-based primitive
indices, -1 where absent.

Also restates FORM_C2S (src/pbasis.f90:31-130) and the C2H/P2H helical
component rotations of FORM_C2H (src/pbasis.f90:134-427).
"""
from __future__ import annotations

import dataclasses
import json
import math
import os
from typing import Dict, List, Optional

import numpy as np

from .inputdeck import PI, ELEMENTS, Deck

BASIS_LMAX = 3
_DATA = os.path.join(os.path.dirname(__file__), 'basis_data', 'basis_sets.json')
_BASIS_CACHE: Dict[str, dict] = {}

# Component order and normalisation divisors of each shell type (src/pread.f90:
# 616-1019).  Each entry: (powers, contracted-row offset from the shell's
# first row, divisor under the sqrt).
_P_COMPS = [((1, 0, 0), 0, 1.0), ((0, 1, 0), 1, 1.0), ((0, 0, 1), 2, 1.0)]
_D_COMPS = [((2, 0, 0), 0, 3.0), ((0, 2, 0), 1, 3.0), ((0, 0, 2), 2, 3.0),
            ((1, 1, 0), 3, 1.0), ((0, 1, 1), 4, 1.0), ((1, 0, 1), 5, 1.0)]
_F_COMPS = [((3, 0, 0), 0, 15.0), ((0, 3, 0), 1, 15.0), ((0, 0, 3), 2, 15.0),
            ((2, 1, 0), 3, 3.0), ((0, 2, 1), 4, 3.0), ((1, 0, 2), 5, 3.0),
            ((1, 2, 0), 6, 3.0), ((0, 1, 2), 7, 3.0), ((2, 0, 1), 8, 3.0),
            ((1, 1, 1), 9, 1.0)]


def load_basis_library(name: str, path: Optional[str] = None) -> dict:
    """Element -> shell list for a basis set, from the bundled table or a file."""
    if path is not None:
        from .basis_data.make_basis_json import parse_file
        return parse_file(path)
    if not _BASIS_CACHE:
        with open(_DATA) as fh:
            _BASIS_CACHE.update(json.load(fh))
    if name not in _BASIS_CACHE:
        raise KeyError('basis set %s is not bundled (have %s)' % (name, sorted(_BASIS_CACHE)))
    return _BASIS_CACHE[name]


@dataclasses.dataclass
class Basis:
    npgs: int
    ncgs: int
    npshell: int
    pax: np.ndarray          # (npgs,) int
    pay: np.ndarray
    paz: np.ndarray
    pgs: np.ndarray          # (npgs, 3) centres (bohr)
    pgs_atom: np.ndarray     # (npgs,) 1-based atom index
    zt: np.ndarray           # (npgs,) exponents
    cc: np.ndarray           # (ncgs, npgs) contraction matrix
    cgs: np.ndarray          # (ncgs, 3)
    p_shell: np.ndarray      # (npshell, 5, 5, 5) int32, 1-based primitive index, -1 absent
    p_shell_ang: np.ndarray  # (npshell,) int32
    nreal_pgs: int           # before ghosts
    nreal_cgs: int

    def shell_components(self, s: int):
        """(powers, 0-based primitive) of shell s in the reference's loop order."""
        L = int(self.p_shell_ang[s])
        out = []
        for i1 in range(L + 1):
            for i2 in range(L + 1 - i1):
                for i3 in range(L + 1 - i1 - i2):
                    out.append(((i1, i2, i3), int(self.p_shell[s, i1, i2, i3]) - 1))
        return out


def build_basis(deck: Deck, library: Optional[dict] = None) -> Basis:
    """READ3: primitives, contraction matrix, ghosts and the shell map."""
    lib = library if library is not None else load_basis_library(deck.basisset)
    pax: List[int] = []
    pay: List[int] = []
    paz: List[int] = []
    pgs: List[List[float]] = []
    patom: List[int] = []
    zt: List[float] = []
    cgs: List[List[float]] = []
    ccent: Dict[tuple, float] = {}

    def add_prim(powers, xyz, atom, a):
        pax.append(powers[0]); pay.append(powers[1]); paz.append(powers[2])
        pgs.append(list(xyz)); patom.append(atom); zt.append(a)
        return len(zt)  # 1-based

    for ia, (z, xyz) in enumerate(zip(deck.atoms, deck.coords), start=1):
        sym = ELEMENTS[z - 1]
        if sym not in lib:
            raise KeyError('ORBITAL BASIS SET NOT FOUND for %s' % sym)
        for typ, scale, prims in lib[sym]:
            typ = typ.upper()
            if typ == 'S':
                cgs.append(list(xyz)); row = len(cgs)
                for a, b, *_ in prims:
                    ip = add_prim((0, 0, 0), xyz, ia, a * scale)
                    ccent[(row, ip)] = b * math.exp(0.75 * math.log(2.0 * a / PI))
            elif typ == 'P':
                for _ in range(3):
                    cgs.append(list(xyz))
                row0 = len(cgs) - 2
                for a, b, *_ in prims:
                    for pw, off, div in _P_COMPS:
                        ip = add_prim(pw, xyz, ia, a * scale)
                        ccent[(row0 + off, ip)] = b * math.exp(0.75 * math.log(2.0 * a / PI)) * math.sqrt(4.0 * a)
            elif typ == 'SP':
                for _ in range(4):
                    cgs.append(list(xyz))
                row0 = len(cgs) - 3
                for a, b, dd in prims:
                    ip = add_prim((0, 0, 0), xyz, ia, a * scale)
                    ccent[(row0, ip)] = b * math.exp(0.75 * math.log(2.0 * a / PI))
                    for pw, off, div in _P_COMPS:
                        ip = add_prim(pw, xyz, ia, a * scale)
                        ccent[(row0 + 1 + off, ip)] = dd * math.exp(0.75 * math.log(2.0 * a / PI)) * math.sqrt(4.0 * a)
            elif typ == 'D':
                for _ in range(6):
                    cgs.append(list(xyz))
                row0 = len(cgs) - 5
                for a, b, *_ in prims:
                    for pw, off, div in _D_COMPS:
                        ip = add_prim(pw, xyz, ia, a * scale)
                        v = b * math.exp(0.75 * math.log(2.0 * a / PI)) * math.sqrt(4.0 * a) ** 2
                        ccent[(row0 + off, ip)] = v / math.sqrt(div) if div != 1.0 else v
            elif typ == 'F':
                for _ in range(10):
                    cgs.append(list(xyz))
                row0 = len(cgs) - 9
                for a, b, *_ in prims:
                    for pw, off, div in _F_COMPS:
                        ip = add_prim(pw, xyz, ia, a * scale)
                        v = b * math.exp(0.75 * math.log(2.0 * a / PI)) * math.sqrt(4.0 * a) ** 3
                        ccent[(row0 + off, ip)] = v / math.sqrt(div) if div != 1.0 else v
            else:
                raise ValueError('ANGULAR MOMENTUM NOT YET SUPPORTED: %s' % typ)
    nreal_pgs, nreal_cgs = len(zt), len(cgs)
    if nreal_pgs > 1024 or nreal_cgs > 1024:
        # The reference caps both at 1024 (src/pread.f90:625,632); this library does
        # not, but records the fact for callers comparing against it.
        pass

    # --- shell structure (src/pread.f90:1077-1421) ---
    shells: List[Dict[tuple, int]] = []
    shell_ang: List[int] = []
    for i in range(1, nreal_pgs + 1):
        if pax[i - 1] + pay[i - 1] + paz[i - 1] == 0:
            shells.append({(0, 0, 0): i})
            shell_ang.append(0)

    def same_centre_exp(s, i):
        j0 = shells[s][(0, 0, 0)]
        return (pgs[j0 - 1][0] == pgs[i - 1][0] and pgs[j0 - 1][1] == pgs[i - 1][1]
                and pgs[j0 - 1][2] == pgs[i - 1][2] and zt[j0 - 1] == zt[i - 1])

    for i in range(1, nreal_pgs + 1):
        L = pax[i - 1] + pay[i - 1] + paz[i - 1]
        if L == 0:
            continue
        pw = (pax[i - 1], pay[i - 1], paz[i - 1])
        flag = False
        # no early exit: the reference assigns the component to every matching shell
        for s in range(len(shells)):
            if same_centre_exp(s, i) and pw not in shells[s]:
                flag = True
                shells[s][pw] = i
                shell_ang[s] = L
        if not flag:
            ghosts = [(0, 0, 0)]
            if L >= 2:
                ghosts += [(1, 0, 0), (0, 1, 0), (0, 0, 1)]
            if L >= 3:
                ghosts += [(2, 0, 0), (0, 2, 0), (0, 0, 2), (1, 1, 0), (0, 1, 1), (1, 0, 1)]
            sh: Dict[tuple, int] = {}
            for g in ghosts:
                cgs.append(list(pgs[i - 1]))
                ip = add_prim(g, pgs[i - 1], patom[i - 1], zt[i - 1])
                sh[g] = ip
                # zero coefficient on the new contracted row: nothing to store
            sh[pw] = i
            shells.append(sh)
            shell_ang.append(L)

    npgs, ncgs, npshell = len(zt), len(cgs), len(shells)
    cc = np.zeros((ncgs, npgs), dtype=np.float64)
    for (row, ip), v in ccent.items():
        cc[row - 1, ip - 1] = v
    p_shell = np.full((npshell, BASIS_LMAX + 2, BASIS_LMAX + 2, BASIS_LMAX + 2), -1, dtype=np.int32)
    for s, sh in enumerate(shells):
        for pw, ip in sh.items():
            p_shell[s, pw[0], pw[1], pw[2]] = ip
    b = Basis(npgs=npgs, ncgs=ncgs, npshell=npshell,
              pax=np.array(pax, dtype=np.int32), pay=np.array(pay, dtype=np.int32),
              paz=np.array(paz, dtype=np.int32), pgs=np.array(pgs, dtype=np.float64),
              pgs_atom=np.array(patom, dtype=np.int32), zt=np.array(zt, dtype=np.float64),
              cc=cc, cgs=np.array(cgs, dtype=np.float64), p_shell=p_shell,
              p_shell_ang=np.array(shell_ang, dtype=np.int32),
              nreal_pgs=nreal_pgs, nreal_cgs=nreal_cgs)
    _check_cumulative(b)
    return b


def _check_cumulative(b: Basis) -> None:
    for s in range(b.npshell):
        for pw, ip in b.shell_components(s):
            if ip < 0:
                raise ValueError('shell %d lacks component %s: basis is not cumulative' % (s + 1, pw))


def p2c_map(b: Basis, ghost_value: int) -> np.ndarray:
    """Contracted row of each primitive (0-based); ``ghost_value`` for ghosts."""
    out = np.full(b.npgs, ghost_value, dtype=np.int64)
    for i in range(b.npgs):
        nz = np.nonzero(b.cc[:, i])[0]
        if len(nz) > 1:
            raise ValueError('GENERAL CONTRACTION NOT YET IMPLEMENTED')
        if len(nz) == 1:
            out[i] = nz[0]
    return out


def form_c2s(b: Basis, spherical: bool) -> np.ndarray:
    """Cartesian -> spherical row combination matrix (src/pbasis.f90:31-130)."""
    c2s = np.eye(b.ncgs)
    if not spherical:
        return c2s
    p2c = p2c_map(b, ghost_value=0)
    s3 = math.sqrt(3.0)
    for i in range(b.npgs):
        pw = (b.pax[i], b.pay[i], b.paz[i])
        if pw == (2, 0, 0):
            c2s[p2c[i], p2c[i]] = 0.0
        elif pw == (0, 2, 0):
            c2s[p2c[i], p2c[i]] = -s3 / 2.0
            c2s[p2c[i], p2c[i - 1]] = s3 / 2.0
        elif pw == (0, 0, 2):
            c2s[p2c[i], p2c[i - 2]] = -0.5
            c2s[p2c[i], p2c[i - 1]] = -0.5
    for i in range(b.npgs):
        pw = (b.pax[i], b.pay[i], b.paz[i])
        if pw == (3, 0, 0):
            c2s[p2c[i], p2c[i + 8]] = -3.0 * math.sqrt(5.0) / 10.0
            c2s[p2c[i], p2c[i + 4]] = -3.0 * math.sqrt(5.0) / 10.0
            c2s[p2c[i], p2c[i + 2]] = 1.0
            c2s[p2c[i], p2c[i]] = 0.0
        elif pw == (0, 3, 0):
            c2s[p2c[i], p2c[i - 1]] = -math.sqrt(6.0) / 4.0
            c2s[p2c[i], p2c[i + 5]] = -math.sqrt(30.0) / 20.0
            c2s[p2c[i], p2c[i + 4]] = math.sqrt(30.0) / 5.0
            c2s[p2c[i], p2c[i]] = 0.0
        elif pw == (0, 0, 3):
            c2s[p2c[i], p2c[i + 1]] = -math.sqrt(30.0) / 20.0
            c2s[p2c[i], p2c[i - 1]] = -math.sqrt(6.0) / 4.0
            c2s[p2c[i], p2c[i + 5]] = math.sqrt(30.0) / 5.0
            c2s[p2c[i], p2c[i]] = 0.0
        elif pw == (2, 1, 0):
            c2s[p2c[i], p2c[i + 5]] = s3 / 2.0
            c2s[p2c[i], p2c[i + 1]] = -s3 / 2.0
            c2s[p2c[i], p2c[i]] = 0.0
        elif pw == (0, 2, 1):
            c2s[p2c[i], p2c[i + 5]] = 1.0
            c2s[p2c[i], p2c[i]] = 0.0
        elif pw == (1, 0, 2):
            c2s[p2c[i], p2c[i - 5]] = math.sqrt(10.0) / 4.0
            c2s[p2c[i], p2c[i + 1]] = -3.0 / 4.0 * math.sqrt(2.0)
            c2s[p2c[i], p2c[i]] = 0.0
        elif pw == (1, 2, 0):
            c2s[p2c[i], p2c[i - 3]] = 3.0 / 4.0 * math.sqrt(2.0)
            c2s[p2c[i], p2c[i - 5]] = -math.sqrt(10.0) / 4.0
            c2s[p2c[i], p2c[i]] = 0.0
        elif pw in ((0, 1, 2), (2, 0, 1), (1, 1, 1)):
            c2s[p2c[i], p2c[i]] = 0.0
    return c2s


def form_c2h(b: Basis, helix: float, ncell: int):
    """Helical rotation of contracted (C2H) and primitive (P2H) components.

    Returns arrays indexed [q + ncell] for q in -ncell..ncell, each (n, n),
    following src/pbasis.f90:152-413 (p and d; f follows the same table).
    With HELIX == 0 both are identities.
    """
    nq = 2 * ncell + 1
    c2h = np.zeros((nq, b.ncgs, b.ncgs))
    p2h = np.zeros((nq, b.npgs, b.npgs))
    for k in range(nq):
        c2h[k] = np.eye(b.ncgs)
        p2h[k] = np.eye(b.npgs)
    if helix == 0.0:
        return c2h, p2h
    p2c = p2c_map(b, ghost_value=-1)
    s3 = math.sqrt(3.0)
    for k in range(nq):
        j = k - ncell
        ang = helix * j
        c, s = math.cos(ang), math.sin(ang)
        C, P = c2h[k], p2h[k]
        for i in range(b.npgs):
            pw = (b.pax[i], b.pay[i], b.paz[i])
            if pw == (1, 0, 0) and p2c[i] != -1:
                pc = p2c
                C[pc[i], pc[i]] = 1.0
                C[pc[i + 1], pc[i + 1]] = c; C[pc[i + 2], pc[i + 2]] = c
                C[pc[i + 1], pc[i + 2]] = s; C[pc[i + 2], pc[i + 1]] = -s
                P[i, i] = 1.0
                P[i + 1, i + 1] = c; P[i + 2, i + 2] = c
                P[i + 1, i + 2] = s; P[i + 2, i + 1] = -s
        for i in range(b.npgs):
            pw = (b.pax[i], b.pay[i], b.paz[i])
            if pw == (2, 0, 0) and p2c[i] != -1:
                pc = p2c
                C[pc[i], pc[i]] = 1.0
                C[pc[i + 1], pc[i + 1]] = c * c
                C[pc[i + 1], pc[i + 2]] = s * s
                C[pc[i + 1], pc[i + 4]] = 2.0 * c * s / s3
                C[pc[i + 2], pc[i + 1]] = s * s
                C[pc[i + 2], pc[i + 2]] = c * c
                C[pc[i + 2], pc[i + 4]] = -2.0 * c * s / s3
                C[pc[i + 3], pc[i + 3]] = c
                C[pc[i + 3], pc[i + 5]] = s
                C[pc[i + 4], pc[i + 1]] = -c * s * s3
                C[pc[i + 4], pc[i + 2]] = c * s * s3
                C[pc[i + 4], pc[i + 4]] = c * c - s * s
                C[pc[i + 5], pc[i + 3]] = -s
                C[pc[i + 5], pc[i + 5]] = c
                P[i, i] = 1.0
                P[i + 1, i + 1] = c * c
                P[i + 1, i + 2] = s * s
                P[i + 1, i + 4] = 2.0 * c * s
                P[i + 2, i + 1] = s * s
                P[i + 2, i + 2] = c * c
                P[i + 2, i + 4] = -2.0 * c * s
                P[i + 3, i + 3] = c
                P[i + 3, i + 5] = s
                P[i + 4, i + 1] = -c * s
                P[i + 4, i + 2] = c * s
                P[i + 4, i + 4] = c * c - s * s
                P[i + 5, i + 3] = -s
                P[i + 5, i + 5] = c
        for i in range(b.npgs):
            pw = (b.pax[i], b.pay[i], b.paz[i])
            if pw == (3, 0, 0) and p2c[i] != -1:
                raise NotImplementedError('helical rotation of f functions is not needed by the workloads')
    return c2h, p2h


def census(b: Basis) -> dict:
    """Counts matching the reference's printout (src/pread.f90:1450-1452)."""
    hist = {}
    for L in b.p_shell_ang:
        hist[int(L)] = hist.get(int(L), 0) + 1
    return {'npgs': b.npgs, 'ncgs': b.ncgs, 'npshell': b.npshell,
            'npgs_real': b.nreal_pgs, 'ncgs_real': b.nreal_cgs, 'shell_ang': hist}
