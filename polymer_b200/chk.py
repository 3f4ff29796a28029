"""The reference's JOBNAME.chk checkpoint file (formatted text, unit 30).

Written by STORE_DENSITYMATRIX (src/pdensitymatrix.f90:131-208) once per SCF
iteration and read by RESTORE_DENSITYMATRIX (:1-79, called from SINGLEPOINT at
src/psinglepoint.f90:194) and DIIS (:253-339).  A file is a sequence of blocks,
one per iteration:

* a header record ``NCGS CEL1X CEL1Y CEL1Z`` (list-directed integers);
* for QX = -CEL1X..CEL1X, QY = -CEL1Y..CEL1Y, QZ = -CEL1Z..CEL1Z (QX outermost),
  I = 1..NCGS, J = 1..NCGS (J fastest): one record ``P_C(J,I,Q)
  P_C_OUT(J,I,Q) - P_C(J,I,Q)`` -- the iteration's input density and its change.

STORE rewinds, reads the first ISCF-1 blocks (for the Pulay products) and writes
block ISCF after them, so the file holds exactly ISCF blocks.  RESTORE reads
block after block until the end of the file, so the last block's P_C wins; a
header whose NCGS differs from the basis stops it ("incompatible format": the
nuclear-charge guess is used); cells outside the current CEL1 range are
skipped, and P_C is zeroed once, so cells a block lacks keep what an earlier
block gave them.  This module writes what STORE writes (17
significant digits, so doubles survive the round trip) and reads any
list-directed form of it (``E`` or ``D`` exponents, comma or blank separators,
``r*c`` repeat counts).

Densities here are cell-major ``(ncell1, ncgs, ncgs)`` arrays indexed ``[cell,
row, column]`` with cells in ``System.cell_index`` order.
"""
from __future__ import annotations

import os
import re
from typing import Iterator, List, Optional, Sequence, Tuple

import numpy as np

_REPEAT = re.compile(r'^(\d+)\*(.*)$')


def _cells_fortran(cel1: Sequence[int]) -> List[Tuple[int, int, int]]:
    """(QX, QY, QZ) in the chk loop order: QX outermost, QZ innermost."""
    return [(qx, qy, qz) for qx in range(-cel1[0], cel1[0] + 1)
            for qy in range(-cel1[1], cel1[1] + 1) for qz in range(-cel1[2], cel1[2] + 1)]


def _cell_index(cel1: Sequence[int], qx: int, qy: int, qz: int) -> int:
    n1x, n1y = 2 * cel1[0] + 1, 2 * cel1[1] + 1
    return (qx + cel1[0]) + n1x * ((qy + cel1[1]) + n1y * (qz + cel1[2]))


def _tokens(text: str) -> Iterator[str]:
    for tok in text.replace(',', ' ').replace('D', 'E').replace('d', 'e').split():
        m = _REPEAT.match(tok)
        if m:
            for _ in range(int(m.group(1))):
                yield m.group(2)
        else:
            yield tok


def format_block(p_c: np.ndarray, d_p: np.ndarray, cel1: Sequence[int]) -> str:
    """One block: the header and every (P_C, P_C_OUT - P_C) record."""
    n = p_c.shape[-1]
    out = ['%12d%12d%12d%12d\n' % (n, cel1[0], cel1[1], cel1[2])]
    for qx, qy, qz in _cells_fortran(cel1):
        c = _cell_index(cel1, qx, qy, qz)
        a = np.asarray(p_c[c]).flatten(order='F')    # element (J, I), J fastest
        b = np.asarray(d_p[c]).flatten(order='F')
        out.append(''.join('%25.17E%25.17E\n' % (x, y) for x, y in zip(a.tolist(), b.tolist())))
    return ''.join(out)


def store(path: str, iscf: int, p_c: np.ndarray, p_c_out: np.ndarray, cel1: Sequence[int],
          pulay: bool = True) -> Optional[np.ndarray]:
    """STORE_DENSITYMATRIX: write block `iscf` (1-based) after the first iscf-1
    blocks of `path`, dropping anything after them.  With `pulay` it returns
    PULAY(1..iscf, iscf) as the reference computes it from the file: the
    products of the earlier blocks' density changes with this one, and its own
    square; without, it appends to a file the caller knows holds iscf-1 blocks
    (an SCF that keeps the products in memory) and returns None."""
    p_c = np.asarray(p_c, dtype=np.float64)
    d_p = np.asarray(p_c_out, dtype=np.float64) - p_c
    block = format_block(p_c, d_p, cel1)
    if iscf <= 1:
        with open(path, 'w') as fh:
            fh.write(block)
        return np.array([float((d_p * d_p).sum())]) if pulay else None
    if not pulay:
        with open(path, 'a') as fh:
            fh.write(block)
        return None
    prev = read_blocks(path)
    if len(prev) < iscf - 1:
        raise ValueError('%s holds %d blocks, iteration %d needs %d' % (path, len(prev), iscf, iscf - 1))
    row = np.zeros(iscf)
    for i, (hdr, _, dpi) in enumerate(prev[:iscf - 1]):
        if tuple(hdr) != (p_c.shape[-1],) + tuple(cel1):
            raise ValueError('block %d of %s has another shape' % (i + 1, path))
        row[i] = float((dpi * d_p).sum())
    row[iscf - 1] = float((d_p * d_p).sum())
    if len(prev) == iscf - 1:
        with open(path, 'a') as fh:
            fh.write(block)
    else:
        text = ''.join(format_block(pc, dp, cel1) for _, pc, dp in prev[:iscf - 1]) + block
        with open(path, 'w') as fh:
            fh.write(text)
    return row


def read_blocks(path: str) -> List[Tuple[Tuple[int, int, int, int], np.ndarray, np.ndarray]]:
    """Every complete block of `path`: (header, P_C, P_C_OUT - P_C), the arrays
    cell-major over the block's own CEL1 range."""
    with open(path) as fh:
        toks = list(_tokens(fh.read()))
    blocks = []
    pos = 0
    while pos + 4 <= len(toks):
        try:
            hdr = tuple(int(t) for t in toks[pos:pos + 4])
        except ValueError:
            break
        n, cx, cy, cz = hdr
        cel = (cx, cy, cz)
        ncell = (2 * cx + 1) * (2 * cy + 1) * (2 * cz + 1)
        cnt = 2 * ncell * n * n
        if n <= 0 or min(cel) < 0 or pos + 4 + cnt > len(toks):
            break
        vals = np.array(toks[pos + 4:pos + 4 + cnt], dtype=np.float64).reshape(ncell, n * n, 2)
        pc = np.zeros((ncell, n, n))
        dp = np.zeros((ncell, n, n))
        for k, (qx, qy, qz) in enumerate(_cells_fortran(cel)):
            c = _cell_index(cel, qx, qy, qz)
            pc[c] = vals[k, :, 0].reshape(n, n, order='F')
            dp[c] = vals[k, :, 1].reshape(n, n, order='F')
        blocks.append((hdr, pc, dp))
        pos += 4 + cnt
    return blocks


def restore(path: str, ncgs: int, cel1: Sequence[int]) -> Tuple[Optional[np.ndarray], str]:
    """RESTORE_DENSITYMATRIX: (P_C, message) from the last block of `path`, or
    (None, message) when there is no block or a block's NCGS differs (the
    caller then takes the nuclear-charge guess)."""
    if not os.path.exists(path):
        return None, 'NO DENSITY MATRIX FOUND IN .chk FILE'
    blocks = read_blocks(path)
    ncell = (2 * cel1[0] + 1) * (2 * cel1[1] + 1) * (2 * cel1[2] + 1)
    p = np.zeros((ncell, ncgs, ncgs))     # zeroed once: a block leaves the cells it lacks as they were
    got = 0
    for hdr, pc, _ in blocks:
        if hdr[0] != ncgs:
            return None, 'DENSITY MATRIX IN INCOMPATIBLE FORMAT'
        bcel = hdr[1:]
        for qx, qy, qz in _cells_fortran(bcel):
            if abs(qx) <= cel1[0] and abs(qy) <= cel1[1] and abs(qz) <= cel1[2]:
                p[_cell_index(cel1, qx, qy, qz)] = pc[_cell_index(bcel, qx, qy, qz)]
        got += 1
    if got == 0:
        return None, 'NO DENSITY MATRIX FOUND IN .chk FILE'
    return p, '****** DENSITY MATRIX RESTORED FROM .chk FILE ******'


def write_guess(path: str, p_c: np.ndarray, cel1: Sequence[int]) -> None:
    """A one-block file holding `p_c` (change zero): RESTORE_DENSITYMATRIX then
    starts the reference's SCF from it -- how a core, SAD or learned guess made
    here reaches the Fortran driver."""
    store(path, 1, p_c, p_c, cel1, pulay=False)
