"""Keyword input deck: the caller-side configuration the Fock build consumes.

Mirrors the reference's READ1 (src/pread.f90:1-502): a keyword-per-line text
file, a GEOMETRY block terminated by a line whose first token is not an element
symbol (conventionally ``X``), unit conversion (src/pread.f90:296-308) and the
HF theory preset (src/pread.f90:318-325).  CHECK_GEOMETRY's helical
re-orientation (src/pread.f90:1809-1871) and SINGLEPOINT's cutoff assignment
(src/psinglepoint.f90:29-64) are applied by :func:`finalize`.

Only what the SCF / Fock-build path reads is interpreted; every other keyword
of the reference's 112-entry table is accepted and its value line skipped, so
the reference's own sample inputs parse unchanged.
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional

# Constants exactly as the reference defines them (src/pmodules.f90:7-12).
PI = 3.14159265358979
ANG_BOHR = 0.529177249
BOLTZMANN = 1.0 / 3.1577464e5

ELEMENTS = ['H', 'He', 'Li', 'Be', 'B', 'C', 'N', 'O', 'F', 'Ne', 'Na', 'Mg', 'Al',
            'Si', 'P', 'S', 'Cl', 'Ar', 'K', 'Ca', 'Sc', 'Ti', 'V', 'Cr', 'Mn', 'Fe',
            'Co', 'Ni', 'Cu', 'Zn', 'Ga', 'Ge', 'As', 'Se', 'Br', 'Kr']

# Keyword table (src/pread.f90:15-47): name -> value kind.
# 'i' integer, 'd' double, 's' string, 'l' logical.
_KW = {
    'JOBNAME': 's', 'BASISSET': 's', 'CHARGE': 'i', 'JOBTYPE': 'i', 'UNITS': 's',
    'PRINT': 'i', 'CUTOFF1': 'i', 'CUTOFF2': 'i', 'INTTOL': 'd', 'SCFCYCLES': 'i',
    'SCFCONV': 'd', 'SCFRELAX': 'd', 'DIIS': 'i', 'AUXILIARY': 's', 'MULTIPOLE': 'i',
    'HFEXCHANGE': 'd', 'SLATER': 'd', 'VWN': 'd', 'BECKE88': 'd', 'LYP': 'd', 'MP2': 'd',
    'DIRECT': 'l', 'MAXDISK': 'd', 'FROZENCORE': 'i', 'MAXMEMORY': 'd', 'CUTOFF3': 'i',
    'VAPPROX': 'l', 'SAPPROX': 'l', 'DYSON': 'l', 'RI_SCF': 'l', 'RI_MP2': 'l',
    'THEORY': 's', 'CIS_ROOTS': 'i', 'RPA_ROOTS': 'i', 'DAVIDSON': 'd', 'SINGLET': 'l',
    'TRIPLET': 'l', 'OPTCONV': 'd', 'GDIIS': 'i', 'CISQP': 'l', 'QPBANDS': 'i',
    'DYSONDAMP': 'd', 'OEP': 'l', 'MP2KJOBS': 'i', 'MP2KJOBE': 'i', 'HIGHMP': 'i',
    'HIGHCIS': 'i', 'HIGHCIE': 'i', 'HIGHCCS': 'i', 'HIGHCCE': 'i', 'CCDIIS': 'i',
    'FROZENVIRT': 'i', 'HIGHCIROOT': 'i', 'EOMORDERS': 'i', 'EOMORDERE': 'i',
    'EOMROOT': 'i', 'IP': 'l', 'EA': 'l', 'CCCONV': 'd', 'CCRELAX': 'd', 'CCALG': 'i',
    'XCC': 'l', 'CCPTROOT': 'i', 'CICONV': 'd', 'CCPTCONV': 'd', 'SPHERICAL': 'l',
    'CCTHEORY': 's', 'OEPALG': 'i', 'SLATER51': 'l', 'KLI': 'l', 'POTDUMP': 'i',
    'DENDUMP': 'i', 'KERNEL_HF': 'd', 'KERNEL_S': 'd', 'KERNEL_VWN': 'd',
    'KERNEL_B88': 'd', 'KERNEL_LYP': 'd', 'RADIAL': 'i', 'ANGULAR': 'i', 'AC': 'l',
    'KERNEL_OEP': 'd', 'LINDEP': 'd', 'POLAR': 'l', 'OMEGA': 'd', 'POLARALG': 'i',
    'POLARX': 'l', 'POLARY': 'l', 'POLARZ': 'l', 'SOS': 'l', 'RELATIVITY': 'l',
    'SINANOGLU': 'l', 'SALG': 'i', 'SINGULAR': 'd', 'HIGHGF': 'i', 'TEMP': 'd',
    'MODULO': 'i', 'NGRID': 'i', 'DELTAH': 'd', 'GEMINAL': 's', 'LMAX': 'i',
    'MBGFALG': 'i', 'MP2ALG': 'i', 'DIAGONAL': 'l', 'DYSONCONV': 'd', 'TEMPHF': 'd',
    'DEGENERATE': 'l', 'TCE': 's', 'CCGUESS': 'l', 'LIPALDUS': 'l',
}


class InputError(ValueError):
    """Raised where the reference would PABORT while reading its input."""


@dataclasses.dataclass
class Deck:
    """Everything the SCF / Fock-build path reads from the input deck (bohr, radians)."""
    atoms: List[int]                 # atomic numbers (IATOM)
    coords: List[List[float]]        # ATOMX/ATOMY/ATOMZ
    period: List[float]              # PERIODX/Y/Z
    helix: float = 0.0               # HELIX (radians)
    kpoints: List[int] = dataclasses.field(default_factory=lambda: [0, 0, 0])
    basisset: str = ''
    jobname: str = 'NONE'
    charge: int = 0
    print_level: int = 0
    cutoff1: int = 0
    cutoff2: int = 0
    cutoff3: int = 0
    inttol: float = 1.0e-10          # DOPTN(12)
    scfcycles: int = 50              # IOPTN(13)
    scfconv: float = 1.0e-8          # DOPTN(14)
    scfrelax: float = 1.0            # DOPTN(15)
    diis: int = 5                    # IOPTN(16)
    hfexchange: float = 1.0          # DOPTN(19)
    direct: bool = True              # LOPTN(25)
    spherical: bool = False          # LOPTN(69)
    lindep: float = 1.0e-6           # DOPTN(85)
    temphf: float = 0.0              # DOPTN(108)
    theory: str = 'SPECIFIED BELOW'
    dft: bool = False                # a DFT preset was requested (XC is not built)
    # derived by finalize()
    cel1: List[int] = dataclasses.field(default_factory=lambda: [0, 0, 0])
    cel2: List[int] = dataclasses.field(default_factory=lambda: [0, 0, 0])
    periodic: List[bool] = dataclasses.field(default_factory=lambda: [False, False, False])

    @property
    def natom(self) -> int:
        return len(self.atoms)

    @property
    def nelectrons(self) -> int:
        return sum(self.atoms) - self.charge


def _value(kind: str, tok: str):
    if kind == 'i':
        return int(tok)
    if kind == 'd':
        return float(tok.replace('D', 'E').replace('d', 'e'))
    if kind == 'l':
        t = tok.strip().upper()
        if t.startswith('.T') or t == 'T':
            return True
        if t.startswith('.F') or t == 'F':
            return False
        raise InputError('bad logical %r' % tok)
    return tok.strip()


def parse(text: str) -> Deck:
    """Parse an input deck in the reference's format (src/pread.f90:178-265)."""
    lines = text.splitlines()
    raw = {}
    atoms: List[int] = []
    coords: List[List[float]] = []
    period = [0.0, 0.0, 0.0]
    helix = 0.0
    kpts = [0, 0, 0]
    seen_geometry = False
    i = 0
    while i < len(lines):
        toks = lines[i].split()
        i += 1
        if not toks:
            continue
        key = toks[0]
        if key.startswith('!'):
            continue
        key = key[:10].upper()
        if key == 'GEOMETRY':
            seen_geometry = True
            atoms, coords = [], []
            while i < len(lines):
                t = lines[i].split()
                i += 1
                sym = t[0][:2] if t else ''
                if sym not in ELEMENTS:
                    break
                atoms.append(ELEMENTS.index(sym) + 1)
                coords.append([float(x.replace('D', 'E')) for x in t[1:4]])
            continue
        if key in ('PERIOD', 'KPOINTS', 'HELIX'):
            vals = lines[i].split()
            i += 1
            if key == 'PERIOD':
                period = [float(v.replace('D', 'E')) for v in vals[:3]]
            elif key == 'KPOINTS':
                kpts = [int(v) for v in vals[:3]]
            else:
                helix = float(vals[0].replace('D', 'E'))
            continue
        if key not in _KW:
            raise InputError('A SYNTAX ERROR : %s ?' % key)
        raw[key] = _value(_KW[key], lines[i].split()[0] if _KW[key] != 's' else lines[i])
        i += 1
    if not seen_geometry or not atoms:
        raise InputError('GEOMETRY NOT FOUND IN INPUT STREAM')
    for required in ('BASISSET', 'CUTOFF1', 'CUTOFF2'):
        if required not in raw:
            raise InputError('%s NOT FOUND IN INPUT STREAM' % required)
    d = Deck(atoms=atoms, coords=coords, period=period, helix=helix, kpoints=kpts)
    d.basisset = raw['BASISSET'].split()[0]
    d.jobname = raw.get('JOBNAME', 'NONE').split()[0] if raw.get('JOBNAME') else 'NONE'
    d.charge = raw.get('CHARGE', 0)
    d.print_level = raw.get('PRINT', 0)
    d.cutoff1 = raw['CUTOFF1']
    d.cutoff2 = raw['CUTOFF2']
    d.cutoff3 = raw.get('CUTOFF3', 0)
    d.inttol = raw.get('INTTOL', d.inttol)
    d.scfcycles = raw.get('SCFCYCLES', d.scfcycles)
    d.scfconv = raw.get('SCFCONV', d.scfconv)
    d.scfrelax = raw.get('SCFRELAX', d.scfrelax)
    d.diis = raw.get('DIIS', d.diis)
    d.hfexchange = raw.get('HFEXCHANGE', d.hfexchange)
    d.direct = raw.get('DIRECT', d.direct)
    d.spherical = raw.get('SPHERICAL', d.spherical)
    d.lindep = raw.get('LINDEP', d.lindep)
    d.temphf = raw.get('TEMPHF', d.temphf)
    d.theory = raw.get('THEORY', d.theory).split()[0] if raw.get('THEORY') else d.theory
    units = raw.get('UNITS', 'BOHR').split()[0].upper()
    if units == 'ANGSTROM':
        d.coords = [[c / ANG_BOHR for c in xyz] for xyz in d.coords]
        d.period = [p / ANG_BOHR for p in d.period]
    elif units != 'BOHR':
        raise InputError('UNIT OF LENGTH MUST BE BOHR OR ANGSTROM')
    d.helix = d.helix * PI / 180.0
    # THEORY presets (src/pread.f90:309-374): HF forces HFEXCHANGE=1; the DFT
    # presets need exchange-correlation code that this package does not have; any
    # other name (e.g. MP2FC, a post-SCF method) sets no preset.
    if d.theory == 'HF':
        d.hfexchange = 1.0
    elif d.theory in ('SNULL', 'BNULL', 'SVWN', 'BLYP', 'SLYP', 'BVWN', 'B3LYP'):
        d.dft = True
    return finalize(d)


def finalize(d: Deck) -> Deck:
    """Cutoffs per periodic axis and helical re-orientation along x.

    src/psinglepoint.f90:29-64 (CEL1/CEL2 per axis, KVC zeroed on
    non-periodic axes) and src/pread.f90:1809-1871 (a y- or z-helix is
    rotated so that its axis is x).
    """
    lx, ly, lz = (p != 0.0 for p in d.period)
    if d.helix != 0.0 and sum((lx, ly, lz)) > 1:
        raise InputError('HELICAL SYMMETRY FOR 1D CRYSTAL ONLY')
    cel1 = [d.cutoff1 if l else 0 for l in (lx, ly, lz)]
    cel2 = [d.cutoff2 if l else 0 for l in (lx, ly, lz)]
    kv = [k if l else 0 for k, l in zip(d.kpoints, (lx, ly, lz))]
    if d.cutoff1 < 0 or d.cutoff2 < 0:
        raise InputError('INVALID CUTOFF PARAMETERS')
    if ly and not lx and not lz and d.helix != 0.0:
        d.coords = [[y, z, x] for x, y, z in d.coords]
        d.period = [d.period[1], d.period[2], d.period[0]]
        kv = [kv[1], kv[2], kv[0]]
        cel1 = [cel1[1], cel1[2], cel1[0]]
        cel2 = [cel2[1], cel2[2], cel2[0]]
        lx, ly, lz = True, False, False
    elif lz and not lx and not ly and d.helix != 0.0:
        d.coords = [[z, x, y] for x, y, z in d.coords]
        d.period = [d.period[2], d.period[0], d.period[1]]
        kv = [kv[2], kv[0], kv[1]]
        cel1 = [cel1[2], cel1[0], cel1[1]]
        cel2 = [cel2[2], cel2[0], cel2[1]]
        lx, ly, lz = True, False, False
    d.cel1, d.cel2, d.kpoints = cel1, cel2, kv
    d.periodic = [lx, ly, lz]
    _check_geometry(d)
    return d


def screw(d: Deck, xyz, kx: int, ky: int = 0, kz: int = 0):
    """Image of a point in cell (kx,ky,kz): rotate by kx*HELIX about x, then translate."""
    c, s = math.cos(kx * d.helix), math.sin(kx * d.helix)
    x, y, z = xyz
    return [x + kx * d.period[0], y * c - z * s + ky * d.period[1], y * s + z * c + kz * d.period[2]]


def _check_geometry(d: Deck) -> None:
    """Zero internuclear separation aborts (src/pread.f90:1873-1903)."""
    n = d.natom
    for i in range(n):
        for j in range(n):
            for kx in range(-d.cel2[0], d.cel2[0] + 1):
                for ky in range(-d.cel2[1], d.cel2[1] + 1):
                    for kz in range(-d.cel2[2], d.cel2[2] + 1):
                        if kx == ky == kz == 0 and i == j:
                            continue
                        p = screw(d, d.coords[j], kx, ky, kz)
                        r2 = sum((a - b) ** 2 for a, b in zip(p, d.coords[i]))
                        if r2 == 0.0:
                            raise InputError('ZERO INTERNUCLEAR SEPARATION')


def nuclear_repulsion(d: Deck) -> float:
    """Nuclear repulsion per unit cell, src/pselfconsistentfield.f90:652-704."""
    e = 0.0
    for i in range(d.natom):
        x0 = d.coords[i]
        for j in range(d.natom):
            for kx in range(-d.cel2[0], d.cel2[0] + 1):
                for ky in range(-d.cel2[1], d.cel2[1] + 1):
                    for kz in range(-d.cel2[2], d.cel2[2] + 1):
                        if kx * kx + ky * ky + kz * kz == 0 and i == j:
                            continue
                        p = screw(d, d.coords[j], kx, ky, kz)
                        r = math.sqrt(sum((a - b) ** 2 for a, b in zip(p, x0)))
                        e += 0.5 * d.atoms[i] * d.atoms[j] / r
    return e


def make_deck(atoms, coords_bohr, basisset, *, period=(0.0, 0.0, 0.0), helix_deg=0.0,
              kpoints=(0, 0, 0), cutoff1=0, cutoff2=0, **opts) -> Deck:
    """Build a deck programmatically (coordinates already in bohr)."""
    d = Deck(atoms=list(atoms), coords=[list(map(float, c)) for c in coords_bohr],
             period=list(map(float, period)), helix=helix_deg * PI / 180.0,
             kpoints=list(kpoints))
    d.basisset = basisset
    d.cutoff1, d.cutoff2 = cutoff1, cutoff2
    for k, v in opts.items():
        if not hasattr(d, k):
            raise InputError('unknown option %s' % k)
        setattr(d, k, v)
    return finalize(d)


def deck_text(geometry, keywords) -> str:
    """Re-assemble an input deck from (symbol, x, y, z) rows and keyword -> value-line pairs."""
    out = ['GEOMETRY']
    for sym, x, y, z in geometry:
        out.append('%s %.15f %.15f %.15f' % (sym, x, y, z))
    out.append('X 0.0 0.0 0.0')
    for k, v in keywords.items():
        out.append(k)
        out.append(v)
    return '\n'.join(out) + '\n'
