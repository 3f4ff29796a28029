"""Seeded synthetic geometries of the benchmark workloads.

* all-trans linear alkanes C_nH_{2n+2} with standard bond lengths (C-C 1.53 A,
  C-H 1.09 A, tetrahedral angles) plus Gaussian jitter;
* water clusters (H2O)_k built from the reference's sample water geometry
  (O-H 0.967 A, data/H2O_CCSD_ccpVDZ) with random orientations and O-O
  nearest distances uniform in 2.7-3.2 A, rejection-sampled against < 2.6 A;
* a helical polyethylene cell (C2H4, screw axis z).

Everything is returned in bohr, ready for :func:`polymer_b200.inputdeck.make_deck`.
"""
from __future__ import annotations

import math
from typing import List, Tuple

import numpy as np

from .inputdeck import ANG_BOHR, Deck, make_deck

TET = math.acos(-1.0 / 3.0)  # 109.4712 deg


def alkane(n: int, jitter: float = 0.02, seed: int = None) -> Tuple[List[int], np.ndarray]:
    """All-trans C_nH_{2n+2}: zig-zag carbon backbone in the xz plane (angstrom in, bohr out)."""
    rng = np.random.default_rng(1000 + n if seed is None else seed)
    cc, ch = 1.53, 1.09
    half = TET / 2.0
    dx = cc * math.sin(half)   # advance along x per C-C bond
    dz = cc * math.cos(half)   # zig-zag amplitude
    carbons = [np.array([i * dx, 0.0, (i % 2) * dz]) for i in range(n)]
    atoms, xyz = [], []
    for c in carbons:
        atoms.append(6)
        xyz.append(c)
    if n == 1:
        for v in ((1, 1, 1), (-1, -1, 1), (-1, 1, -1), (1, -1, -1)):
            atoms.append(1)
            xyz.append(carbons[0] + ch * np.array(v, dtype=float) / math.sqrt(3.0))
    else:
        for i, c in enumerate(carbons):
            # the two backbone neighbours sit on the other side of the zig-zag, so the
            # CH2 hydrogens point away from them: -z on even carbons, +z on odd ones
            out = np.array([0.0, 0.0, 1.0 if i % 2 else -1.0])
            hs = []
            for sgn in (1.0, -1.0):
                v = out * math.cos(half) + np.array([0.0, sgn, 0.0]) * math.sin(half)
                hs.append(v / np.linalg.norm(v))
            if i in (0, n - 1):
                # terminal carbon: the C-C bond, the two hydrogens above and a third
                # hydrogen complete a tetrahedron (four unit vectors summing to zero)
                nb = carbons[1] if i == 0 else carbons[n - 2]
                u = (nb - c) / np.linalg.norm(nb - c)
                w = -(u + hs[0] + hs[1])
                hs.append(w / np.linalg.norm(w))
            for v in hs:
                atoms.append(1)
                xyz.append(c + ch * v)
    xyz = np.array(xyz)
    xyz = xyz + rng.normal(0.0, jitter, size=xyz.shape)
    return atoms, xyz / ANG_BOHR


def alkane_deck(n: int, basis: str = '6-31Gss', jitter: float = 0.02, **opts) -> Deck:
    atoms, xyz = alkane(n, jitter)
    opts.setdefault('inttol', 1.0e-10)
    return make_deck(atoms, xyz, basis, **opts)


# water monomer of the reference's sample input (bohr), O at the origin
_WATER = np.array([[0.0, 0.0, 0.0],
                   [0.0, 1.079252144093028, 1.474611055780858],
                   [0.0, 1.079252144093028, -1.474611055780858]])


def _random_rotation(rng) -> np.ndarray:
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    a, b, c, d = q
    return np.array([[a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)],
                     [2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)],
                     [2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d]])


def water_cluster(k: int, seed: int) -> Tuple[List[int], np.ndarray]:
    rng = np.random.default_rng(seed)
    oxygens: List[np.ndarray] = []
    atoms, xyz = [], []
    lo, hi, rej = 2.7 / ANG_BOHR, 3.2 / ANG_BOHR, 2.6 / ANG_BOHR
    for i in range(k):
        for _ in range(10000):
            if not oxygens:
                o = np.zeros(3)
            else:
                base = oxygens[rng.integers(len(oxygens))]
                d = rng.normal(size=3)
                d /= np.linalg.norm(d)
                o = base + rng.uniform(lo, hi) * d
                if min(np.linalg.norm(o - p) for p in oxygens) < rej:
                    continue
            break
        else:
            raise RuntimeError('water cluster placement failed')
        oxygens.append(o)
        r = _random_rotation(rng)
        for z, p in zip((8, 1, 1), _WATER):
            atoms.append(z)
            xyz.append(o + r @ p)
    return atoms, np.array(xyz)


def water_single_point_deck(**opts) -> Deck:
    """The water single point: O (0, 0, 0.1173) A, H (0, +-0.7572, -0.4692) A,
    cc-pVDZ with spherical d, a molecule (no lattice), INTTOL 1e-12, SCFCONV 1e-8."""
    xyz = np.array([[0.0, 0.0, 0.1173], [0.0, 0.7572, -0.4692], [0.0, -0.7572, -0.4692]])
    opts.setdefault('inttol', 1.0e-12)
    opts.setdefault('scfconv', 1.0e-8)
    opts.setdefault('spherical', True)
    return make_deck([8, 1, 1], xyz / ANG_BOHR, 'cc-pVDZ', **opts)


def water_deck(k: int, seed: int, basis: str = 'cc-pVDZ', **opts) -> Deck:
    atoms, xyz = water_cluster(k, seed)
    opts.setdefault('inttol', 1.0e-10)
    return make_deck(atoms, xyz, basis, **opts)


def polyethylene_deck(basis: str = '6-31G', cutoff1: int = 5, cutoff2: int = 10, kpoints: int = 16,
                      jitter: float = 0.01, seed: int = 3000, **opts) -> Deck:
    """Helical polyethylene-like chain: C2H4 cell, period 2.55 A along z, 180 deg screw.

    A 180-degree screw with a two-carbon cell cannot generate the planar
    all-trans zig-zag (the rotation flips the lateral offset every cell), so
    the cell is the closest valid screw-symmetric chain: carbons at lateral
    offsets (a,0) and (0,a) a half period apart, a chosen so that every C-C
    bond is 1.54 A (the carbons then spiral four per turn, C-C-C ~133 deg);
    each carbon carries two hydrogens at 1.09 A, radially outward and tilted
    +/- along the chain.  Seeded jitter of 0.01 A per coordinate.  The input
    axis is z; the reference's CHECK_GEOMETRY re-orients a z-helix along x.
    """
    rng = np.random.default_rng(seed)
    period = 2.55
    half = period / 2.0
    a = math.sqrt(0.5 * (1.54 ** 2 - half ** 2))
    carbons = [np.array([a, 0.0, 0.0]), np.array([0.0, a, half])]
    atoms, xyz = [6, 6], list(carbons)
    for c in carbons:
        u = np.array([c[0], c[1], 0.0]) / a
        for sgn in (1.0, -1.0):
            v = math.cos(TET / 2) * u + sgn * math.sin(TET / 2) * np.array([0.0, 0.0, 1.0])
            atoms.append(1)
            xyz.append(c + 1.09 * v)
    xyz = np.array(xyz) + rng.normal(0.0, jitter, size=(len(xyz), 3))
    opts.setdefault('inttol', 1.0e-10)
    return make_deck(atoms, xyz / ANG_BOHR, basis, period=(0.0, 0.0, period / ANG_BOHR), helix_deg=180.0,
                     kpoints=(0, 0, kpoints), cutoff1=cutoff1, cutoff2=cutoff2, **opts)


def water_batch_decks(n: int = 256, seed: int = 2000, kmax: int = 16, basis: str = 'cc-pVDZ',
                      **opts) -> List[Deck]:
    """The batch workload of uneven water clusters: sizes k ~ U{1..kmax} drawn
    from default_rng(seed), cluster i generated from default_rng(seed + 1 + i)."""
    ks = np.random.default_rng(seed).integers(1, kmax + 1, size=n)
    return [water_deck(int(k), seed=seed + 1 + i, basis=basis, **opts) for i, k in enumerate(ks)]
