"""The parallel oracle used by the full-size parity tests (tests/oracle_pool.py)
sums its pieces to the single-call oracle: bra-shell residue classes for a
molecule, cell-pair tickets for a helical chain."""
import numpy as np
import torch

import oracle
import oracle_pool
from polymer_b200 import geometry, scf, system


def test_molecule_pieces_sum_to_the_whole_build():
    s = system.build_system(geometry.alkane_deck(2), oracle.onee)
    rng = np.random.default_rng(2)
    n = s.basis.ncgs
    a = rng.normal(size=(n, n))
    pp = np.einsum('ai,cab,bj->cij', s.basis.cc, (a + a.T)[None], s.basis.cc, optimize=True)
    c1, x1 = oracle.fourindex_eri(s, pp)
    c2, x2 = oracle_pool.fourindex_eri(s, pp, nproc=2)
    assert np.abs(c1 - c2).max() <= 1e-12 * np.abs(c1).max()
    assert np.abs(x1 - x2).max() <= 1e-12 * np.abs(x1).max()


def test_lattice_tickets_sum_to_the_whole_build():
    s = system.build_system(geometry.polyethylene_deck('STO-3G', cutoff1=1, cutoff2=2, kpoints=4), oracle.onee)
    rng = np.random.default_rng(3)
    n = s.basis.ncgs
    pc = rng.normal(size=(s.ncell1, n, n)) * 0.1
    for c, q in enumerate(s.cells):
        cm = s.cell_index(-q[0], -q[1], -q[2])
        if cm == c:
            pc[c] = 0.5 * (pc[c] + pc[c].T)
        elif cm < c:
            pc[c] = pc[cm].T
    pp = np.einsum('ai,cab,bj->cij', s.basis.cc, pc, s.basis.cc, optimize=True)
    ph = scf.rotate(scf.HostState(s), torch.tensor(pp)).numpy()
    c1, x1 = oracle.fourindex_eri(s, pp, ph)
    c2, x2 = oracle_pool.fourindex_eri(s, pp, ph, nproc=2)
    assert np.abs(c1 - c2).max() <= 1e-12 * np.abs(c1).max()
    assert np.abs(x1 - x2).max() <= 1e-12 * np.abs(x1).max()


def test_fullsize_fixtures_describe_the_test_systems():
    """The projected oracle fixtures of the full-size parity tests belong to the
    systems and seeded densities the GPU test builds (sizes and seeds)."""
    import os
    from conftest import GOLDEN
    from golden import make_fullsize
    for name, make in make_fullsize.cases().items():
        g = np.load(os.path.join(GOLDEN, 'fullsize_%s.npz' % name))
        s, seed = make()
        assert int(g['npgs']) == s.basis.npgs and int(g['ncgs']) == s.basis.ncgs and int(g['seed']) == seed
        assert g['cr'].shape == (s.basis.ncgs, 4) and g['xr'].shape == (s.basis.ncgs, 4)
        assert float(g['cmax']) > 0.0 and float(g['xmax']) > 0.0
