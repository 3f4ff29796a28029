"""READ3 emulation census (polymer_b200/basis.py) on the workloads' systems:
primitive and contracted counts with ghosts, shell counts and the shell
angular-momentum histogram, against the reference's READ3 arithmetic (the
water figures are also printed by the reference's own run,
data/H2O_CCSD_ccpVDZ_out: 67 and 36 including ghosts)."""
import numpy as np
import pytest

from polymer_b200 import basis, geometry

CENSUS = [
    ('water_ccpvdz', lambda: geometry.water_deck(1, seed=1), (67, 36, 37), (29, 7, 1)),
    ('c10h22_631gss', lambda: geometry.alkane_deck(10), (496, 322, 220), (148, 62, 10)),
    ('c20h42_631gss', lambda: geometry.alkane_deck(20), (976, 632, 430), (288, 122, 20)),
    ('c40h82_631gss', lambda: geometry.alkane_deck(40), (1936, 1252, 850), None),
    ('water5_ccpvdz', lambda: geometry.water_deck(5, seed=2), (5 * 67, 5 * 36, 5 * 37), None),
    ('pe_cell_631g', lambda: geometry.polyethylene_deck('6-31G'), (60, 26, 36), None),
]


@pytest.mark.parametrize('name,deck,sizes,hist', CENSUS, ids=[c[0] for c in CENSUS])
def test_read3_census(name, deck, sizes, hist):
    b = basis.build_basis(deck(), None)
    assert (b.npgs, b.ncgs, b.npshell) == sizes
    if hist is not None:
        ang = np.asarray(b.p_shell_ang)
        assert tuple(int((ang == l).sum()) for l in range(3)) == hist
