"""The JOBNAME.chk checkpoint format (polymer_b200/chk.py), the interchange of
STORE_DENSITYMATRIX / RESTORE_DENSITYMATRIX / DIIS (src/pdensitymatrix.f90).

* blocks written as STORE writes them read back bit for bit, and the Pulay
  products STORE forms from the file are the products of the stored changes;
* records in other list-directed forms (D exponents, commas, repeat counts, the
  header with fewer fields read by DIIS) parse to the same numbers;
* RESTORE semantics: the last block wins, P_C is zeroed once (cells a block
  lacks keep an earlier block's values), cells outside CEL1 are skipped, an
  NCGS mismatch or an empty/missing file gives the guess;
* the SCF mirror writes one block per iteration, and a second run restored
  from that file starts at the converged density: it converges at once to the
  same energy.
"""
import os

import numpy as np
import pytest

import oracle
from conftest import deck_of
from polymer_b200 import chk, scf, system


def _sym(rng, ncell, n):
    a = rng.normal(size=(ncell, n, n))
    return a + a.transpose(0, 2, 1)


def test_blocks_round_trip_and_pulay(tmp_path):
    rng = np.random.default_rng(5)
    path = str(tmp_path / 'job.chk')
    cel1, n = (1, 0, 0), 4
    ins = [_sym(rng, 3, n) for _ in range(3)]
    outs = [_sym(rng, 3, n) for _ in range(3)]
    for i in range(3):
        row = chk.store(path, i + 1, ins[i], outs[i], cel1)
        d = [outs[j] - ins[j] for j in range(i + 1)]
        assert np.allclose(row, [float((d[j] * d[i]).sum()) for j in range(i + 1)], rtol=1e-14, atol=0)
    blocks = chk.read_blocks(path)
    assert len(blocks) == 3
    for i, (hdr, pc, dp) in enumerate(blocks):
        assert hdr == (n,) + cel1
        assert np.array_equal(pc, ins[i])
        assert np.array_equal(dp, outs[i] - ins[i])
    # storing iteration 2 again drops block 3
    chk.store(path, 2, ins[0], outs[0], cel1)
    assert len(chk.read_blocks(path)) == 2


def test_list_directed_forms(tmp_path):
    path = str(tmp_path / 'f.chk')
    # element order (J, I), J fastest: P(1,1), P(2,1), P(1,2), P(2,2)
    text = ('           2           0           0           0\n'
            '   1.0000000000000000       -2.5000000000000000E-002\n'
            '  0.50000000000000000D+00,  0.0\n'
            '   0.5,0.0\n'
            '   1*2.0000000000000000        1.0D-003\n')
    with open(path, 'w') as fh:
        fh.write(text)
    (hdr, pc, dp), = chk.read_blocks(path)
    assert hdr == (2, 0, 0, 0)
    assert np.array_equal(pc[0], np.array([[1.0, 0.5], [0.5, 2.0]]))
    assert np.array_equal(dp[0], np.array([[-0.025, 0.0], [0.0, 1e-3]]))


def test_restore_semantics(tmp_path):
    rng = np.random.default_rng(6)
    path = str(tmp_path / 'r.chk')
    n = 3
    p_wide = _sym(rng, 5, n)           # CEL1X = 2
    p_narrow = _sym(rng, 1, n)         # CEL1X = 0, written later
    chk.store(path, 1, p_wide, p_wide, (2, 0, 0))
    with open(path, 'a') as fh:
        fh.write(chk.format_block(p_narrow, 0 * p_narrow, (0, 0, 0)))
    p, msg = chk.restore(path, n, (1, 0, 0))
    assert 'RESTORED' in msg
    assert np.array_equal(p[1], p_narrow[0])            # cell 0: the last block
    assert np.array_equal(p[0], p_wide[1])              # cell -1: kept from the first block
    assert np.array_equal(p[2], p_wide[3])              # cell +1
    assert chk.restore(path, n + 1, (1, 0, 0))[0] is None        # incompatible NCGS
    assert chk.restore(str(tmp_path / 'none.chk'), n, (0, 0, 0))[0] is None
    open(str(tmp_path / 'empty.chk'), 'w').close()
    assert chk.restore(str(tmp_path / 'empty.chk'), n, (0, 0, 0))[0] is None


@pytest.fixture(scope='module')
def bh(reference_runs):
    return system.build_system(deck_of(reference_runs['BH_MBGF']), oracle.onee)


def test_scf_writes_and_resumes_from_chk(bh, tmp_path):
    path = str(tmp_path / 'bh.chk')
    f = oracle.fock_builder(bh)
    first = scf.run_scf(bh, lambda pp, ph=None: f(pp, ph), chk=path)
    assert first.converged
    blocks = chk.read_blocks(path)
    assert len(blocks) == len(first.iterations)
    # block 1 holds the nuclear-charge guess the first run started from
    assert np.array_equal(blocks[0][1], scf.guess_density(bh))
    msgs = []
    second = scf.run_scf(bh, lambda pp, ph=None: f(pp, ph), chk=path, log=msgs.append)
    assert any('RESTORED' in m for m in msgs)
    assert second.converged
    assert len(second.iterations) <= 3 < len(first.iterations)
    assert abs(second.energy - first.energy) < 1e-9
    assert os.path.getsize(path) > 0


def test_guess_file_restores_the_guess(tmp_path):
    rng = np.random.default_rng(8)
    p = _sym(rng, 1, 5)
    path = str(tmp_path / 'g.chk')
    chk.write_guess(path, p, (0, 0, 0))
    got, _ = chk.restore(path, 5, (0, 0, 0))
    assert np.array_equal(got, p)
