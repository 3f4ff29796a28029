"""The batched SCF on the GPU (DeviceBatch builds, batched DIIS and SP2).

* every molecule of a batch of uneven water clusters converges to the energy of
  its own plain FP64 GPU SCF (the reference's loop) within 1e-8 Eh, with
  incremental density-screened builds, in eager mode and with each iteration
  replayed from a CUDA graph (replays counted);
* the same with FP32 recursion below 1e-6 and the learned guess (purified in the
  batch): converged, within 1e-8 Eh.
"""
import numpy as np
import pytest
import torch

from polymer_b200 import batch_scf, fock, geometry, guess, scf, system

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def clusters():
    decks = [geometry.water_deck(k, seed=6100 + i) for i, k in enumerate((1, 3, 2, 3, 4, 1))]
    systems = [system.build_system(d, fock.onee) for d in decks]
    plain = []
    for s in systems:
        df = fock.DeviceFock(s)
        plain.append(scf.run_scf(s, df, device='cuda', variational=True).energy_variational)
        df.close()
    return systems, np.array(plain)


@pytest.mark.parametrize('graph', [False, True], ids=['eager', 'graph'])
def test_batched_scf_matches_plain(clusters, graph):
    systems, plain = clusters
    res = batch_scf.run_batch_scf(systems, batch_scf.BatchOptions(), graph=graph, profile=True)
    assert res.converged.all()
    assert np.abs(res.energy - plain).max() < 1e-8
    if graph:
        assert res.phases['graph_replays'] > 0


def test_batched_scf_learned_mixed(clusters):
    systems, plain = clusters
    lg = guess.LearnedGuess.load(guess.MODEL)
    res = batch_scf.run_batch_scf(systems, batch_scf.BatchOptions(guess=lg, mixed_cutoff=1e-6), graph=True)
    assert res.converged.all()
    assert np.abs(res.energy - plain).max() < 1e-8
