"""Frame machinery of the learned guess on the CPU (oracle SCF, no network):
the frame blocks of a converged water density do not depend on the water's
orientation, assembling them back gives the density, and FP64 purification
leaves a converged (idempotent) density unchanged."""
import numpy as np
import pytest
import torch

import oracle
from polymer_b200 import guess, inputdeck, scf, system
from polymer_b200.geometry import _WATER, _random_rotation


def _water(rot, shift):
    xyz = np.array([rot @ p for p in _WATER]) + shift
    s = system.build_system(inputdeck.make_deck([8, 1, 1], xyz, 'cc-pVDZ', inttol=1e-12), oracle.onee)
    r = scf.run_scf(s, oracle.fock_builder(s), scfconv=1e-9)
    info, frames, pairs, x, t, w = guess.cluster_data(s, r.p_c[0].numpy())
    return s, info, frames, pairs, x, t, r


def test_frame_blocks_are_orientation_independent():
    a = _water(np.eye(3), np.zeros(3))
    b = _water(_random_rotation(np.random.default_rng(5)), np.array([0.3, -0.2, 0.1]))
    assert np.abs(a[5] - b[5]).max() < 1e-7 * np.abs(a[5]).max()
    assert np.abs(a[4] - b[4]).max() < 1e-12          # features too
    s, info, frames, pairs, x, t, r = b
    back = guess.assemble(s, info, frames, pairs, t)
    assert np.abs(back - r.p_c[0].numpy()).max() < 1e-12
    pp = guess.purify(scf.HostState(s), torch.tensor(back), s.deck.nelectrons // 2)
    assert float((pp - r.p_c[0]).abs().max()) < 1e-7
