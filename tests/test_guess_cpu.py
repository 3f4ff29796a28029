"""Frame machinery of the learned guess on the CPU (oracle SCF, no network):
the frame blocks of a converged water density do not depend on the water's
orientation, assembling them back gives the density, and FP64 purification
leaves a converged (idempotent) density unchanged; the monomial transforms
of a rotation are exact (on points and under composition), a cluster's frame
blocks assemble back to its density on every block the pairs cover, and the
frame transforms computed for all waters at once equal the per-water form;
the basis's shell groups (6-31G** with cumulative sp shells, cc-pVDZ) are
whole shell instances: one atom, one angular momentum, one radial part."""
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


def test_monomial_transforms_are_exact():
    # m_i(R u) = sum_j Q_ij m_j(u) at random points, and Q(R1 R2) = Q(R1) Q(R2)
    rng = np.random.default_rng(11)
    R1, R2 = _random_rotation(rng), _random_rotation(rng)
    u = rng.normal(size=(7, 3))
    for L in range(4):
        pws, q = guess.monomial_transforms(L, np.stack([R1, R2, R1 @ R2]))
        ev = lambda pts: np.stack([pts[:, 0] ** a * pts[:, 1] ** b * pts[:, 2] ** c for a, b, c in pws], axis=1)
        assert np.abs(ev(u @ R1.T) - ev(u) @ q[0].T).max() < 1e-13
        assert np.abs(q[2] - q[0] @ q[1]).max() < 1e-13


def test_assemble_inverts_the_frame_blocks_of_a_cluster():
    # any symmetric density of a three-water cluster: its frame blocks, assembled
    # back, give it on every (A, B) block the pair list covers and zero elsewhere
    from polymer_b200 import geometry
    s = system.build_system(geometry.water_deck(3, seed=41), oracle.onee)
    rng = np.random.default_rng(12)
    n = s.basis.ncgs
    a = rng.normal(size=(n, n))
    info, frames, pairs, x = guess.cluster_data(s)
    p = (a + a.T) * info.live[:, None] * info.live[None, :]
    t, w = guess.targets(s, info, frames, pairs, p)
    back = guess.assemble(s, info, frames, pairs, t)
    covered = np.zeros((n, n), dtype=bool)
    for i, j, _ in pairs:
        covered[np.ix_(info.atom_funcs[i], info.atom_funcs[j])] = True
    assert covered.any() and not covered.all()
    assert np.abs(back[covered] - p[covered]).max() < 1e-12 * np.abs(p).max()
    assert not back[~covered].any()


def test_batched_frame_transforms_match_the_per_water_form():
    from polymer_b200 import geometry
    s = system.build_system(geometry.water_deck(4, seed=43), oracle.onee)
    info, frames, pairs, x = guess.cluster_data(s)
    cache = {}
    u = guess.frame_transforms(info, frames, s.deck.natom, cache)
    for m, (_, R, atoms) in enumerate(frames):
        for a in atoms:
            ref = guess.frame_transform(info, R, info.atom_funcs[a])
            got = u[guess._layout(info, a, cache)][m]
            assert np.abs(got - ref).max() < 1e-14


@pytest.mark.parametrize('which', ['alkane_631gss', 'water_ccpvdz'])
def test_shell_groups_of_the_basis(which):
    # every live contracted function sits in exactly one group; a group is one
    # shell instance: one atom, one angular momentum, all its Cartesian
    # components (1, 3 or 6) with the same radial part, in function order
    from polymer_b200 import geometry
    deck = geometry.alkane_deck(2) if which == 'alkane_631gss' else geometry.water_deck(2, seed=44)
    s = system.build_system(deck, oracle.onee)
    info = guess.ao_info(s)
    members = sorted(i for g in info.groups for i in g)
    assert members == list(np.nonzero(info.live)[0])
    firsts = [g[0] for g in info.groups]
    assert firsts == sorted(firsts)
    cc = s.basis.cc
    for g in info.groups:
        L = {sum(info.powers[i]) for i in g}
        assert len(L) == 1 and len(g) == {0: 1, 1: 3, 2: 6}[L.pop()]
        assert len({int(info.atom[i]) for i in g}) == 1
        assert len({info.powers[i] for i in g}) == len(g)
        zs = [tuple(sorted(np.round(s.basis.zt[np.nonzero(cc[i])[0]], 10))) for i in g]
        assert len(set(zs)) == 1
    for a, funcs in enumerate(info.atom_funcs):
        assert all(info.atom[i] == a and info.live[i] for i in funcs)
