"""Batched molecular Fock builds (pfe_batch_*): one launch per quartet class
over the work of every molecule in the batch.

* each molecule's C_C/X_C from the batched build equals its own
  pfe_context_fock_pc build to 1e-11 of max|C_C| (only the order of the FP64
  atomics differs), for water clusters of several sizes in cc-pVDZ, alkanes in
  6-31G** and a batch that mixes both;
* a second build from another packed buffer (the per-molecule launch records
  are rebuilt for the new pointer) and screening set on the whole batch match
  the per-molecule builds the same way;
* the census of a batch sums its molecules' quartets while the class launches
  do not grow with the number of molecules;
* after the batch autotuner has timed every variant of every class, builds
  still match the per-molecule ones.
"""
import numpy as np
import pytest
import torch

import oracle
from polymer_b200 import fock, geometry, system

pytestmark = pytest.mark.gpu

RTOL = 1e-11


def _sys(deck):
    return system.build_system(deck, oracle.onee)


def _pc(sysm, seed, scale=0.1):
    rng = np.random.default_rng(seed)
    n = sysm.basis.ncgs
    a = rng.normal(size=(n, n)) * scale
    return a + a.T


def _close(got, ref, what, rtol=RTOL):
    scale = float(np.abs(ref).max())
    err = float(np.abs(got - ref).max())
    assert err <= rtol * scale + 1e-13, '%s: max|diff| %.3e (scale %.3e)' % (what, err, scale)


def _singles(systems, pcs, **screen):
    out = []
    for s, pc in zip(systems, pcs):
        df = fock.DeviceFock(s)
        if screen:
            df.set_screening(**screen)
        c, x = df.from_pc(torch.tensor(pc, device='cuda'))
        out.append((c.cpu().numpy(), x.cpu().numpy()))
        df.close()
    return out


def _check(batch_out, single_out, tag, rtol=RTOL):
    assert len(batch_out) == len(single_out)
    for k, ((cb, xb), (cs, xs)) in enumerate(zip(batch_out, single_out)):
        _close(cb.cpu().numpy(), cs, '%s[%d] C_C' % (tag, k), rtol)
        _close(xb.cpu().numpy(), xs, '%s[%d] X_C' % (tag, k), rtol)


DECKS = {
    'water_ccpvdz': lambda: [geometry.water_deck(k, seed=3000 + k) for k in (1, 2, 3, 5)],
    'alkane_631gss': lambda: [geometry.alkane_deck(n) for n in (1, 2, 4)],
    'mixed': lambda: [geometry.water_deck(2, seed=3100), geometry.alkane_deck(3), geometry.water_deck(1, seed=3101)],
}


@pytest.mark.parametrize('name', list(DECKS))
def test_batch_matches_single_builds(name):
    systems = [_sys(d) for d in DECKS[name]()]
    pcs = [_pc(s, 10 + k) for k, s in enumerate(systems)]
    ref = _singles(systems, pcs)
    b = fock.DeviceBatch(systems)
    got = b([torch.tensor(pc, device='cuda') for pc in pcs])
    torch.cuda.synchronize()
    _check(got, ref, name)
    # a second density in a different packed buffer
    pcs2 = [_pc(s, 50 + k, scale=0.05) for k, s in enumerate(systems)]
    packed = torch.zeros_like(b.p_c)
    for k, pc in enumerate(pcs2):
        b.view(packed, k).copy_(torch.tensor(pc, device='cuda'))
    oc, ox = torch.empty_like(packed), torch.empty_like(packed)
    b.run_packed(packed, oc, ox)
    torch.cuda.synchronize()
    got2 = [(b.view(oc, k), b.view(ox, k)) for k in range(len(b))]
    _check(got2, _singles(systems, pcs2), name + '/second')
    b.close()


def test_batch_screening_matches_single_builds():
    systems = [_sys(geometry.water_deck(k, seed=3200 + k)) for k in (2, 4)]
    pcs = [_pc(s, 70 + k, scale=1e-4) for k, s in enumerate(systems)]
    screen = dict(mixed_cutoff=1e-6, density_tol=1e-11)
    ref = _singles(systems, pcs, **screen)
    b = fock.DeviceBatch(systems)
    b.set_screening(**screen)
    got = b([torch.tensor(pc, device='cuda') for pc in pcs])
    torch.cuda.synchronize()
    _check(got, ref, 'screened', rtol=1e-10)
    b.close()


def test_batch_census():
    systems = [_sys(geometry.water_deck(k, seed=3300 + k)) for k in (1, 2, 3)]
    singles = []
    for s in systems:
        df = fock.DeviceFock(s)
        singles.append(df.census())
        df.close()
    b = fock.DeviceBatch(systems)
    c = b.census()
    assert c['quartets'] == pytest.approx(sum(x['quartets'] for x in singles), rel=1e-12)
    assert c['flops'] == pytest.approx(sum(x['flops'] for x in singles), rel=1e-12)
    assert c['pairs'] == sum(x['pairs'] for x in singles)
    assert c['kernel_launches'] <= max(x['kernel_launches'] for x in singles)
    b.close()


def test_batch_autotune_keeps_results():
    systems = [_sys(geometry.water_deck(k, seed=3400 + k)) for k in (2, 3)]
    pcs = [_pc(s, 90 + k) for k, s in enumerate(systems)]
    ref = _singles(systems, pcs)
    b = fock.DeviceBatch(systems)
    for k, pc in enumerate(pcs):
        b.view(b.p_c, k).copy_(torch.tensor(pc, device='cuda'))
    b.autotune(b.p_c)
    sched = b.schedule()
    assert sched and all(max(x['tuned_ms']) > 0.0 for x in sched)
    got = b([torch.tensor(pc, device='cuda') for pc in pcs])
    torch.cuda.synchronize()
    _check(got, ref, 'autotuned')
    b.close()
