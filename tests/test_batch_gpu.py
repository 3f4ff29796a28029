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
  still match the per-molecule ones;
* a set-up refused for one instance leaves no half-built batch: later calls
  answer that the batch is not set up, and the handle can be set up again.
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


def test_failed_setup_leaves_no_batch():
    """A set-up refused for one instance (an f shell) frees every instance: later
    calls on the handle answer that the batch is not set up, and a good set-up on
    the same handle builds as the per-molecule context does."""
    import ctypes
    from polymer_b200 import basis, capi
    lib = {k: list(v) for k, v in basis.load_basis_library('cc-pVDZ').items()}
    lib['O'] = lib['O'] + [['F', 1.0, [[1.428, 1.0]]]]
    good = _sys(geometry.water_deck(1, seed=3500))
    def zero_onee(sysm):   # the one-electron integrals play no part in the refusal
        z = np.zeros((sysm.ncell1, sysm.basis.npgs, sysm.basis.npgs))
        return z, z.copy(), z.copy()

    bad = system.build_system(geometry.water_deck(1, seed=3501), zero_onee, library=lib)
    L = capi.lib()
    h = ctypes.c_void_p()
    capi.check(L, L.pfe_batch_create(0, ctypes.byref(h)))
    try:
        args = [s.pfe_args(None, None) for s in (good, bad)]
        arr = (capi.PfeArgs * 2)(*[a for a, _ in args])
        assert L.pfe_batch_setup(h, arr, 2) == -3                      # PFE_EUNSUPPORTED
        n = good.basis.ncgs
        buf = torch.zeros(4 * n * n, dtype=torch.float64, device='cuda')
        p = ctypes.c_void_p(buf.data_ptr())
        assert L.pfe_batch_fock_pc(h, p, p, p, None) == -1             # PFE_EINVAL
        assert 'not set up' in capi.last_error(L)
        off = (ctypes.c_int64 * 3)()
        assert L.pfe_batch_offsets(h, off) == 0
        c = capi.PfeCensus()
        capi.check(L, L.pfe_batch_census(h, ctypes.byref(c)))
        assert c.kernel_launches == 0 and c.quartets == 0
        # the same handle, set up again with the good molecule alone
        arr1 = (capi.PfeArgs * 1)(args[0][0])
        capi.check(L, L.pfe_batch_setup(h, arr1, 1))
        assert L.pfe_batch_offsets(h, off) == 1 and off[1] == n * n
        pc = _pc(good, 11)
        dp = torch.tensor(pc.T.copy(), device='cuda').reshape(-1)
        oc, ox = torch.empty_like(dp), torch.empty_like(dp)
        capi.check(L, L.pfe_batch_fock_pc(h, ctypes.c_void_p(dp.data_ptr()), ctypes.c_void_p(oc.data_ptr()),
                                          ctypes.c_void_p(ox.data_ptr()), None))
        torch.cuda.synchronize()
        (cs, xs), = _singles([good], [pc])
        _close(oc.reshape(n, n).T.cpu().numpy(), cs, 'reset C_C')
        _close(ox.reshape(n, n).T.cpu().numpy(), xs, 'reset X_C')
    finally:
        L.pfe_batch_destroy(h)
