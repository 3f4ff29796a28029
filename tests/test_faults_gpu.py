"""Error paths of the set-up under injected device-allocation failures
(pfe_debug_fail_allocation: the n-th allocation a context or batch set-up asks
for is reported as out of memory without being attempted, so nothing reaches
the GPU).  For several positions of the failure:

* pfe_context_setup returns PFE_ENOMEM with the CUDA message, the context is
  left not set up (a build on it is refused with PFE_EINVAL), and the same
  context set up again builds J and K equal to those of a context that never
  failed;
* pfe_batch_setup (two molecules) returns PFE_ENOMEM, the batch refuses builds
  until a set-up succeeds, and its rebuilt batch equals the undisturbed one.
"""
import ctypes

import numpy as np
import pytest
import torch

from polymer_b200 import capi, fock, geometry, scf, system

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def waters():
    return [system.build_system(geometry.water_deck(k, seed=70 + k), fock.onee) for k in (2, 3)]


def _pc(sysm):
    return torch.tensor(scf.guess_density(sysm)[0], dtype=torch.float64, device='cuda')


def _build(L, h, sysm, pc):
    """J, K of context h from the contracted density pc through the C ABI."""
    n = sysm.basis.ncgs
    pcf = pc.t().contiguous()
    oc = torch.empty((n, n), dtype=torch.float64, device='cuda')
    ox = torch.empty_like(oc)
    s = torch.cuda.current_stream().cuda_stream
    rc = L.pfe_context_fock_pc(h, ctypes.c_void_p(pcf.data_ptr()), ctypes.c_void_p(oc.data_ptr()),
                               ctypes.c_void_p(ox.data_ptr()), ctypes.c_void_p(s))
    torch.cuda.synchronize()
    return rc, oc, ox


def _close(a, b, rel=1e-12):
    assert float((a - b).abs().max()) <= rel * max(float(b.abs().max()), 1e-300)


@pytest.mark.parametrize('after', [0, 2, 7, 15])
def test_context_setup_recovers_from_allocation_failure(waters, after):
    L = capi.lib()
    sysm = waters[0]
    pc = _pc(sysm)
    ref = fock.DeviceFock(sysm)
    c_ref, x_ref = ref.from_pc(pc)
    ref.close()
    h = ctypes.c_void_p()
    capi.check(L, L.pfe_context_create(0, ctypes.byref(h)))
    try:
        a, keep = sysm.pfe_args(None, None)
        L.pfe_debug_fail_allocation(after)
        rc = L.pfe_context_setup(h, ctypes.byref(a))
        L.pfe_debug_fail_allocation(-1)
        assert rc == -5, (rc, capi.last_error(L))
        assert 'out of memory' in capi.last_error(L)
        rc, _, _ = _build(L, h, sysm, pc)
        assert rc == -1 and 'not set up' in capi.last_error(L)
        capi.check(L, L.pfe_context_setup(h, ctypes.byref(a)))
        rc, oc, ox = _build(L, h, sysm, pc)
        assert rc == 0, capi.last_error(L)
        _close(oc.t(), c_ref)
        _close(ox.t(), x_ref)
    finally:
        L.pfe_debug_fail_allocation(-1)
        L.pfe_context_destroy(h)


@pytest.mark.parametrize('after', [1, 12])
def test_batch_setup_recovers_from_allocation_failure(waters, after):
    L = capi.lib()
    ref = fock.DeviceBatch(waters, 0)
    pc = torch.zeros_like(ref.p_c)
    for k, s in enumerate(waters):
        ref.view(pc, k).copy_(_pc(s))
    ref.run_packed(pc, ref.out_c, ref.out_x)
    torch.cuda.synchronize()
    c_ref, x_ref = ref.out_c.clone(), ref.out_x.clone()
    off = list(ref.off)
    ref.close()
    h = ctypes.c_void_p()
    capi.check(L, L.pfe_batch_create(0, ctypes.byref(h)))
    try:
        args, keep = [], []
        for s in waters:
            a, kp = s.pfe_args(None, None)
            args.append(a)
            keep.append(kp)
        arr = (capi.PfeArgs * len(args))(*args)
        L.pfe_debug_fail_allocation(after)
        rc = L.pfe_batch_setup(h, arr, len(args))
        L.pfe_debug_fail_allocation(-1)
        assert rc == -5, (rc, capi.last_error(L))
        assert 'out of memory' in capi.last_error(L)
        outc, outx = torch.empty_like(pc), torch.empty_like(pc)
        s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        rc = L.pfe_batch_fock_pc(h, ctypes.c_void_p(pc.data_ptr()), ctypes.c_void_p(outc.data_ptr()),
                                 ctypes.c_void_p(outx.data_ptr()), s)
        assert rc == -1
        capi.check(L, L.pfe_batch_setup(h, arr, len(args)))
        o = (ctypes.c_int64 * (len(args) + 1))()
        assert L.pfe_batch_offsets(h, o) == len(args) and list(o) == off
        capi.check(L, L.pfe_batch_fock_pc(h, ctypes.c_void_p(pc.data_ptr()), ctypes.c_void_p(outc.data_ptr()),
                                          ctypes.c_void_p(outx.data_ptr()), s))
        torch.cuda.synchronize()
        _close(outc, c_ref)
        _close(outx, x_ref)
    finally:
        L.pfe_debug_fail_allocation(-1)
        L.pfe_batch_destroy(h)
