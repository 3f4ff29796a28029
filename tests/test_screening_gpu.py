"""Builds from the contracted density, the decontraction check, and the
density-screened / mixed-precision builds of the molecular path.

* pfe_context_fock_pc(P_C) equals pfe_context_fock(CC^T P_C CC) for contracted
  targets, in 6-31G** and in cc-pVDZ (whose shared primitives READ3 copies
  once per contracted function);
* a P_P that is not a decontracted density is refused by the device path,
  handled (primitive targets) by the host path, to the oracle's tolerance;
* the FP32 recursion (PFE_PREC_MIXED) stays within 1e-10 * max|C_C| of the
  FP64 build at a cutoff of 1e-6 and runs a share of the quartets in FP32;
* density screening with tolerance t changes C_C/X_C by at most 1e-7 per 1e-10
  of t (about 1000 skipped contributions of size t per element at most) and is
  exact at t = 0 (to the order of the FP64 atomics); an incremental build
  J(P) = J(P0) + J(P - P0) from a dense random difference of 1e-5 with t = 1e-11
  and FP32 below 1e-6 agrees with the full build to 5e-8.
"""
import numpy as np
import pytest
import torch

import oracle
from polymer_b200 import capi, fock, geometry, scf, system

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


@pytest.mark.parametrize('deck', [lambda: geometry.alkane_deck(3), lambda: geometry.water_deck(2, seed=2001)],
                         ids=['c3h8_631gss', 'h2o2_ccpvdz'])
def test_fock_from_pc_matches_fock_from_pp(deck):
    s = _sys(deck())
    pc = _pc(s, 1)
    pp = s.basis.cc.T @ pc @ s.basis.cc
    df = fock.DeviceFock(s)
    c1, x1 = df(torch.tensor(pp[None], device='cuda'))
    c2, x2 = df.from_pc(torch.tensor(pc, device='cuda'))
    torch.cuda.synchronize()
    _close(c2.cpu().numpy(), c1.cpu().numpy(), 'C_C')
    _close(x2.cpu().numpy(), x1.cpu().numpy(), 'X_C')
    df.close()


def test_density_that_is_not_decontracted():
    s = _sys(geometry.alkane_deck(2, inttol=1e-12))
    rng = np.random.default_rng(9)
    n = s.basis.npgs
    a = rng.normal(size=(n, n)) * 0.1
    live = np.any(s.basis.cc != 0.0, axis=0)          # primitives with a coefficient
    pp = (a + a.T) * np.outer(live, live)
    # host path: falls back to primitive targets and matches the oracle
    c_ref, x_ref = oracle.fourindex_eri(s, pp[None])
    c_h, x_h = fock.fourindex_eri(s, pp[None])
    _close(c_h, c_ref, 'C_C host')
    _close(x_h, x_ref, 'X_C host')
    # device path with contracted targets refuses it ...
    df = fock.DeviceFock(s)
    with pytest.raises(capi.FockError) as e:
        df(torch.tensor(pp[None], device='cuda'))
    assert e.value.code == -1 and 'decontraction' in str(e.value)
    df.close()
    # ... and a context set up with primitive targets computes it
    dp = fock.DeviceFock(s, primitive_targets=True)
    c_d, x_d = dp(torch.tensor(pp[None], device='cuda'))
    torch.cuda.synchronize()
    _close(c_d.cpu().numpy(), c_ref, 'C_C primitive targets')
    _close(x_d.cpu().numpy(), x_ref, 'X_C primitive targets')
    dp.close()


@pytest.fixture(scope='module')
def c6():
    s = system.build_system(geometry.alkane_deck(6), fock.onee)
    df = fock.DeviceFock(s)
    r = scf.run_scf(s, df, device='cuda', max_cycles=4, raise_on_fail=False)   # a realistic density
    yield s, df, r.p_c[0].contiguous()
    df.close()


def test_mixed_precision_error_bound(c6):
    s, df, pc = c6
    df.set_screening()
    c0, x0 = df.from_pc(pc)
    df.set_screening(mixed_cutoff=1e-6)
    c1, x1 = df.from_pc(pc)
    torch.cuda.synchronize()
    cen = df.census()
    df.set_screening()
    assert 0.1 * cen['quartets'] < cen['quartets_fp32'] < cen['quartets']
    for a, b, w in ((c1, c0, 'C_C'), (x1, x0, 'X_C')):
        err = float((a - b).abs().max())
        assert err <= 1e-10 * float(b.abs().max()), '%s mixed: %.3e' % (w, err)
    assert float((c1 - c0).abs().max()) > 0.0     # the FP32 path did run


@pytest.mark.parametrize('dtol', [0.0, 1e-12, 1e-10])
def test_density_screening_error_bound(c6, dtol):
    s, df, pc = c6
    df.set_screening()
    c0, x0 = df.from_pc(pc)
    df.set_screening(density_tol=dtol)
    c1, x1 = df.from_pc(pc)
    torch.cuda.synchronize()
    df.set_screening()
    bound = max(1e-7 * dtol / 1e-10, 1e-12)   # dtol = 0: FP64 atomics in another order only
    for a, b, w in ((c1, c0, 'C_C'), (x1, x0, 'X_C')):
        err = float((a - b).abs().max())
        assert err <= bound, '%s dtol %g: %.3e' % (w, dtol, err)


def test_incremental_build_matches_full_build(c6):
    s, df, pc = c6
    torch.manual_seed(3)
    d = 1e-5 * torch.randn_like(pc)
    pc2 = pc + 0.5 * (d + d.T)
    df.set_screening()
    c0, x0 = df.from_pc(pc)
    cf, xf = df.from_pc(pc2)
    df.set_screening(mixed_cutoff=1e-6, density_tol=1e-11)
    cd, xd = df.from_pc(pc2 - pc)
    torch.cuda.synchronize()
    df.set_screening()
    assert float((c0 + cd - cf).abs().max()) <= 5e-8
    assert float((x0 + xd - xf).abs().max()) <= 5e-8
